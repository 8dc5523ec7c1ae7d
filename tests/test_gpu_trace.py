"""Batched closest-hit / any-hit queries (the device side of TriangleMesh::intersect_closest
and intersect_any) against the CPU checker's own BVH: triangle ids are bit-exact
except for rays within 1e-6 (barycentric) of a triangle edge, where either
neighbour is a valid answer."""
import numpy as np
import pytest

import oracle
from helpers import random_rays

pytestmark = pytest.mark.gpu


def gpu_trace(scene, rays, any_hit):
    import torch
    from sol_b200.renderer import GpuScene
    gs = GpuScene(scene)
    r = torch.from_numpy(rays).cuda()
    hits = torch.zeros((rays.shape[0], 4), dtype=torch.float32, device="cuda")
    gs.trace(r.data_ptr(), rays.shape[0], any_hit, hits.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return hits.cpu().numpy()


@pytest.mark.parametrize("kind", ["cornell", "spheres"])
def test_closest_hit_ids_match(built, kind):
    from sol_b200 import scenes
    if kind == "cornell":
        scene = scenes.cornell_box(0)
        rays = random_rays(1 << 16, (0.05, 0.05, 0.05), (0.95, 0.95, 0.95), seed=1)
    else:
        scene = scenes.sphere_field(16, seed=3, bands=33, segments=64)
        rays = random_rays(1 << 18, (0, 0.2, 0), (10, 10, 10), seed=2)
    g = gpu_trace(scene, rays, False)
    o = oracle.trace(scene, rays, False)
    gid, oid = g[:, 0].view(np.int32), o[:, 0].view(np.int32)
    u, v = o[:, 2], o[:, 3]
    near_edge = (oid >= 0) & (np.minimum(np.minimum(u, v), 1 - u - v) < 1e-6)
    ok = ~near_edge
    assert np.mean(oid >= 0) > 0.3
    assert np.array_equal(gid[ok], oid[ok])
    hit = ok & (oid >= 0)
    assert np.array_equal(g[hit, 1], o[hit, 1])                     # same t, bit for bit
    assert np.array_equal(g[hit, 2:4], o[hit, 2:4])


def test_any_hit_agrees(built):
    from sol_b200 import scenes
    scene = scenes.sphere_field(16, seed=3, bands=33, segments=64)
    rays = random_rays(1 << 16, (0, 0.2, 0), (10, 10, 10), seed=4)
    rays[:, 7] = 2.0          # short segments
    g = gpu_trace(scene, rays, True)
    o = oracle.trace(scene, rays, True)
    closest = oracle.trace(scene, rays, False)
    cu, cv = closest[:, 2], closest[:, 3]
    cid = closest[:, 0].view(np.int32)
    near_edge = (cid >= 0) & (np.minimum(np.minimum(cu, cv), 1 - cu - cv) < 1e-6)
    assert np.array_equal((g[~near_edge, 0].view(np.int32) >= 0), (o[~near_edge, 0].view(np.int32) >= 0))


def test_no_geometry_misses(built):
    from sol_b200 import scenes
    from sol_b200.scene import Scene
    s = scenes.cornell_box(0)
    empty = Scene(vertices=np.zeros((0, 3), np.float32), normals=np.zeros((0, 3), np.float32),
                  tex_coords=np.zeros((0, 2), np.float32), indices=np.zeros((0, 3), np.uint32),
                  tri_bsdf=np.zeros(0, np.int32), tri_light=np.zeros(0, np.int32), textures=s.textures,
                  bsdfs=s.bsdfs, lights=s.lights, camera=s.camera)
    rays = random_rays(1000, (0, 0, 0), (1, 1, 1))
    g = gpu_trace(empty, rays, False)
    assert np.all(g[:, 0].view(np.int32) == -1)
