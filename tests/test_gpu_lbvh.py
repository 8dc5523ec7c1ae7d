"""Scenes whose BVH is built on the device (SOL_GPU_SCENE_GPU_BVH, linear BVH).

The hierarchy differs from the host build, but a closest hit is the same
triangle at the same distance unless two triangles are hit at exactly the same
distance (a ray through a shared edge), so hit ids, distances and renders must
match the CPU checker as closely as with the host-built hierarchy."""
import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity, random_rays

pytestmark = pytest.mark.gpu


def _trace(gs, rays, any_hit):
    import torch
    r = torch.from_numpy(rays).cuda()
    hits = torch.zeros((rays.shape[0], 4), dtype=torch.float32, device="cuda")
    gs.trace(r.data_ptr(), rays.shape[0], any_hit, hits.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return hits.cpu().numpy()


@pytest.mark.parametrize("kind", ["cornell", "spheres"])
def test_gpu_built_hits_match(built, kind):
    from sol_b200 import scenes
    from sol_b200.renderer import GpuScene
    if kind == "cornell":
        scene = scenes.cornell_box(0)
        rays = random_rays(1 << 16, (0.05, 0.05, 0.05), (0.95, 0.95, 0.95), seed=1)
    else:
        scene = scenes.sphere_field(16, seed=3, bands=33, segments=64)
        rays = random_rays(1 << 18, (0, 0.2, 0), (10, 10, 10), seed=2)
    gs = GpuScene(scene, gpu_bvh=True)
    info = gs.info()
    assert 0 < info.bvh_depth <= 64 and info.num_triangles == scene.num_triangles
    g = _trace(gs, rays, False)
    o = oracle.trace(scene, rays, False)
    gid, oid = g[:, 0].view(np.int32), o[:, 0].view(np.int32)
    u, v = o[:, 2], o[:, 3]
    ok = ~((oid >= 0) & (np.minimum(np.minimum(u, v), 1 - u - v) < 1e-6))
    assert np.mean(oid >= 0) > 0.3
    assert np.array_equal(gid[ok], oid[ok])
    hit = ok & (oid >= 0)
    assert np.array_equal(g[hit, 1], o[hit, 1])
    a = _trace(gs, rays, True)
    assert np.array_equal(a[ok, 0].view(np.int32) >= 0, oid[ok] >= 0)


@pytest.mark.parametrize("kind", ["cornell", "spheres"])
def test_gpu_built_render_matches_oracle(built, kind):
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene, Image
    if kind == "cornell":
        scene, cfg, w, h, spp = scenes.cornell_box(0, textured=True, tex_size=32), scenes.CORNELL_CONFIG, 64, 48, 4
    else:
        scene, cfg, w, h, spp = scenes.sphere_field(8, seed=5, bands=33, segments=64), scenes.SPHERES_CONFIG, 96, 54, 4
    img = Image(w, h)
    GpuPathTracer(GpuScene(scene, gpu_bvh=True), cfg).render(img, 5, spp)
    o = oracle.render(scene, cfg, w, h, spp, sample_index=5)
    exact, bad = per_pixel_parity(img.channels, o)
    assert bad == 0 and exact >= 0.99


def test_gpu_build_of_a_million_triangles(built):
    """The benchmark scene (1,048,586 triangles): device build (the faster of two,
    so that one-time start-up costs do not count) in less time than the host
    build, a usable depth, an SAH cost within 10 % of the host build's (treelet
    restructuring), and a frame that matches the host-built scene's on nearly
    every pixel."""
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene
    scene, cfg = scenes.sphere_field(64, seed=1), scenes.SPHERES_CONFIG
    host, dev = GpuScene(scene), GpuScene(scene, gpu_bvh=True)
    hi, di = host.info(), dev.info()
    dev_ms = min(di.build_ms, GpuScene(scene, gpu_bvh=True).info().build_ms)
    assert di.num_triangles == hi.num_triangles == scene.num_triangles
    assert 0 < di.bvh_depth <= 64
    assert dev_ms < hi.build_ms
    assert 0 < di.sah_cost <= 1.1 * hi.sah_cost
    films = []
    for gs in (host, dev):
        f = torch.zeros((3, 90, 160), device="cuda")
        GpuPathTracer(gs, cfg).render_device(f.data_ptr(), 160, 90, 0, 4, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        films.append(f.cpu().numpy())
    exact, bad = per_pixel_parity(films[1], films[0])
    assert bad == 0 and exact >= 0.99
    print(f"host build {hi.build_ms:.0f} ms, device build {dev_ms:.0f} ms, depth {hi.bvh_depth} / {di.bvh_depth}, "
          f"SAH {hi.sah_cost:.3f} / {di.sah_cost:.3f}")
