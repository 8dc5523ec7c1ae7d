"""Host-side checks of the C ABI: the library loads, exports every entry point
of include/sol_gpu.h, rejects invalid scenes before touching the GPU, and
builds well-formed BVHs."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from sol_b200 import scenes
from sol_b200.scene import Bsdf, Light, Texture, build_bvh

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "sol_gpu.h").read_text()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(sol_gpu_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_header_function(built):
    from sol_b200 import capi
    names = header_functions()
    assert len(names) >= 12
    bound = {n for n, _, _ in capi.SIGNATURES}
    for n in names:
        assert hasattr(capi.lib, n), n
        assert n in bound, n


def test_abi_version(built):
    from sol_b200 import capi
    assert capi.lib.sol_gpu_abi_version() == 3


def _create(scene):
    from sol_b200 import capi
    d = scene.desc()
    h = capi.ScenePtr()
    return capi.lib.sol_gpu_scene_create(d.ptr, 0, C.byref(h)), capi.lib.sol_gpu_last_error().decode()


@pytest.mark.parametrize("mutate,msg", [
    (lambda s: s.indices.__setitem__((0, 0), 10**6), "vertex index out of range"),
    (lambda s: s.tri_bsdf.__setitem__(0, 99), "BSDF out of range"),
    (lambda s: s.tri_light.__setitem__(0, 99), "light out of range"),
    (lambda s: s.bsdfs.__setitem__(0, Bsdf(0, (6, -1, -1))), "colour texture"),
    (lambda s: s.bsdfs.append(Bsdf(4, (6, -1, -1), a=99, b=0)), "interp"),
    (lambda s: s.bsdfs.append(Bsdf(9, (0, -1, -1))), "bad BSDF type"),
    (lambda s: s.textures.append(Texture(2, image=5)), "image out of range"),
    (lambda s: s.lights.append(Light(1, intensity_tex=6)), "colour texture"),
    (lambda s: s.lights.append(Light(7)), "bad light type"),
])
def test_invalid_scenes_are_rejected_on_the_host(built, mutate, msg):
    from sol_b200 import capi
    s = scenes.cornell_box(0)
    mutate(s)
    rc, err = _create(s)
    assert rc == capi.ERR_INVALID_ARG
    assert msg in err


def test_nested_interp_is_rejected(built):
    from sol_b200 import capi
    s = scenes.cornell_box(0)
    s.textures.append(Texture(0, (0.5, 0, 0)))
    k = len(s.textures) - 1
    s.bsdfs.append(Bsdf(4, (k, -1, -1), a=0, b=5))
    s.bsdfs.append(Bsdf(4, (k, -1, -1), a=len(s.bsdfs) - 1, b=0))
    rc, err = _create(s)
    assert rc == capi.ERR_INVALID_ARG and "nested" in err


def _check_bvh(nodes, count, prims, nt):
    seen = np.zeros(nt, np.int32)
    stack = [0]
    depth = {0: 1}
    while stack:
        i = stack.pop()
        n = nodes[i]
        if n.count == 0:
            for c in (n.first, n.first + 1):
                ch = nodes[c]
                for k in range(3):
                    assert n.lo[k] <= ch.lo[k] and ch.hi[k] <= n.hi[k]
                depth[c] = depth[i] + 1
                stack.append(c)
        else:
            assert 1 <= n.count <= 8
            seen[prims[n.first:n.first + n.count]] += 1
    assert np.all(seen == 1)
    assert max(depth.values()) <= 64
    assert count <= 2 * nt - 1


def test_build_bvh_cornell(built):
    s = scenes.cornell_box(0)
    nodes, count, prims = build_bvh(s)
    _check_bvh(nodes, count, prims, s.num_triangles)


def test_build_bvh_spheres_deterministic(built):
    s = scenes.sphere_field(6, seed=2, bands=17, segments=32)
    a = build_bvh(s)
    b = build_bvh(s)
    _check_bvh(*a, s.num_triangles)
    assert a[1] == b[1] and np.array_equal(a[2], b[2])
    assert bytes(a[0])[: a[1] * C.sizeof(a[0]._type_)] == bytes(b[0])[: b[1] * C.sizeof(b[0]._type_)]


def test_uv_sphere_has_16384_triangles():
    v, t, uv = scenes.uv_sphere(65, 128)
    assert t.shape == (16384, 3)
    a = np.linalg.norm(np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]]), axis=1)
    assert np.all(a > 0)
