"""Scene files (TOML + OBJ/MTL) into a Scene, against SoL's own loader.

Where SoL's sources are built (oracle/_ref), each of SoL's four test scenes is
loaded by sol::Scene::load (src/scene_loader.cpp, src/formats/obj.cpp, over the
TOML subset reader in oracle/shim) and by sol_b200.loader; both scenes are
rendered by SoL's PathTracer and must give the same film bit for bit, with the
same light, BSDF and texture tables.  Small files written here cover the format
cases the test scenes do not use."""
import numpy as np
import pytest

import oracle
from sol_b200 import capi, loader
from sol_b200.scene import Config

CFG = Config(max_path_len=16, min_rr_path_len=3, min_survival_prob=0.05, max_survival_prob=0.75, ray_offset=1e-5)


@pytest.mark.parametrize("name", oracle.REFERENCE_SCENES)
def test_matches_sol_loader_on_sol_test_scenes(built, name):
    path = oracle.reference_scene(name)
    if path is None or not oracle.ref_available():
        pytest.skip("SoL's sources and test scenes are not present here")
    sol = oracle.RefScene.load(str(path), 1.5)
    ours = loader.load_scene(str(path), 1.5)
    c = sol.counts()
    assert (c["lights"], c["bsdfs"], c["textures"]) == (len(ours.lights), len(ours.bsdfs), len(ours.textures))
    a, _ = sol.render(CFG, 48, 32, 4, sample_index=7)
    b, _ = oracle.RefScene(ours).render(CFG, 48, 32, 4, sample_index=7)
    assert np.array_equal(a, b)
    assert float(a.mean()) > 0.01


OBJ = """# two quads, a triangle with negative indices, a pentagon, an unknown material
mtllib mats.mtl
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
vt 0 0
vt 1 0
vt 1 1
vn 0 0 1
usemtl mix
f 1/1/1 2/2/1 3/3/1 4/1/1
usemtl glass
f -4 -3 -2
usemtl lamp
f 1//1 2//1 3//1 4//1
usemtl nowhere
f 1 2 3
v 2 0 0
v 3 0 0
v 3 1 0
v 2.5 2 0
v 2 1 0
usemtl mirror
f 5 6 7 8 9
f 1 2
"""

MTL = """newmtl mix
Kd 0.5 0.25 0.125
Ks 0.1 0.2 -0.3
Ns 32
newmtl glass
illum 7
Ks 1 1 1
Tf 0.9 0.9 0.9
Ni 1.5
newmtl lamp
Kd 0.8 0.8 0.8
Ke 10 5 2
newmtl mirror
illum 5
Ks 0.7 0.7 0.7
"""

TOML = """root = "thing"
[camera]
type = "perspective"
eye = [0, 0.5, 3]
dir = [0, 0, -1]
fov = 45

[[objects]]
name = "thing"
type = "import"
file = "thing.obj"
"""


def _write(tmp_path):
    (tmp_path / "thing.obj").write_text(OBJ)
    (tmp_path / "mats.mtl").write_text(MTL)
    (tmp_path / "scene.toml").write_text(TOML)
    return tmp_path / "scene.toml"


def test_format_cases(tmp_path):
    s = loader.load_scene(str(_write(tmp_path)), 2.0)
    # quad (2) + triangle (1) + quad (2) + triangle (1) + pentagon (3); "f 1 2" is dropped
    assert s.num_triangles == 9
    kinds = [s.bsdfs[i].type if i >= 0 else -1 for i in s.tri_bsdf]
    assert kinds[:2] == [capi.BSDF_INTERP] * 2 and kinds[2] == capi.BSDF_GLASS
    assert kinds[3:5] == [capi.BSDF_DIFFUSE] * 2 and kinds[5] == -1 and kinds[6:] == [capi.BSDF_MIRROR] * 3
    # the emissive quad gives two triangle lights, in face order
    assert list(s.tri_light) == [-1, -1, -1, 0, 1, -1, -1, -1, -1] and len(s.lights) == 2
    assert s.textures[s.lights[0].intensity_tex].value == (10.0, 5.0, 2.0)
    # Ks clamped at 0; interpolation weight lum(Ks) / (lum(Kd) + lum(Ks)) in float
    interp = s.bsdfs[s.tri_bsdf[0]]
    phong = s.bsdfs[interp.b]
    assert s.textures[phong.tex[0]].value == (np.float32(0.1), np.float32(0.2), 0.0)
    lum = lambda c: np.float32(np.float32(np.float32(c[0] * np.float32(0.2126)) + np.float32(c[1] * np.float32(0.7152)))
                               + np.float32(c[2] * np.float32(0.0722)))
    ks, kd = (np.float32(0.1), np.float32(0.2), 0.0), (np.float32(0.5), np.float32(0.25), np.float32(0.125))
    assert s.textures[interp.tex[0]].value[0] == float(np.float32(lum(ks) / np.float32(lum(kd) + lum(ks))))
    glass = s.bsdfs[s.tri_bsdf[2]]
    assert s.textures[glass.tex[2]].value[0] == float(np.float32(1.0) / np.float32(1.5))
    # faces without normals get normalized sums of the unit face normals; the camera keeps defaults
    assert np.allclose(s.normals[:, 2], 1.0) and s.camera.up == (0.0, 1.0, 0.0) and s.camera.aspect == 2.0
    assert s.camera.fov == 45.0 and s.camera.eye == (0.0, 0.5, 3.0)


def test_format_cases_match_sol_loader(built, tmp_path):
    if not oracle.ref_available():
        pytest.skip("SoL's sources are not built here")
    path = str(_write(tmp_path))
    sol = oracle.RefScene.load(path, 2.0)
    ours = loader.load_scene(path, 2.0)
    c = sol.counts()
    assert (c["lights"], c["bsdfs"], c["textures"]) == (len(ours.lights), len(ours.bsdfs), len(ours.textures))
    a, _ = sol.render(CFG, 40, 20, 3)
    b, _ = oracle.RefScene(ours).render(CFG, 40, 20, 3)
    assert np.array_equal(a, b)


def test_errors(tmp_path):
    (tmp_path / "a.toml").write_text('root = "missing"\n')
    with pytest.raises(loader.SceneFormatError, match="cannot be found"):
        loader.load_scene(str(tmp_path / "a.toml"))
    (tmp_path / "b.toml").write_text('root = "x"\n[[objects]]\nname = "x"\ntype = "import"\nfile = "x.ply"\n')
    with pytest.raises(loader.SceneFormatError, match="Unknown file format"):
        loader.load_scene(str(tmp_path / "b.toml"))
    (tmp_path / "c.toml").write_text('[camera]\ntype = "orthographic"\n')
    with pytest.raises(loader.SceneFormatError, match="Unknown camera type"):
        loader.load_scene(str(tmp_path / "c.toml"))


@pytest.mark.parametrize("name", oracle.REFERENCE_SCENES)
def test_stored_sol_scenes_render_like_sol(name):
    """The stored scenes (tests/golden/sol_scenes) rendered by the CPU checker
    match the film SoL's PathTracer made from its own load of the file."""
    import sys
    from pathlib import Path
    golden = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(golden))
    import make_sol_scenes as fixtures
    d = np.load(golden / "sol_scenes" / f"{name}.npz")
    scene = fixtures.arrays_to_scene(d)
    o = oracle.render(scene, fixtures.config(), fixtures.W, fixtures.H, fixtures.SPP, sample_index=fixtures.INDEX)
    from helpers import per_pixel_parity
    exact, bad = per_pixel_parity(o, d["film"])
    assert bad == 0 and exact >= 0.99
