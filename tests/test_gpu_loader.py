"""SoL's own test scenes (test/data/*.toml: the Cornell boxes with glossy,
mirror, glass and water materials) on the GPU.

The scenes come from tests/golden/sol_scenes (made by make_sol_scenes.py):
the tables sol_b200.loader builds from SoL's files, which tests/test_loader.py
checks against SoL's own loader, and the film SoL's PathTracer renders from its
own load of each file.  The GPU render of the stored scene must match that
film per pixel; where SoL's files are present, the scene is also loaded afresh
and rendered against the CPU checker."""
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_sol_scenes as fixtures  # noqa: E402


@pytest.mark.parametrize("name", oracle.REFERENCE_SCENES)
def test_sol_test_scene_on_gpu_matches_sol_film(built, name):
    from sol_b200.renderer import GpuPathTracer, Image
    d = np.load(GOLDEN / "sol_scenes" / f"{name}.npz")
    scene = fixtures.arrays_to_scene(d)
    img = Image(fixtures.W, fixtures.H)
    GpuPathTracer(scene, fixtures.config()).render(img, fixtures.INDEX, fixtures.SPP)
    exact, bad = per_pixel_parity(img.channels, d["film"])
    print(f"{name}: {exact:.4f} of pixels bit-identical, {bad} above 1e-4")
    assert bad == 0 and exact >= 0.99
    assert float(img.channels.mean()) > 0.01


@pytest.mark.parametrize("name", oracle.REFERENCE_SCENES)
def test_sol_test_scene_file_on_gpu(built, name):
    path = oracle.reference_scene(name)
    if path is None:
        pytest.skip("SoL's scene files are not present here (the stored scenes above cover them)")
    from sol_b200 import loader
    from sol_b200.renderer import GpuPathTracer, Image
    cfg = fixtures.config()
    scene = loader.load_scene(str(path), 1.0)
    img = Image(64, 64)
    GpuPathTracer(scene, cfg).render(img, 3, 8)
    o = oracle.render(scene, cfg, 64, 64, 8, sample_index=3)
    exact, bad = per_pixel_parity(img.channels, o)
    assert bad == 0 and exact >= 0.99
