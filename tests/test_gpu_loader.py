"""SoL's own test scenes (test/data/*.toml: the Cornell boxes with glossy,
mirror, glass and water materials), loaded by sol_b200.loader and rendered on
the GPU, against the CPU checker.  Runs where the scene files are present."""
import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", oracle.REFERENCE_SCENES)
def test_sol_test_scene_on_gpu(built, name):
    path = oracle.reference_scene(name)
    if path is None:
        pytest.skip("SoL's test scenes are not present here")
    from sol_b200 import loader
    from sol_b200.renderer import GpuPathTracer, Image
    from sol_b200.scene import Config
    cfg = Config(max_path_len=16, min_rr_path_len=3, min_survival_prob=0.05, max_survival_prob=0.75, ray_offset=1e-5)
    scene = loader.load_scene(str(path), 1.0)
    img = Image(64, 64)
    GpuPathTracer(scene, cfg).render(img, 3, 8)
    o = oracle.render(scene, cfg, 64, 64, 8, sample_index=3)
    exact, bad = per_pixel_parity(img.channels, o)
    assert bad == 0 and exact >= 0.99
    assert float(img.channels.mean()) > 0.01
