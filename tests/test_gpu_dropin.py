"""sol::GpuPathTracer, the C++ drop-in for sol::PathTracer, on the same sol::Scene
objects SoL's own renderer uses (built by SoL's constructors in oracle/_ref).

The comparison is SoL's PathTracer::render against GpuPathTracer::render, and
both driven by SoL's RenderJob, per pixel within 1e-4 relative."""
import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.dropin_available(), reason="SoL's sources were not built into oracle/_ref")]


def test_dropin_matches_sol_pathtracer_cornell(built):
    from sol_b200 import scenes
    scene, cfg, *_ = scenes.cornell_frame()
    ref = oracle.RefScene(scene)
    cpu, _ = ref.render(cfg, 64, 64, 4)
    gpu = ref.render_gpu_dropin(cfg, 64, 64, 4)
    exact, bad = per_pixel_parity(gpu, cpu)
    assert bad == 0 and exact >= 0.999


def test_dropin_matches_sol_pathtracer_textured_and_spheres(built):
    from sol_b200 import scenes
    for scene, cfg, (w, h) in ((scenes.cornell_box(0, textured=True, tex_size=64), scenes.CORNELL_CONFIG, (48, 48)),
                               (scenes.sphere_field(6, seed=4, bands=17, segments=32), scenes.SPHERES_CONFIG, (64, 36))):
        ref = oracle.RefScene(scene)
        cpu, _ = ref.render(cfg, w, h, 3, sample_index=11)
        gpu = ref.render_gpu_dropin(cfg, w, h, 3, sample_index=11)
        exact, bad = per_pixel_parity(gpu, cpu)
        assert bad == 0 and exact >= 0.99


@pytest.mark.parametrize("spf", [4, 1])
def test_dropin_under_render_job(built, spf):
    """RenderJob (src/render_job.cpp:23-40) drives either renderer on its own thread;
    with samples_per_frame < sample_count SoL re-renders some samples, and the
    drop-in reproduces that too."""
    from sol_b200 import scenes
    scene, cfg, *_ = scenes.cornell_frame()
    ref = oracle.RefScene(scene)
    cpu = ref.render_job(cfg, 32, 32, 4, spf)
    gpu = ref.render_gpu_dropin(cfg, 32, 32, 4, render_job=True, samples_per_frame=spf)
    exact, bad = per_pixel_parity(gpu, cpu)
    assert bad == 0 and exact >= 0.99
