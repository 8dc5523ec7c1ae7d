"""The kernels' self-checks, made to fire without a fault: a bound lowered to
a few steps runs out, the kernel records the fault and stops the ray or the
loop instead of running on, and the call reports the status (the error
surface SoL's job control offers, src/render_job.cpp:42-59, is a timeout on
the host).  The next render on the same handle is correct again."""
import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity

pytestmark = pytest.mark.gpu


def test_traversal_bound_reports_bad_index_then_recovers(built):
    from sol_b200 import capi, scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene, Image
    scene = scenes.sphere_field(6, seed=4, bands=17, segments=32)
    cfg = scenes.SPHERES_CONFIG
    gs = GpuScene(scene)
    pt = GpuPathTracer(gs, cfg)
    gs.set_traversal_limit(2)
    with pytest.raises(capi.SolGpuError) as e:
        pt.render(Image(32, 18), 0, 2)
    assert e.value.code == capi.ERR_BAD_INDEX
    assert "traversal" in str(e.value)
    gs.set_traversal_limit(0)
    img = Image(32, 18)
    pt.render(img, 0, 2)
    ref = oracle.render(scene, cfg, 32, 18, 2)
    exact, bad = per_pixel_parity(img.channels, ref)
    assert bad == 0


@pytest.mark.parametrize("schedule", [0, 1])
def test_batch_traversal_bound_then_recovers(built, schedule):
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    scene = scenes.cornell_box(0)
    cfg = scenes.CORNELL_CONFIG
    gs = GpuScene(scene)
    br = BatchRenderer([gs], schedule=schedule)
    film = torch.zeros((3, 24, 24), device="cuda")
    views = br.views([(0, scene.camera, 24, 24, 0, 3, film.data_ptr())])
    gs.set_traversal_limit(1)
    br.render(cfg, views)
    with pytest.raises(capi.SolGpuError) as e:
        br.stats()
    assert e.value.code == capi.ERR_BAD_INDEX
    gs.set_traversal_limit(0)
    film.zero_()
    br.render(cfg, views)
    br.stats()
    ref = torch.zeros_like(film)
    GpuPathTracer(gs, cfg).render_device(ref.data_ptr(), 24, 24, 0, 3)
    torch.cuda.synchronize()
    assert torch.equal(film, ref)


def test_wavefront_iteration_bound_reports_timeout_then_recovers(built):
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    scene = scenes.cornell_box(0)
    cfg = scenes.CORNELL_CONFIG
    gs = GpuScene(scene)
    for host_loop in (False, True):
        br = BatchRenderer([gs], schedule=capi.BATCH_WAVEFRONT, host_loop=host_loop)
        film = torch.zeros((3, 20, 28), device="cuda")
        views = br.views([(0, scene.camera, 28, 20, 5, 4, film.data_ptr())])
        br.set_iteration_limit(1)
        if host_loop:
            with pytest.raises(capi.SolGpuError) as e:
                br.render(cfg, views)
                br.stats()
        else:
            br.render(cfg, views)
            with pytest.raises(capi.SolGpuError) as e:
                br.stats()
        assert e.value.code == capi.ERR_TIMEOUT
        br.set_iteration_limit(0)
        film.zero_()
        br.render(cfg, views)
        st = br.stats()
        assert st.paths == 28 * 20 * 4
        ref = torch.zeros_like(film)
        GpuPathTracer(gs, cfg).render_device(ref.data_ptr(), 28, 20, 5, 4)
        torch.cuda.synchronize()
        assert torch.equal(film, ref)
