"""Batched renderer, both schedules: the wavefront (generate / extend / shade /
shadow stages, CUDA-graph bounce loop) and the persistent multi-view megakernel.
Every view's film must equal what the per-view megakernel adds for the same
camera and sample range, bit for bit, and match the CPU checker."""
import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity

pytestmark = pytest.mark.gpu


def _views(scene, n, seed, max_side=96, max_spp=6):
    from sol_b200.scene import Camera
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        w = int(rng.integers(1, max_side))
        h = int(rng.integers(1, max_side))
        spp = int(rng.integers(1, max_spp + 1))
        idx = int(rng.integers(0, 1000))
        c = scene.camera
        jitter = rng.normal(scale=0.05, size=3)
        cam = Camera(eye=tuple(np.add(c.eye, jitter)), dir=c.dir, up=c.up, fov=c.fov * float(rng.uniform(0.7, 1.3)),
                     aspect=w / h)
        out.append((cam, w, h, idx, spp))
    return out


def _render_both(scenes, specs, cfg, scratch_limit=0, **opts):
    import torch
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    gscenes = [GpuScene(s) for s in scenes]
    films_b = [torch.full((3, h, w), 0.5, dtype=torch.float32, device="cuda") for (_, _, w, h, _, _) in specs]
    films_m = [f.clone() for f in films_b]
    br = BatchRenderer(gscenes, **opts)
    if scratch_limit:
        br.set_scratch_limit(scratch_limit)
    br.render(cfg, br.views([(si, cam, w, h, idx, spp, f.data_ptr()) for (si, cam, w, h, idx, spp), f in zip(specs, films_b)]),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    st = br.stats()
    for (si, cam, w, h, idx, spp), f in zip(specs, films_m):
        pt = GpuPathTracer(gscenes[si], cfg, camera=cam)
        pt.render_device(f.data_ptr(), w, h, idx, spp, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return [f.cpu().numpy() for f in films_b], [f.cpu().numpy() for f in films_m], st


@pytest.mark.parametrize("opts", [dict(), dict(capacity=4096, block_size=64), dict(sort_threshold=0xFFFFFFFF),
                                  dict(sort_threshold=0), dict(capacity=32, block_size=128),
                                  dict(ray_order=1), dict(ray_order=2, sort_threshold=0),
                                  dict(ray_order=2, host_loop=True, capacity=1000),
                                  dict(ray_order=3, sort_threshold=0), dict(ray_order=3, capacity=777, host_loop=True),
                                  dict(host_loop=True, block_size=256), dict(schedule=1),
                                  # scratch for about two samples of every view: the samples run in chunks
                                  dict(scratch_limit=2 * 3 * 4 * 96 * 96 * 12)])
def test_batch_equals_megakernel_cornell(built, opts):
    from sol_b200 import scenes
    scene = scenes.cornell_box(0)
    specs = [(0,) + v for v in _views(scene, 12, seed=1)]
    b, m, st = _render_both([scene], specs, scenes.CORNELL_CONFIG, **opts)
    for fb, fm in zip(b, m):
        assert np.array_equal(fb, fm)
    assert st.paths == sum(w * h * spp for (_, _, w, h, _, spp) in specs)


@pytest.mark.parametrize("schedule", [0, 1])
def test_batch_multi_scene_matches_oracle(built, schedule):
    from sol_b200 import scenes
    sc = [scenes.cornell_box(0), scenes.sphere_field(5, seed=7, bands=17, segments=32),
          scenes.cornell_box(1, textured=True, tex_size=32)]
    specs = []
    for si, s in enumerate(sc):
        specs += [(si,) + v for v in _views(s, 3, seed=10 + si, max_side=40, max_spp=3)]
    b, m, _ = _render_both(sc, specs, scenes.CORNELL_CONFIG, schedule=schedule)
    for (si, cam, w, h, idx, spp), fb, fm in zip(specs, b, m):
        assert np.array_equal(fb, fm)
        o = oracle.render(sc[si], scenes.CORNELL_CONFIG, w, h, spp, sample_index=idx, camera=cam,
                          film=np.full((3, h, w), 0.5, np.float32))
        exact, bad = per_pixel_parity(fb, o)
        assert bad == 0


def test_autotune_picks_and_caches(built, tmp_path):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import BatchRenderer, GpuScene
    scene = scenes.cornell_box(0)
    gs = GpuScene(scene)
    films = [torch.zeros((3, 64, 64), device="cuda") for _ in range(4)]
    br = BatchRenderer([gs])
    views = br.views([(0, scene.camera, 64, 64, 0, 4, f.data_ptr()) for f in films])
    cache = tmp_path / "tune.txt"
    chosen = br.autotune(scenes.CORNELL_CONFIG, views, str(cache))
    assert chosen.block_size in (64, 128, 256) and chosen.capacity >= 1 << 18
    assert cache.exists() and cache.read_text().strip()
    again = br.autotune(scenes.CORNELL_CONFIG, views, str(cache))
    assert (again.capacity, again.block_size, again.sort_threshold) == (chosen.capacity, chosen.block_size,
                                                                         chosen.sort_threshold)
    assert all(float(f.abs().sum()) == 0.0 for f in films)   # tuning renders into scratch films


def test_autotune_auto_chooses_a_schedule(built, tmp_path):
    """With schedule AUTO the tuner also times the megakernel schedule and
    reports the winner explicitly; rendering with it keeps the films' bits."""
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    scene = scenes.cornell_box(0)
    gs = GpuScene(scene)
    specs = [(scene.camera, 48, 40, 3, 5), (scene.camera, 20, 64, 100, 2)]
    films = [torch.zeros((3, h, w), device="cuda") for (_, w, h, _, _) in specs]
    br = BatchRenderer([gs], schedule=capi.BATCH_AUTO)
    views = br.views([(0, cam, w, h, idx, spp, f.data_ptr()) for (cam, w, h, idx, spp), f in zip(specs, films)])
    chosen = br.autotune(scenes.CORNELL_CONFIG, views, str(tmp_path / "tune.txt"))
    assert chosen.schedule in (capi.BATCH_WAVEFRONT, capi.BATCH_MEGAKERNEL)
    br.render(scenes.CORNELL_CONFIG, views, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for (cam, w, h, idx, spp), f in zip(specs, films):
        ref = torch.zeros_like(f)
        GpuPathTracer(gs, scenes.CORNELL_CONFIG, camera=cam).render_device(ref.data_ptr(), w, h, idx, spp,
                                                                          torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert torch.equal(f, ref)


def test_wavefront_sample_chunks_match_megakernel(built):
    """Views of many samples under a scratch limit of a few samples: the
    wavefront renders them in chunks, carrying each pixel's sum between chunks,
    and the films keep the megakernel's bits."""
    from sol_b200 import scenes
    scene = scenes.cornell_box(2)
    specs = [(0, scene.camera, 33, 17, 5, 13), (0, scene.camera, 8, 40, 0, 1), (0, scene.camera, 24, 24, 77, 7)]
    limit = 4 * 3 * (33 * 17 + 8 * 40 + 24 * 24) * 3   # about three samples of each view, with running sums
    b, m, st = _render_both([scene], specs, scenes.CORNELL_CONFIG, scratch_limit=limit)
    assert st.launches > 1   # several sample chunks
    for fb, fm in zip(b, m):
        assert np.array_equal(fb, fm)
    assert st.paths == sum(w * h * spp for (_, _, w, h, _, spp) in specs)
