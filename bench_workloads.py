"""The per-configuration measurements of bench.py (one GPU).

  cornell  the Cornell box: 256x256, 16 spp, max path length 16, Russian
           roulette from bounce 3, one megakernel render per step.
  views    64 seeded views (square side log-uniform 64-1024, 1-64 spp) of a
           4,194,314-triangle sphere field (256 displaced spheres): the batched
           renderer in one call (autotuned schedule), the wavefront and the
           multi-view megakernel each on their own, against 64 plain megakernel
           launches.  All give bit-identical films (same estimator, same
           seeds), so their RMSE is equal; it is reported against a 256-spp
           render of every view.
  adjoint  the textured Cornell box (two 256x256 RGB albedo images): forward
           render 128x128 x 16 spp, then the L2 loss against a 1024-spp target
           and the path-replay adjoint; the ratio adjoint / forward time is the
           value.  The gradient is checked per parameter against central
           finite differences (eps 1e-3, common random numbers) of the GPU
           forward on 64 seeded parameters, and on 8 of them against central
           differences of SoL's own CPU renderer.
  scenes   32 independent textured sphere fields (10k-2M triangles, films
           128^2-512^2, 16 spp): forward + L2 adjoint of all 32 in one fused
           launch, against the forward alone (batched and plain); gradients
           checked per scene and per parameter against finite differences on
           16 parameters.

Every timed launch is preceded by a 256 MiB write that flushes L2, and timed
with CUDA events on the launching stream.  Each record carries the CPU
baseline measured in the same run: SoL's own path tracer (oracle/_ref, which
links nothing of this library) on the host's threads, on a stated sample of
the same workload.
"""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path

import numpy as np

METRIC = "Mpaths/s"
EPS = 1e-3
GRAD_REL_TOL = 0.02


# ---------------------------------------------------------------------------
# CPU reference (SoL's PathTracer)
# ---------------------------------------------------------------------------

def cpu_model() -> str:
    """The host CPU's model name (first /proc/cpuinfo entry)."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_renderer(scene, threads: int, camera=None):
    """SoL's own path tracer (oracle/_ref, which links nothing of this
    library) on `threads` host threads, or the oracle restatement where SoL's
    sources were not built; returns (kind, run(sample_index, spp, w, h, cfg) ->
    (film, seconds of the render call alone))."""
    import oracle
    if oracle.ref_available():
        ref = oracle.RefScene(scene, camera=camera)

        def run(index, spp, w, h, cfg):
            film, ms = ref.render(cfg, w, h, spp, sample_index=index, threads=threads)
            return film, ms / 1000.0
        run.ref = ref
        return "reference", run

    def run_port(index, spp, w, h, cfg):
        t = time.perf_counter()
        film = oracle.render(scene, cfg, w, h, spp, sample_index=index, threads=threads, camera=camera)
        return film, time.perf_counter() - t
    return "port", run_port


def cpu_baseline(paths: float, seconds: float, kind: str, sample: str) -> dict:
    threads = os.cpu_count() or 1
    return {"value": paths / seconds / 1e6, "unit": METRIC, "cores": threads, "cpu_model": cpu_model(),
            "kind": kind, "sample": sample}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def _events(torch, n):
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def _timed(torch, flush, stream, fn, steps, warmup):
    """Runs fn(i) warmup times, then steps times with an L2 flush before each;
    returns the per-step device times in ms."""
    for i in range(warmup):
        fn(i)
    torch.cuda.synchronize()
    ev = _events(torch, steps)
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        fn(warmup + i)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def single_view_schedules(gs, cfg, cam, w, h, spp, plain_ms: float, steps: int, warmup: int) -> dict:
    """The batch schedules on a configuration of one view: the wavefront (16M
    path slots, 256 threads; the capacity the views workload's autotuner
    picks) and the multi-view megakernel, each rendering the view through
    sol_gpu_batch_render, timed like the plain launch, with its Mpaths/s, its
    ratio to the plain launch's and whether its film has the plain film's
    bits."""
    import torch
    from sol_b200 import capi
    from sol_b200.renderer import BatchRenderer, GpuPathTracer
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    plain = torch.zeros((3, h, w), device="cuda")
    GpuPathTracer(gs, cfg).render_device(plain.data_ptr(), w, h, 0, spp, stream.cuda_stream)
    paths = float(w * h * spp)
    out = {"note": "one view through the batch entry point; the plain launch is sol_gpu_render_device",
           "plain_mpaths_s": paths / plain_ms / 1e3}
    for name, kw in (("wavefront", dict(capacity=1 << 24, block_size=256, schedule=capi.BATCH_WAVEFRONT)),
                     ("multi_view_megakernel", dict(schedule=capi.BATCH_MEGAKERNEL))):
        br = BatchRenderer([gs], **kw)
        film = torch.zeros((3, h, w), device="cuda")
        arr = br.views([(0, cam, w, h, 0, spp, film.data_ptr())])

        def render(i, br=br, arr=arr, film=film):
            film.zero_()
            br.render(cfg, arr, stream.cuda_stream)
        ms = float(np.mean(_timed(torch, flush, stream, render, steps, warmup)))
        torch.cuda.synchronize()
        out[name] = {"value": paths / ms / 1e3, "unit": METRIC, "ms": ms, "vs_plain": plain_ms / ms,
                     "same_film_bits": bool(torch.equal(film, plain))}
        br.close()
        del film
    return out


def grad_check(g, fd, rel: float = GRAD_REL_TOL, floor_frac: float = 0.01) -> dict:
    """Per-parameter comparison of adjoint gradients with finite differences.

    A parameter passes when |g - fd| <= rel * max(|fd|, floor), where the
    absolute floor is `floor_frac` of the largest |fd| in the checked set (the
    finite difference of a float32 render carries rounding noise of that
    order for parameters with almost no effect on the loss)."""
    g = np.asarray(g, np.float64)
    fd = np.asarray(fd, np.float64)
    floor = floor_frac * float(np.max(np.abs(fd))) if fd.size else 0.0
    scale = np.maximum(np.abs(fd), floor)
    err = np.abs(g - fd) / np.where(scale > 0, scale, 1.0)
    ok = err <= rel
    worst = int(np.argmax(err)) if err.size else -1
    return {"params": int(fd.size), "within_tol": int(np.sum(ok)), "tol_rel": rel, "abs_floor": floor,
            "max_rel_err": float(np.max(err)) if err.size else 0.0,
            "median_rel_err": float(np.median(err)) if err.size else 0.0,
            "vector_rel_err": float(np.linalg.norm(g - fd) / max(np.linalg.norm(fd), 1e-30)),
            "worst": None if worst < 0 else {"index": worst, "adjoint": float(g[worst]), "fd": float(fd[worst])}}


def roulette_misses(g, fd, fd_half, check: dict) -> list:
    """The parameters that miss the per-parameter tolerance, with their central
    differences at eps and eps / 2.  With Russian roulette on, a survival
    decision that flips inside [x - eps, x + eps] adds its jump to the
    difference quotient (and, the loss being quadratic, the jump's square
    always with the same sign), which no derivative of the estimate has."""
    floor = check["abs_floor"]
    out = []
    for j, (a, f, h) in enumerate(zip(g, fd, fd_half)):
        scale = max(abs(f), floor)
        if abs(a - f) > check["tol_rel"] * scale:
            out.append({"index": j, "adjoint": float(a), "fd": float(f), "fd_half_eps": float(h),
                        "jumps": bool(abs(f - h) > check["tol_rel"] * scale)})
    return out


def fd_step(value: float, eps: float = EPS) -> float:
    """The central-difference step of a parameter: eps, scaled by the value
    above 1 (emissions of 10-20 move the float32 film by less than its
    rounding at an absolute step of 1e-3)."""
    return eps * max(1.0, abs(float(value)))


def fd_gradient(gs, render_loss, indices, eps: float = EPS):
    """Central differences of render_loss() over the given parameter indices
    (step fd_step(value, eps) per parameter)."""
    base = gs.get_params()
    out = []
    for j in indices:
        h = fd_step(base[j], eps)
        v = base.copy()
        v[j] = base[j] + h
        gs.set_params(v)
        lp = render_loss()
        v[j] = base[j] - h
        gs.set_params(v)
        lm = render_loss()
        out.append((lp - lm) / (2.0 * h))
    gs.set_params(base)
    return np.asarray(out)


def choose_params(gs, n, seed, scalars=False):
    """n seeded parameter indices: about an eighth from the constant colour
    textures (albedos, specular colours, emission) and, with `scalars`, the
    constant scalar textures; the rest texels."""
    from sol_b200 import capi
    count, tex_off, img_off = gs.param_layout()
    rng = np.random.default_rng(seed)
    consts = []
    for t, off in zip(gs.scene.textures, tex_off):
        if t.type == capi.TEX_CONSTANT_COLOR:
            consts += [off, off + 1, off + 2]
        elif t.type == capi.TEX_CONSTANT and scalars:
            consts.append(off)
    n_c = min(len(consts), max(4, n // 8)) if img_off else min(len(consts), n)
    pick = list(rng.choice(consts, size=n_c, replace=False))
    if img_off:
        pick += list(rng.choice(np.arange(img_off[0], count), size=n - n_c, replace=False))
    return sorted(int(j) for j in pick)


def _base(args, metric, value, unit, ms, hib, config, clocks, launches, steps, warmup, **extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scenes)", "config": config, "gpu_launches": launches,
            "clocks": clocks}
    line.update(extra)
    return line


def _alg_bytes(st, paths_split=0):
    """Algorithmic bytes of a counted render: 64 B per BVH node, 48 B per
    triangle, 32 B per ray, and 24 B per path of split-schedule colour scratch."""
    return 64.0 * st.nodes_visited + 48.0 * st.tris_tested + 32.0 * st.rays + 24.0 * paths_split


# ---------------------------------------------------------------------------
# cornell: the reference's own configuration
# ---------------------------------------------------------------------------

def run_cornell(args, ClockSampler, load_peaks, steps=None, warmup=None, cpu=True):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import GpuPathTracer, GpuScene, Image
    # A render takes about 2 ms: at least 200 timed steps, so that the clock
    # sampler (one sample per 100 ms) sees the timed region.
    steps = max(steps or args.steps, 200)
    warmup = warmup or args.warmup
    scene, cfg, w, h, spp = scenes.cornell_frame()
    gs = GpuScene(scene)
    pt = GpuPathTracer(gs, cfg)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    film = torch.zeros((3, h, w), device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def render(i):
        pt.render_device(film.data_ptr(), w, h, i * spp, spp, sp)

    with ClockSampler(torch.cuda.current_device()) as clocks:
        ms = _timed(torch, flush, stream, render, steps, warmup)
    st = pt.stats()
    gs.set_instrumented(True)
    render(0)
    torch.cuda.synchronize()
    ist = pt.stats()
    gs.set_instrumented(False)
    paths = float(w * h * spp)
    alg = _alg_bytes(ist, ist.paths if st.sample_chunk > 0 else 0)
    mean_s = float(np.mean(ms)) / 1000.0
    peak, src = load_peaks()
    img = Image(w, h)
    pt.render(img, 0, spp)
    t0 = time.perf_counter()
    for i in range(steps):
        pt.render(img, (1 + i) * spp, spp)
    e2e_s = (time.perf_counter() - t0) / steps
    extra = {"batched": single_view_schedules(gs, cfg, scene.camera, w, h, spp, float(np.mean(ms)), 50, 3)}
    if cpu:
        kind, run = cpu_renderer(scene, os.cpu_count() or 1)
        run(0, 1, w, h, cfg)
        _, t = run(0, spp, w, h, cfg)
        extra["cpu_baseline"] = cpu_baseline(paths, t, kind, f"the whole {w}x{h} x {spp} spp render, one call")
    import ctypes
    from sol_b200 import capi
    return _base(args, METRIC, paths / mean_s / 1e6, METRIC, mean_s * 1000.0, True,
                 {"workload": f"Cornell box (36 triangles: room, light quad, glass and Phong boxes), {w}x{h}, "
                              f"{spp} spp, max path length {cfg.max_path_len}, Russian roulette from bounce "
                              f"{cfg.min_rr_path_len}", "width": w, "height": h, "spp": spp,
                  "max_path_len": cfg.max_path_len, "l2": "flushed between steps (256 MiB write)"},
                 clocks.summary(), steps * st.launches, steps, warmup,
                 mrays_per_s=st.rays / mean_s / 1e6, rays_per_path=st.rays / paths,
                 roofline={"bound": "hbm", "achieved": alg / mean_s / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": alg / mean_s / 1e9 / peak, "traffic": None, "peak_source": src,
                           "algorithmic_bytes_per_launch": alg,
                           "note": "36 triangles: the scene sits in L1/L2; launch-latency bound at 1M paths"},
                 e2e={"value": paths / e2e_s / 1e6, "unit": METRIC,
                      "h2d_bytes_per_step": ctypes.sizeof(capi.SolGpuCamera) + ctypes.sizeof(capi.SolGpuConfig) + 20,
                      "d2h_bytes_per_step": 3 * w * h * 4}, **extra)


# ---------------------------------------------------------------------------
# views: batched renderer vs plain megakernel launches
# ---------------------------------------------------------------------------

def run_views(args, ClockSampler, load_peaks, steps=None, warmup=None, cpu=True):
    import ctypes

    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    steps = steps or args.steps
    warmup = warmup or args.warmup
    small = args.small
    scene = scenes.sphere_field(16 if small else 256, seed=1)
    views = scenes.view_set(8 if small else 64, seed=2, max_side=256 if small else 1024)
    cfg = scenes.SPHERES_CONFIG
    gs = GpuScene(scene)
    info = gs.info()
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    films = [torch.zeros((3, s, s), device="cuda") for _, s, _ in views]
    tracers = [GpuPathTracer(gs, cfg, camera=cam) for cam, _, _ in views]
    paths = float(sum(s * s * p for _, s, p in views))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def plain(i):
        for (cam, s, p), pt, f in zip(views, tracers, films):
            pt.render_device(f.data_ptr(), s, s, i * 64, p, sp)

    renderers = {"batched": BatchRenderer([gs], schedule=capi.BATCH_AUTO),
                 "wavefront": BatchRenderer([gs], schedule=capi.BATCH_WAVEFRONT),
                 "megakernel": BatchRenderer([gs], schedule=capi.BATCH_MEGAKERNEL)}

    def varr(r, i, fl=None):
        fl = fl or films
        return r.views([(0, cam, s, s, i * 64, p, f.data_ptr()) for (cam, s, p), f in zip(views, fl)])

    tune = {}
    for name, r in renderers.items():
        t0 = time.perf_counter()
        o = r.autotune(cfg, varr(r, 0))
        tune[name] = {"schedule": ["wavefront", "megakernel", "auto"][o.schedule], "capacity": o.capacity,
                      "block_size": o.block_size, "sort_threshold": o.sort_threshold,
                      "ray_order": ["default", "queue", "sorted", "packed_shadows"][o.ray_order],
                      "seconds": time.perf_counter() - t0}
    arrays = {name: {i: varr(r, i) for i in range(warmup + steps)} for name, r in renderers.items()}
    times = {}
    with ClockSampler(torch.cuda.current_device()) as clocks:
        times["plain"] = _timed(torch, flush, stream, plain, steps, warmup)
        for name, r in renderers.items():
            times[name] = _timed(torch, flush, stream, lambda i, r=r, name=name: r.render(cfg, arrays[name][i], sp),
                                 steps, warmup)
    mean = {k: float(np.mean(v)) / 1000.0 for k, v in times.items()}
    wf_stats = renderers["wavefront"].stats()

    # Same films from every schedule (one fresh render each).
    ref_films = [torch.zeros_like(f) for f in films]
    for (cam, s, p), pt, f in zip(views, tracers, ref_films):
        pt.render_device(f.data_ptr(), s, s, 0, p, sp)
    identical = {}
    for name, r in renderers.items():
        fb = [torch.zeros_like(f) for f in films]
        r.render(cfg, varr(r, 0, fb), sp)
        torch.cuda.synchronize()
        identical[name] = all(torch.equal(a, b) for a, b in zip(ref_films, fb))

    # RMSE of the films against a 256-spp render of every view.
    gt_spp = 16 if small else 256
    rmse = []
    for (cam, s, p), pt, a in zip(views, tracers, ref_films):
        g = torch.zeros_like(a)
        pt.render_device(g.data_ptr(), s, s, 1 << 20, gt_spp, sp)
        torch.cuda.synchronize()
        rmse.append(float(torch.sqrt(torch.mean((a / p - g / gt_spp) ** 2))))

    # Algorithmic bytes of the same rays (counting build of the megakernel, one view at a time).
    gs.set_instrumented(True)
    nodes = tris = rays = 0
    alg = 0.0
    for (cam, s, p), pt in zip(views, tracers):
        tmp = torch.zeros((3, s, s), device="cuda")
        pt.render_device(tmp.data_ptr(), s, s, 0, p, sp)
        torch.cuda.synchronize()
        st = pt.stats()
        alg += _alg_bytes(st, st.paths if st.sample_chunk > 0 else 0)
    gs.set_instrumented(False)

    # End to end through the batch entry point: view table built and uploaded,
    # films read back to pinned host memory.
    best = min(renderers, key=lambda k: mean[k])
    r = renderers["batched"]
    host = [torch.empty(f.shape, dtype=torch.float32, pin_memory=True) for f in films]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(steps):
        r.render(cfg, varr(r, 100 + i), sp)
        for h_, f in zip(host, films):
            h_.copy_(f, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / steps

    extra = {}
    if cpu:
        # SoL's PathTracer on every 16th view (4 views), up to 4 samples each.
        kind = None
        cpu_paths, cpu_s = 0.0, 0.0
        sample_views = list(range(0, len(views), 16))
        for k in sample_views:
            cam, s, p = views[k]
            kind, run = cpu_renderer(scene, os.cpu_count() or 1, camera=cam)
            n = min(p, 4)
            _, t = run(0, n, s, s, cfg)
            cpu_paths += s * s * n
            cpu_s += t
        extra["cpu_baseline"] = cpu_baseline(cpu_paths, cpu_s, kind,
                                             f"views {sample_views} at min(spp, 4) samples each "
                                             f"({int(cpu_paths)} paths); scene build excluded")
    peak, src = load_peaks()
    value = paths / mean["batched"] / 1e6
    cfgd = {"workload": f"{len(views)} uneven views (side log-U[64,1024], 1-64 spp) of a "
                        f"{info.num_triangles}-triangle sphere field, batched in one call (autotuned schedule)",
            "triangles": info.num_triangles, "views": len(views), "paths_per_step": int(paths),
            "pixels": int(sum(s * s for _, s, _ in views)), "max_path_len": cfg.max_path_len,
            "l2": "flushed between steps (256 MiB write); scene larger than L2", "small": bool(small)}
    return _base(
        args, METRIC, value, METRIC, 1000.0 * mean["batched"], True, cfgd, clocks.summary(), steps, steps, warmup,
        launch_note="per batched step: one call (the wavefront's stage kernels in a CUDA graph, or one "
                    "multi-view megakernel launch) plus the in-order sum pass; per plain step: one launch per view",
        schedules={k: {"value": paths / v / 1e6, "unit": METRIC, "ms_per_step": 1000.0 * v,
                       "vs_plain": mean["plain"] / v} for k, v in mean.items()},
        autotune=tune, fastest=best,
        wavefront_stats={"rays": wf_stats.rays, "shadow_rays": wf_stats.shadow_rays, "launches": wf_stats.launches},
        equal_rmse={"films_bit_identical_to_plain": identical, "reference": f"{gt_spp}-spp megakernel render per view",
                    "rmse_mean": float(np.mean(rmse)), "note": "identical films, so identical RMSE per schedule"},
        roofline={"bound": "hbm", "achieved": alg / mean["batched"] / 1e9, "peak": peak, "unit": "GB/s",
                  "frac": alg / mean["batched"] / 1e9 / peak, "traffic": None, "peak_source": src,
                  "algorithmic_bytes_per_launch": alg},
        e2e={"value": paths / e2e_s / 1e6, "unit": METRIC,
             "h2d_bytes_per_step": len(views) * ctypes.sizeof(capi.SolGpuView) + ctypes.sizeof(capi.SolGpuConfig),
             "d2h_bytes_per_step": int(sum(f.numel() * 4 for f in films))},
        scene={"triangles": info.num_triangles, "bvh_inner_nodes": info.num_nodes, "bvh_depth": info.bvh_depth,
               "device_mb": info.device_bytes / 2**20, "build_ms": info.build_ms}, **extra)


# ---------------------------------------------------------------------------
# adjoint: path-replay adjoint vs forward on the textured Cornell box
# ---------------------------------------------------------------------------

def run_adjoint(args, ClockSampler, load_peaks, steps=None, warmup=None, cpu=True):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene, image_l2
    # Each timed call takes a few milliseconds: at least 50 steps of each, so
    # that the ratio is not one launch's jitter and the clock sampler (one
    # sample per 100 ms) sees the timed region.
    steps = max(steps or args.steps, 50)
    warmup = warmup or args.warmup
    W = H = 64 if args.small else 128
    SPP = 16
    tex = 64 if args.small else 256
    cfg = scenes.CORNELL_CONFIG
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    truth = GpuScene(scenes.cornell_box(0, textured=True, tex_size=tex, tex_seed=3))
    target = torch.zeros((3, H, W), device="cuda")
    GpuPathTracer(truth, cfg).render_device(target.data_ptr(), W, H, 1 << 24, 1024, sp)
    torch.cuda.synchronize()
    target /= 1024
    scene = scenes.cornell_box(0, textured=True, tex_size=tex, tex_seed=11)
    gs = GpuScene(scene)
    pt = GpuPathTracer(gs, cfg)
    count = gs.param_layout()[0]
    film = torch.zeros((3, H, W), device="cuda")
    dl = torch.zeros((3, H, W), device="cuda")
    grad = torch.zeros(count, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    n = 3 * W * H

    def forward(i):
        pt.render_device(film.data_ptr(), W, H, i * SPP, SPP, sp)

    def adjoint(i):
        image_l2(film.data_ptr(), target.data_ptr(), n, 1.0 / SPP, dl.data_ptr(), loss.data_ptr(), sp)
        pt.adjoint(dl.data_ptr(), grad.data_ptr(), W, H, i * SPP, SPP, sp)

    br = BatchRenderer([gs])

    def fused(i):
        br.forward_adjoint(cfg, [(0, gs.scene.camera, W, H, i * SPP, SPP, film.data_ptr(), target.data_ptr(),
                                  grad.data_ptr(), loss.data_ptr())], sp)

    with ClockSampler(torch.cuda.current_device()) as clocks:
        f_ms = _timed(torch, flush, stream, forward, steps, warmup)
        a_ms = _timed(torch, flush, stream, adjoint, steps, warmup)
        x_ms = _timed(torch, flush, stream, fused, steps, warmup)
    fwd, adj, fus = np.mean(f_ms), np.mean(a_ms), np.mean(x_ms)

    # Gradient at one sample range against central differences of the GPU forward.
    film.zero_()
    grad.zero_()
    loss.zero_()
    forward(7)
    adjoint(7)
    torch.cuda.synchronize()
    g = grad.cpu().numpy()
    tgt = target.double()

    def render_loss():
        f = torch.zeros((3, H, W), device="cuda")
        pt.render_device(f.data_ptr(), W, H, 7 * SPP, SPP, sp)
        torch.cuda.synchronize()
        return float(((f.double() / SPP - tgt) ** 2).sum())

    idx = choose_params(gs, 64, seed=5)
    fd = fd_gradient(gs, render_loss, idx)
    check = grad_check(g[idx], fd)
    miss = [j for j in range(len(idx)) if abs(g[idx][j] - fd[j]) > GRAD_REL_TOL * max(abs(fd[j]), check["abs_floor"])]
    if miss:   # central differences at eps / 2 for the misses (roulette jumps)
        half = np.array(fd)
        half[miss] = fd_gradient(gs, render_loss, [idx[j] for j in miss], eps=EPS / 2)
        check["roulette_misses"] = roulette_misses(g[idx], fd, half, check)
    extra = {}
    if cpu:
        # SoL's renderer: its forward rate on the loss render, and central
        # differences of its loss on 8 of the parameters (same sample range).
        import oracle
        tgt_np = target.cpu().numpy().astype(np.float64)
        kind, run = cpu_renderer(scene, os.cpu_count() or 1)
        _, t_fwd = run(7 * SPP, SPP, W, H, cfg)
        sub = idx[::8]
        base = gs.get_params()
        fd_sol = []
        t0 = time.perf_counter()
        for j in sub:
            vals = []
            for sgn in (1.0, -1.0):
                v = base.copy()
                v[j] = base[j] + sgn * EPS
                s2 = _with_params(scene, gs, v)
                _, r2 = cpu_renderer(s2, os.cpu_count() or 1)
                f, _ = r2(7 * SPP, SPP, W, H, cfg)
                vals.append(float(((f.astype(np.float64) / SPP - tgt_np) ** 2).sum()))
            fd_sol.append((vals[0] - vals[1]) / (2 * EPS))
        fd_s = time.perf_counter() - t0
        extra["cpu_baseline"] = cpu_baseline(W * H * SPP, t_fwd, kind, f"the forward loss render ({W}x{H} x {SPP} spp)")
        extra["gradient_check_vs_sol_fd"] = dict(grad_check(g[sub], np.asarray(fd_sol)),
                                                 cpu_fd_seconds_8_params=fd_s)
    paths = float(W * H * SPP)
    cfgd = {"workload": f"textured Cornell box ({tex}x{tex} RGB albedo images on back wall and floor), "
                        f"{W}x{H} x {SPP} spp loss render, max path length {cfg.max_path_len}",
            "params": count, "width": W, "height": H, "spp": SPP, "target_spp": 1024,
            "l2": "flushed between steps (256 MiB write)", "small": bool(args.small)}
    return _base(
        args, "PRB adjoint / forward time", adj / fwd, "ratio", adj, False, cfgd, clocks.summary(), 2 * steps,
        steps, warmup, forward_ms=fwd, adjoint_ms=adj, fused_ms=fus, fused_over_forward=fus / fwd,
        forward_mpaths_s=paths / fwd / 1e3, adjoint_mpaths_s=paths / adj / 1e3,
        gradient_check=dict(check, eps=EPS, nonzero_fd=int(np.count_nonzero(fd))),
        e2e={"value": adj / fwd, "unit": "ratio", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}, **extra)


def _with_params(scene, gs, values):
    """A copy of `scene` whose textures hold the parameter vector `values`
    (the layout of sol_gpu_param_layout: constants, then texel planes)."""
    import copy
    from sol_b200 import capi
    _, tex_off, img_off = gs.param_layout()
    s = copy.copy(scene)
    s.textures = [copy.copy(t) for t in scene.textures]
    s.images = [np.array(im, np.float32, copy=True) for im in scene.images]
    for t, off in zip(s.textures, tex_off):
        if t.type == capi.TEX_CONSTANT_COLOR:
            t.value = tuple(float(x) for x in values[off:off + 3])
        elif t.type == capi.TEX_CONSTANT:
            t.value = (float(values[off]),) + tuple(t.value[1:])
    for k, off in enumerate(img_off):
        im = s.images[k]
        s.images[k] = np.asarray(values[off:off + im.size], np.float32).reshape(im.shape)
    return s


# ---------------------------------------------------------------------------
# scenes: fused forward + adjoint over 32 scenes in one launch
# ---------------------------------------------------------------------------

def run_scenes(args, ClockSampler, load_peaks, steps=None, warmup=None, cpu=True):
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
    steps = steps or args.steps
    warmup = warmup or args.warmup
    SPP = 16
    num = 4 if args.small else 32
    t0 = time.perf_counter()
    made = scenes.scene_set(num, max_tris=200_000 if args.small else 2_000_000)
    gen_s = time.perf_counter() - t0
    cfg = scenes.SPHERES_CONFIG
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    gss = [GpuScene(s) for s, _ in made]
    infos = [g.info() for g in gss]
    sides = [side for _, side in made]
    tracers = [GpuPathTracer(g, cfg) for g in gss]
    counts = [g.param_layout()[0] for g in gss]
    films = [torch.zeros((3, s, s), device="cuda") for s in sides]
    targets = []
    for pt, s in zip(tracers, sides):
        t = torch.zeros((3, s, s), device="cuda")
        pt.render_device(t.data_ptr(), s, s, 1 << 22, 64, sp)
        targets.append(t * (0.9 / 64))
    grads = [torch.zeros(c, device="cuda") for c in counts]
    losses = torch.zeros(num, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    br = BatchRenderer(gss)
    paths = float(sum(s * s * SPP for s in sides))

    def specs(i):
        return [(k, made[k][0].camera, s, s, i * SPP, SPP, films[k].data_ptr(), targets[k].data_ptr(),
                 grads[k].data_ptr(), losses[k:k + 1].data_ptr()) for k, s in enumerate(sides)]

    def fused(i):
        br.forward_adjoint(cfg, specs(i), sp)

    renderers = {"wavefront": BatchRenderer(gss, schedule=capi.BATCH_WAVEFRONT),
                 "megakernel": BatchRenderer(gss, schedule=capi.BATCH_MEGAKERNEL)}

    def varr(r, i):
        return r.views([(k, made[k][0].camera, s, s, i * SPP, SPP, films[k].data_ptr()) for k, s in enumerate(sides)])
    tune = {}
    for name, r in renderers.items():
        o = r.autotune(cfg, varr(r, 0))
        tune[name] = {"capacity": o.capacity, "block_size": o.block_size, "sort_threshold": o.sort_threshold,
                      "ray_order": ["default", "queue", "sorted", "packed_shadows"][o.ray_order]}
    arrays = {name: {i: varr(r, i) for i in range(warmup + steps)} for name, r in renderers.items()}

    def plain(i):
        for pt, s, f in zip(tracers, sides, films):
            pt.render_device(f.data_ptr(), s, s, i * SPP, SPP, sp)

    times = {}
    with ClockSampler(torch.cuda.current_device()) as clocks:
        times["fused"] = _timed(torch, flush, stream, fused, steps, warmup)
        for name, r in renderers.items():
            times[name] = _timed(torch, flush, stream, lambda i, r=r, name=name: r.render(cfg, arrays[name][i], sp),
                                 steps, warmup)
        times["plain"] = _timed(torch, flush, stream, plain, steps, warmup)
    mean = {k: float(np.mean(v)) for k, v in times.items()}
    fwd_batched = min(mean["wavefront"], mean["megakernel"])

    # Per-scene gradient check: 16 parameters against central differences of the forward.
    for f in films:
        f.zero_()
    for g in grads:
        g.zero_()
    losses.zero_()
    fused(3)
    torch.cuda.synchronize()
    checks = []
    for k, (gs, pt, s) in enumerate(zip(gss, tracers, sides)):
        tgt = targets[k].double()

        def render_loss(pt=pt, s=s, tgt=tgt):
            f = torch.zeros((3, s, s), device="cuda")
            pt.render_device(f.data_ptr(), s, s, 3 * SPP, SPP, sp)
            torch.cuda.synchronize()
            return float(((f.double() / SPP - tgt) ** 2).sum())
        idx = choose_params(gs, 16, seed=100 + k)
        fd = fd_gradient(gs, render_loss, idx)
        gk = grads[k].cpu().numpy()[idx]
        c = grad_check(gk, fd)
        miss = [j for j in range(len(idx)) if abs(gk[j] - fd[j]) > GRAD_REL_TOL * max(abs(fd[j]), c["abs_floor"])]
        if miss:   # central differences at eps / 2 for the misses (roulette jumps)
            half = np.array(fd)
            half[miss] = fd_gradient(gs, render_loss, [idx[j] for j in miss], eps=EPS / 2)
            c["roulette_misses"] = [dict(m, scene=k) for m in roulette_misses(gk, fd, half, c)]
        checks.append(c)
    extra = {}
    if cpu:
        # SoL's PathTracer on scenes 0 and 1 at their full size and 16 spp.
        cpu_paths, cpu_s, kind = 0.0, 0.0, None
        for k in (0, 1):
            kind, run = cpu_renderer(made[k][0], os.cpu_count() or 1)
            _, t = run(0, SPP, sides[k], sides[k], cfg)
            cpu_paths += sides[k] ** 2 * SPP
            cpu_s += t
        extra["cpu_baseline"] = cpu_baseline(cpu_paths, cpu_s, kind,
                                             f"scenes 0 and 1 at {SPP} spp ({int(cpu_paths)} paths); scene build excluded")
    tris = [i.num_triangles for i in infos]
    cfgd = {"workload": f"{num} independent textured sphere fields ({min(tris)}-{max(tris)} triangles, "
                        f"{sum(tris)} in all), films {min(sides)}^2-{max(sides)}^2, {SPP} spp, fused forward + "
                        f"L2 path-replay adjoint in one launch",
            "scenes": num, "triangles_total": sum(tris), "paths_per_step": int(paths),
            "max_path_len": cfg.max_path_len, "l2": "flushed between steps (256 MiB write)", "small": bool(args.small)}
    return _base(
        args, METRIC, paths / mean["fused"] / 1e3, METRIC, mean["fused"], True, cfgd, clocks.summary(), steps,
        steps, warmup, note="value: paths rendered and differentiated per second by the fused launch",
        forward={k: {"ms": mean[k], "value": paths / mean[k] / 1e3, "vs_plain": mean["plain"] / mean[k]}
                 for k in ("wavefront", "megakernel", "plain")},
        autotune=tune, fused_ms=mean["fused"], fused_over_forward=mean["fused"] / fwd_batched,
        adjoint_over_forward=(mean["fused"] - fwd_batched) / fwd_batched,
        gradient_check={"params_per_scene": 16, "eps": EPS, "tol_rel": GRAD_REL_TOL,
                        "params_within_tol": int(sum(c["within_tol"] for c in checks)),
                        "params_checked": int(sum(c["params"] for c in checks)),
                        "scenes_all_within_tol": int(sum(c["within_tol"] == c["params"] for c in checks)),
                        "max_rel_err_per_scene": [float(f"{c['max_rel_err']:.3g}") for c in checks],
                        "roulette_misses": [m for c in checks for m in c.get("roulette_misses", [])],
                        "worst_scene": int(np.argmax([c["max_rel_err"] for c in checks])),
                        "worst": checks[int(np.argmax([c["max_rel_err"] for c in checks]))]["worst"]},
        e2e={"value": paths / mean["fused"] / 1e3, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        scene_generation_s=gen_s, bvh_build_ms=float(sum(i.build_ms for i in infos)), **extra)


def run_stages(args, ClockSampler, load_peaks, steps=None, warmup=None, cpu=False):
    """One wavefront render of the views workload (or, with --small, 16 views
    of at most 512^2 at 8 spp of the 1M-triangle field) through the
    host-driven bounce loop, which launches the same stage kernels as the
    CUDA graph one by one, so that a profiler lists them (kernels inside a
    graph's WHILE body are not profiled)."""
    import torch
    from sol_b200 import capi, scenes
    from sol_b200.renderer import BatchRenderer, GpuScene
    cfg = scenes.SPHERES_CONFIG
    if args.small:
        scene = scenes.sphere_field(64, seed=1)
        views = [(c, s, 8) for c, s, _ in scenes.view_set(16, seed=2, max_side=512)]
    else:
        scene = scenes.sphere_field(256, seed=1)
        views = scenes.view_set(64, seed=2)
    gs = GpuScene(scene)
    films = [torch.zeros((3, s, s), device="cuda") for _, s, _ in views]
    br = BatchRenderer([gs], capacity=1 << 22, block_size=256, sort_threshold=0, host_loop=True,
                       schedule=capi.BATCH_WAVEFRONT)
    arr = br.views([(0, c, s, s, 0, p, f.data_ptr()) for (c, s, p), f in zip(views, films)])
    br.render(cfg, arr)
    torch.cuda.synchronize()
    st = br.stats()
    return {"metric": "wavefront render through the host-driven loop", "value": st.kernel_ms, "unit": "ms",
            "paths": st.paths, "rays": st.rays, "shadow_rays": st.shadow_rays, "views": len(views),
            "small": bool(args.small), "note": "for profiler launch lists; not a bench number"}


RUNS = {"cornell": run_cornell, "views": run_views, "adjoint": run_adjoint, "scenes": run_scenes,
        "stages": run_stages}


def run(args, ClockSampler, load_peaks) -> int:
    """One workload's full JSON line (bench.py --workload NAME)."""
    import torch
    from sol_b200 import build
    build.build()
    torch.cuda.set_device(0)
    line = RUNS[args.workload](args, ClockSampler, load_peaks)
    print(json.dumps(line), flush=True)
    return 0


def sub_records(args, ClockSampler, load_peaks, steps: int = 5, warmup: int = 3) -> dict:
    """Every other configuration, measured in the default bench run (fewer
    steps each, so that the whole run stays within a few minutes); a record
    that fails carries its error instead."""
    out = {}
    for name, fn in (("cornell", run_cornell), ("views", run_views), ("adjoint", run_adjoint),
                     ("scenes", run_scenes)):
        t0 = time.perf_counter()
        try:
            out[name] = fn(args, ClockSampler, load_peaks, steps=steps, warmup=warmup, cpu=not args.no_cpu_baseline)
        except Exception as e:   # reported in the line, not fatal to the headline
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = time.perf_counter() - t0
    return out
