"""The multi-view, adjoint and multi-scene measurements of bench.py (one GPU).

  views    64 seeded views (square side log-uniform 64-1024, 1-64 spp) of a
           4,194,314-triangle sphere field (256 displaced spheres), rendered by
           the batched wavefront in one call against 64 plain megakernel
           launches.  Both give bit-identical films (same estimator, same
           seeds), so their RMSE is equal; it is reported against a 256-spp
           render of every view.
  adjoint  the textured Cornell box (two 256x256 RGB albedo images): forward
           render 128x128 x 16 spp, then the L2 loss against a 1024-spp target
           and the path-replay adjoint; the ratio adjoint / forward time is the
           value.  The gradient is checked against central finite differences
           (eps 1e-3, common random numbers) of the GPU forward on 64 seeded
           parameters.
  scenes   32 independent textured sphere fields (10k-2M triangles, films
           128^2-512^2, 16 spp): forward + L2 adjoint of all 32 in one fused
           launch, against the forward alone; gradients checked per scene
           against finite differences on 16 parameters.

Every timed launch is preceded by a 256 MiB write that flushes L2, and timed
with CUDA events on the launching stream.
"""
from __future__ import annotations

import json
import math
import time

import numpy as np

METRIC = "Mpaths/s"
EPS = 1e-3


def _events(torch, n):
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def _ms(evs):
    return [a.elapsed_time(b) for a, b in evs]


def _timed(torch, flush, stream, fn, steps, warmup, clocks=None):
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
    return _ms(ev)


def _rel_err(g, fd):
    g = np.asarray(g, np.float64)
    fd = np.asarray(fd, np.float64)
    den = float(np.linalg.norm(fd))
    return float(np.linalg.norm(g - fd) / den) if den > 0 else float(np.linalg.norm(g))


def _fd_gradient(torch, gs, render_loss, indices):
    """Central differences (eps 1e-3) of render_loss() over the given parameter indices."""
    base = gs.get_params()
    out = []
    for j in indices:
        v = base.copy()
        v[j] = base[j] + EPS
        gs.set_params(v)
        lp = render_loss()
        v[j] = base[j] - EPS
        gs.set_params(v)
        lm = render_loss()
        out.append((lp - lm) / (2.0 * EPS))
    gs.set_params(base)
    return np.asarray(out)


def _common(args, metric, value, unit, ms, hib, config, clocks, launches, **extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scenes)", "config": config, "gpu_launches": launches,
            "clocks": clocks}
    line.update(extra)
    return line


# ---------------------------------------------------------------------------
# views: batched wavefront vs plain megakernel launches
# ---------------------------------------------------------------------------

def run_views(args, ClockSampler, load_peaks):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
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

    from sol_b200 import capi
    br = BatchRenderer([gs], schedule=capi.BATCH_AUTO)        # autotuned: wavefront or multi-view megakernel
    br_wf = BatchRenderer([gs], schedule=capi.BATCH_WAVEFRONT)

    def varr(i, fl=None, r=None):
        fl = fl or films
        return (r or br).views([(0, cam, s, s, i * 64, p, f.data_ptr()) for (cam, s, p), f in zip(views, fl)])

    t0 = time.perf_counter()
    opts = br.autotune(cfg, varr(0))
    tune_s = time.perf_counter() - t0
    opts_wf = br_wf.autotune(cfg, varr(0, r=br_wf))
    arrays = {i: varr(i) for i in range(args.warmup + args.steps)}
    arrays_wf = {i: varr(i, r=br_wf) for i in range(args.warmup + args.steps)}

    def batched(i):
        br.render(cfg, arrays[i], sp)

    def wavefront(i):
        br_wf.render(cfg, arrays_wf[i], sp)

    with ClockSampler(torch.cuda.current_device()) as clocks:
        plain_ms = _timed(torch, flush, stream, plain, args.steps, args.warmup)
        batch_ms = _timed(torch, flush, stream, batched, args.steps, args.warmup)
        wf_ms = _timed(torch, flush, stream, wavefront, args.steps, args.warmup)
    plain_s, batch_s, wf_s = sum(plain_ms) / 1000.0, sum(batch_ms) / 1000.0, sum(wf_ms) / 1000.0

    # Same films from both schedules (one fresh render each).
    fa = [torch.zeros_like(f) for f in films]
    fb = [torch.zeros_like(f) for f in films]
    for (cam, s, p), pt, f in zip(views, tracers, fa):
        pt.render_device(f.data_ptr(), s, s, 0, p, sp)
    br.render(cfg, varr(0, fb), sp)
    fc = [torch.zeros_like(f) for f in films]
    br_wf.render(cfg, varr(0, fc, br_wf), sp)
    torch.cuda.synchronize()
    identical = all(torch.equal(a, b) and torch.equal(a, c) for a, b, c in zip(fa, fb, fc))

    # RMSE of each schedule's images against a 256-spp render of every view.
    gt_spp = 256
    rmse_a, rmse_b = [], []
    for (cam, s, p), pt, a, b in zip(views, tracers, fa, fb):
        g = torch.zeros_like(a)
        pt.render_device(g.data_ptr(), s, s, 1 << 20, gt_spp, sp)
        torch.cuda.synchronize()
        g /= gt_spp
        rmse_a.append(float(torch.sqrt(torch.mean((a / p - g) ** 2))))
        rmse_b.append(float(torch.sqrt(torch.mean((b / p - g) ** 2))))

    # Algorithmic bytes of the same rays (counting build of the megakernel, one view at a time).
    gs.set_instrumented(True)
    nodes = tris = rays = 0
    for (cam, s, p), pt in zip(views, tracers):
        tmp = torch.zeros((3, s, s), device="cuda")
        pt.render_device(tmp.data_ptr(), s, s, 0, p, sp)
        torch.cuda.synchronize()
        st = pt.stats()
        nodes, tris, rays = nodes + st.nodes_visited, tris + st.tris_tested, rays + st.rays
    gs.set_instrumented(False)
    alg = 64.0 * nodes + 48.0 * tris + 32.0 * rays

    # End to end: view table built and uploaded, films read back to pinned host memory.
    host = [torch.empty(f.shape, dtype=torch.float32, pin_memory=True) for f in films]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        br.render(cfg, varr(100 + i), sp)
        for h_, f in zip(host, films):
            h_.copy_(f, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    peak, src = load_peaks()
    achieved = alg / (batch_s / args.steps) / 1e9
    import ctypes
    cfgd = {"workload": f"{len(views)} uneven views (side log-U[64,{views and max(s for _, s, _ in views)}], "
                        f"1-64 spp) of a {info.num_triangles}-triangle sphere field, batched (one call, autotuned "
                        f"schedule) vs {len(views)} plain megakernel launches",
            "triangles": info.num_triangles, "views": len(views), "paths_per_step": int(paths),
            "pixels": int(sum(s * s for _, s, _ in views)), "max_path_len": cfg.max_path_len,
            "l2": "flushed between steps (256 MiB write); scene larger than L2",
            "batch_options": {"schedule": ["wavefront", "megakernel", "auto"][opts.schedule],
                              "capacity": opts.capacity, "block_size": opts.block_size,
                              "sort_threshold": opts.sort_threshold},
            "wavefront_options": {"capacity": opts_wf.capacity, "block_size": opts_wf.block_size,
                                  "sort_threshold": opts_wf.sort_threshold}, "small": bool(small)}
    return _common(
        args, METRIC, paths * args.steps / batch_s / 1e6, METRIC, 1000.0 * batch_s / args.steps, True, cfgd,
        clocks.summary(), args.steps,
        launch_note="per batched step: one call (one megakernel launch, or the wavefront's stage kernels in a CUDA "
                    "graph); per plain step: one launch per view",
        plain={"value": paths * args.steps / plain_s / 1e6, "unit": METRIC,
               "ms_per_step": 1000.0 * plain_s / args.steps, "launches_per_step": len(views)},
        speedup_vs_plain=plain_s / batch_s,
        wavefront={"value": paths * args.steps / wf_s / 1e6, "unit": METRIC, "ms_per_step": 1000.0 * wf_s / args.steps,
                   "speedup_vs_plain": plain_s / wf_s},
        equal_rmse={"films_bit_identical": identical, "reference": f"{gt_spp}-spp megakernel render per view",
                    "rmse_plain_mean": float(np.mean(rmse_a)), "rmse_batched_mean": float(np.mean(rmse_b))},
        roofline={"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                  "traffic": None, "peak_source": src,
                  "algorithmic_bytes_per_launch": alg},
        e2e={"value": paths * args.steps / e2e_s / 1e6, "unit": METRIC,
             "h2d_bytes_per_step": len(views) * ctypes.sizeof(capi.SolGpuView) + ctypes.sizeof(capi.SolGpuConfig),
             "d2h_bytes_per_step": int(sum(f.numel() * 4 for f in films))},
        autotune_s=tune_s,
        scene={"triangles": info.num_triangles, "bvh_inner_nodes": info.num_nodes, "bvh_depth": info.bvh_depth,
               "device_mb": info.device_bytes / 2**20, "build_ms": info.build_ms})


# ---------------------------------------------------------------------------
# adjoint: path-replay adjoint vs forward on the textured Cornell box
# ---------------------------------------------------------------------------

def _choose_params(gs, n, seed, scalars=False):
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


def run_adjoint(args, ClockSampler, load_peaks):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene, image_l2
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
    gs = GpuScene(scenes.cornell_box(0, textured=True, tex_size=tex, tex_seed=11))
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
        f_ms = _timed(torch, flush, stream, forward, args.steps, args.warmup)
        a_ms = _timed(torch, flush, stream, adjoint, args.steps, args.warmup)
        x_ms = _timed(torch, flush, stream, fused, args.steps, args.warmup)
    fwd, adj, fus = np.mean(f_ms), np.mean(a_ms), np.mean(x_ms)

    # Gradient check at one sample range against central differences of the GPU forward.
    film.zero_()
    grad.zero_()
    loss.zero_()
    forward(7)
    adjoint(7)
    torch.cuda.synchronize()
    g = grad.cpu().numpy()

    def render_loss():
        f = torch.zeros((3, H, W), device="cuda")
        pt.render_device(f.data_ptr(), W, H, 7 * SPP, SPP, sp)
        torch.cuda.synchronize()
        return float(((f.double() / SPP - target.double()) ** 2).sum())

    idx = _choose_params(gs, 64, seed=5)
    fd = _fd_gradient(torch, gs, render_loss, idx)
    err = _rel_err(g[idx], fd)
    # Paths are the unit for the time-per-path figures.
    paths = float(W * H * SPP)
    cfgd = {"workload": f"textured Cornell box ({tex}x{tex} RGB albedo images on back wall and floor), "
                        f"{W}x{H} x {SPP} spp loss render, max path length {cfg.max_path_len}",
            "params": count, "width": W, "height": H, "spp": SPP, "target_spp": 1024,
            "l2": "flushed between steps (256 MiB write)", "small": bool(args.small)}
    return _common(
        args, "PRB adjoint / forward time", adj / fwd, "ratio", adj, False, cfgd, clocks.summary(), 2 * args.steps,
        forward_ms=fwd, adjoint_ms=adj, fused_ms=fus, fused_over_forward=fus / fwd,
        forward_mpaths_s=paths / fwd / 1e3, adjoint_mpaths_s=paths / adj / 1e3,
        gradient_check={"params": len(idx), "eps": EPS, "rel_err_vs_gpu_fd": err,
                        "nonzero_fd": int(np.count_nonzero(fd))},
        e2e={"value": adj / fwd, "unit": "ratio", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})


# ---------------------------------------------------------------------------
# scenes: fused forward + adjoint over 32 scenes in one launch
# ---------------------------------------------------------------------------

def run_scenes(args, ClockSampler, load_peaks):
    import torch
    from sol_b200 import scenes
    from sol_b200.renderer import BatchRenderer, GpuPathTracer, GpuScene
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

    def varr(i):
        return br.views([(k, made[k][0].camera, s, s, i * SPP, SPP, films[k].data_ptr())
                         for k, s in enumerate(sides)])
    opts = br.autotune(cfg, varr(0))
    arrays = {i: varr(i) for i in range(args.warmup + args.steps)}
    from sol_b200 import capi
    br_mk = BatchRenderer(gss, schedule=capi.BATCH_MEGAKERNEL)
    arrays_mk = {i: br_mk.views([(k, made[k][0].camera, s, s, i * SPP, SPP, films[k].data_ptr())
                                 for k, s in enumerate(sides)]) for i in range(args.warmup + args.steps)}

    def batched(i):
        br.render(cfg, arrays[i], sp)

    def batched_mk(i):
        br_mk.render(cfg, arrays_mk[i], sp)

    def plain(i):
        for pt, s, f in zip(tracers, sides, films):
            pt.render_device(f.data_ptr(), s, s, i * SPP, SPP, sp)

    with ClockSampler(torch.cuda.current_device()) as clocks:
        x_ms = _timed(torch, flush, stream, fused, args.steps, args.warmup)
        b_ms = _timed(torch, flush, stream, batched, args.steps, args.warmup)
        m_ms = _timed(torch, flush, stream, batched_mk, args.steps, args.warmup)
        p_ms = _timed(torch, flush, stream, plain, args.steps, args.warmup)
    fus, bat, bmk, pla = np.mean(x_ms), np.mean(b_ms), np.mean(m_ms), np.mean(p_ms)
    fwd = min(bat, bmk, pla)

    # Per-scene gradient check: 16 parameters against central differences of the forward.
    for f in films:
        f.zero_()
    for g in grads:
        g.zero_()
    losses.zero_()
    fused(3)
    torch.cuda.synchronize()
    errs = []
    worst = None
    for k, (gs, pt, s) in enumerate(zip(gss, tracers, sides)):
        def render_loss(pt=pt, s=s, k=k):
            f = torch.zeros((3, s, s), device="cuda")
            pt.render_device(f.data_ptr(), s, s, 3 * SPP, SPP, sp)
            torch.cuda.synchronize()
            return float(((f.double() / SPP - targets[k].double()) ** 2).sum())
        idx = _choose_params(gs, 16, seed=100 + k)
        fd = _fd_gradient(torch, gs, render_loss, idx)
        gk = grads[k].cpu().numpy()[idx]
        errs.append(_rel_err(gk, fd))
        if errs[-1] >= max(errs):
            worst = {"scene": k, "params": idx, "adjoint": [float(f"{x:.5g}") for x in gk],
                     "fd": [float(f"{x:.5g}") for x in fd]}
    tris = [i.num_triangles for i in infos]
    cfgd = {"workload": f"{num} independent textured sphere fields ({min(tris)}-{max(tris)} triangles, "
                        f"{sum(tris)} in all), films {min(sides)}^2-{max(sides)}^2, {SPP} spp, fused forward + "
                        f"L2 path-replay adjoint in one launch",
            "scenes": num, "triangles_total": sum(tris), "paths_per_step": int(paths),
            "max_path_len": cfg.max_path_len, "l2": "flushed between steps (256 MiB write)",
            "batch_options": {"capacity": opts.capacity, "block_size": opts.block_size,
                              "sort_threshold": opts.sort_threshold}, "small": bool(args.small)}
    return _common(
        args, METRIC, paths / fus / 1e3, METRIC, fus, True, cfgd, clocks.summary(), args.steps,
        note="value: paths rendered and differentiated per second by the fused launch",
        forward_ms={"batched_wavefront": bat, "batched_megakernel": bmk, "plain_megakernel_launches": pla},
        fused_ms=fus, fused_over_forward=fus / fwd, adjoint_over_forward=(fus - fwd) / fwd,
        gradient_check={"params_per_scene": 16, "eps": EPS, "rel_err_max": float(np.max(errs)),
                        "rel_err_median": float(np.median(errs)),
                        "scenes_within_2pct": int(np.sum(np.asarray(errs) <= 0.02)),
                        "rel_err_per_scene": [float(f"{e:.3g}") for e in errs],
                        "worst": worst},
        e2e={"value": paths / fus / 1e3, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        scene_generation_s=gen_s, bvh_build_ms=float(sum(i.build_ms for i in infos)))


def run(args, ClockSampler, load_peaks) -> int:
    import torch
    from sol_b200 import build
    build.build()
    torch.cuda.set_device(0)
    fn = {"views": run_views, "adjoint": run_adjoint, "scenes": run_scenes}[args.workload]
    line = fn(args, ClockSampler, load_peaks)
    print(json.dumps(line), flush=True)
    return 0
