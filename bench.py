"""Benchmark of the B200 path tracer (one JSON line on rank 0).

Workload: the plain per-pixel megakernel on the sphere field of 1,048,576
sphere triangles (+ 2 ground, 8 light triangles), 1920x1080, 64 samples per pixel,
maximum path length 8 -- one step renders that whole frame (132,710,400 paths).
With N GPUs (torchrun) every rank renders its own 64-sample range of the same
frame (weak scaling: independent sample ranges, no collective on the data path).

  value  device-timed Mpaths/s of the render kernel (scene resident on the GPU,
         L2 flushed between steps), summed over ranks
  e2e    Mpaths/s through the C ABI entry point a SoL renderer calls
         (sol_gpu_render with the host film: the film's device->host copy and
         the host-side accumulate are inside the timed region)

`--impl reference` times SoL's own CPU path tracer (oracle/_ref, or the oracle
restatement when SoL's sources were not built) on all host threads instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = {"workload": "one frame per render call, sphere field (64 displaced UV spheres x 16,384 tris + 10), "
                        "1920x1080, 64 spp, max path length 8",
            "triangles": 1048586, "width": 1920, "height": 1080, "spp": 64, "max_path_len": 8,
            "l2": "flushed between steps (256 MiB write)"}
METRIC = "Mpaths/s"
PUBLISHED_VALUE = None   # no published number exists for this metric


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--small", action="store_true", help="quick run on a reduced frame (not a bench number)")
    p.add_argument("--workload", default="frame", choices=["frame", "cornell", "views", "adjoint", "scenes", "stages"],
                   help="frame: one large frame per render call (default; the other configurations are added "
                        "under `configs`); cornell: the Cornell box at 256^2 x 16 spp; views: 64 uneven views of a "
                        "4,194,314-triangle field, batched vs 64 plain launches; adjoint: path-replay adjoint vs "
                        "forward on the textured Cornell box; scenes: fused forward + adjoint over 32 independent "
                        "scenes; stages: one wavefront render of the views workload through the host-driven loop, "
                        "for profiler launch lists")
    p.add_argument("--no-configs", action="store_true", help="frame only: skip the other configurations")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def rank_sample_base(rank: int, spp: int, warmup: int, steps: int) -> int:
    """First sample index of a rank: every rank renders its own sample range of
    the frame (warm-up, timed steps and the end-to-end pass, spp samples each),
    so ranks never render the same path (weak scaling, no collective on the
    data path; summing the films afterwards would give the frame over all
    ranks' samples)."""
    return rank * spp * (warmup + steps + 1)


def reduce_max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time (every rank calls this in the same order)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    """HBM copy bandwidth (GB/s) for the roofline and where it comes from: the
    measured copy in MEASURED_PEAKS.json, else an earlier B200 copy measurement."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback: MEASURED_PEAKS.json absent, 6.65 TB/s copy measured earlier on a B200"


def l2_read_peak_gbs():
    """L2 read bandwidth of this GPU in GB/s: 16-byte L1-bypassing loads over a
    64 MiB buffer that L2 holds, 20 passes per launch, best of 5 launches
    (sol_b200/csrc/probe.cu).  None where the probe library is missing."""
    import ctypes
    lib_path = ROOT / "sol_b200" / "lib" / "libsol_probe.so"
    if not lib_path.exists():
        return None
    lib = ctypes.CDLL(str(lib_path))
    lib.sol_probe_l2_read_gbs.restype = ctypes.c_double
    lib.sol_probe_l2_read_gbs.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
    v = lib.sol_probe_l2_read_gbs(64 << 20, 20, 5)
    return v if v > 0 else None


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def workload_config(small: bool) -> dict:
    """The frame workload's `config` (identical in both arms)."""
    return dict(WORKLOAD, small=True, width=480, height=270, spp=8) if small else dict(WORKLOAD)


def make_workload(small: bool):
    from sol_b200 import scenes
    scene = scenes.sphere_field(64, seed=1)
    w, h, spp = (480, 270, 8) if small else (1920, 1080, 64)
    return scene, scenes.SPHERES_CONFIG, w, h, spp


from bench_workloads import cpu_model, cpu_renderer, single_view_schedules  # noqa: E402  (one definition for every workload)


def cpu_reference_mpaths(scene, cfg, w, h, target_s: float = 12.0, max_spp: int = 64):
    """SoL's own path tracer on all host threads over whole frames; 1 spp first,
    then enough samples for about `target_s` seconds (paths are independent)."""
    threads = os.cpu_count() or 1
    kind, run = cpu_renderer(scene, threads)
    _, t1 = run(0, 1, w, h, cfg)
    spp = int(min(max_spp, max(1, math.floor(target_s / max(t1, 1e-3)))))
    t = run(1, spp, w, h, cfg)[1] if spp > 1 else t1
    paths = w * h * spp
    return {"value": paths / t / 1e6, "unit": METRIC, "cores": threads, "cpu_model": cpu_model(), "kind": kind,
            "sample": f"{spp} spp of the full {w}x{h} frame ({paths} paths) on {threads} threads, "
                      f"{t:.2f} s; BVH build excluded (test/driver.cpp:232 starts the clock after scene load)"}


def run_reference(args):
    """SoL's CPU PathTracer on the same frame: every step renders all spp
    samples of every pixel in one Renderer::render call (the work of one step
    of this library's arm), timed around the call as test/driver.cpp:232-238
    times a render."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    scene, cfg, w, h, spp = make_workload(args.small)
    threads = os.cpu_count() or 1
    kind, run = cpu_renderer(scene, threads)
    for i in range(args.warmup):
        run(i * spp, spp, w, h, cfg)
    times = [run((args.warmup + i) * spp, spp, w, h, cfg)[1] for i in range(args.steps)]
    total = sum(times)
    paths = w * h * spp * args.steps
    value = paths / total / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene)", "config": workload_config(args.small),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "cpu_model": cpu_model(), "kind": kind,
                             "sample": f"{spp} spp of the full {w}x{h} frame per step (one render call), "
                                       f"{args.steps} steps on {threads} threads"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    from sol_b200 import build
    build.build()
    from sol_b200.renderer import GpuPathTracer, GpuScene, Image

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))

    scene, cfg, w, h, spp = make_workload(args.small)
    gscene = GpuScene(scene, device=local)
    info = gscene.info()
    pt = GpuPathTracer(gscene, cfg)
    film = torch.zeros((3, h, w), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    base = rank_sample_base(rank, spp, args.warmup, args.steps)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def reduce_max(x: float) -> float:
        return reduce_max_over_ranks(x, world)

    # Warm-up.
    for i in range(args.warmup):
        pt.render_device(film.data_ptr(), w, h, base + i * spp, spp, stream.cuda_stream)
    barrier()

    # Device-timed steps: L2 flushed before each, render timed with events on its stream.
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        barrier()
        t0 = time.perf_counter()
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            pt.render_device(film.data_ptr(), w, h, base + (args.warmup + i) * spp, spp, stream.cuda_stream)
            ev[i][1].record(stream)
        barrier()
        wall = time.perf_counter() - t0
    kernel_s = sum(a.elapsed_time(b) for a, b in ev) / 1000.0
    kernel_s = reduce_max(kernel_s)
    st = pt.stats()
    rays_per_step = st.rays

    # Algorithmic bytes per launch from the counting variant of the same render.
    gscene.set_instrumented(True)
    pt.render_device(film.data_ptr(), w, h, base, spp, stream.cuda_stream)
    torch.cuda.synchronize()
    ist = pt.stats()
    gscene.set_instrumented(False)
    # Split schedule: each path's colour is written to scratch and read back by the sum pass.
    scratch_bytes = 24.0 * ist.paths if st.sample_chunk > 0 else 0.0
    alg_bytes = 64.0 * ist.nodes_visited + 48.0 * ist.tris_tested + 32.0 * ist.rays + scratch_bytes

    # End to end through the C ABI with the host film.
    img = Image(w, h)
    pt.render(img, base, spp)                     # warm the staging buffers
    barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        pt.render(img, base + i * spp, spp)
    barrier()
    e2e_s = reduce_max(time.perf_counter() - t0)

    from sol_b200 import capi
    import ctypes
    # Per-step inputs: camera, configuration and the sample range, passed by value to the kernel.
    h2d_bytes = ctypes.sizeof(capi.SolGpuCamera) + ctypes.sizeof(capi.SolGpuConfig) + 8 + 4 * 3
    paths = float(w * h * spp)
    value = world * paths * args.steps / kernel_s / 1e6
    e2e = world * paths * args.steps / e2e_s / 1e6
    peak, peak_src = load_peaks()
    achieved = alg_bytes / (kernel_s / args.steps) / 1e9
    traffic = None
    measured = {}
    captured_on = None
    tfile = ROOT / "profiles" / "megakernel_sphere_field_traffic.txt"
    if tfile.exists() and not args.small:
        for line in tfile.read_text().splitlines():
            if line.startswith("# captured on commit:"):
                captured_on = line.split(":", 1)[1].strip()
            elif ":" in line and not line.startswith("#"):
                key, val = line.split(":", 1)
                measured[key.strip()] = float(val)
        traffic = measured.get("dram_bytes_per_launch")
    l2_peak = l2_read_peak_gbs()
    l2_achieved = measured.get("lts_bytes", 0.0) / (kernel_s / args.steps) / 1e9 if measured else None
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * kernel_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None if PUBLISHED_VALUE is None else value / PUBLISHED_VALUE,
            "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": workload_config(args.small),
            "parallelism": f"{world} GPU(s), one {spp}-sample range per rank",
            "mrays_per_s": world * rays_per_step * args.steps / kernel_s / 1e6,
            "rays_per_path": rays_per_step / paths,
            "bytes_per_ray": alg_bytes / ist.rays,
            "ncu_bytes_per_ray": None if not measured else {
                "dram_read": measured.get("dram_bytes_read", 0.0) / ist.rays,
                "dram_write": measured.get("dram_bytes_write", 0.0) / ist.rays,
                "lts": measured.get("lts_bytes", 0.0) / ist.rays,
                "source": "profiles/megakernel_sphere_field_traffic.txt (one-pass ncu capture of a full launch"
                          + (f", build of commit {captured_on})" if captured_on else ")")},
            "achieved_gbs": None if not measured else {
                "dram": (measured.get("dram_bytes_read", 0.0) + measured.get("dram_bytes_write", 0.0))
                        / (kernel_s / args.steps) / 1e9,
                "l2": measured.get("lts_bytes", 0.0) / (kernel_s / args.steps) / 1e9,
                "note": "ncu bytes of one launch over this run's per-launch kernel time"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_src,
                         "l2": None if not (l2_peak and l2_achieved) else {
                             "achieved": l2_achieved, "peak": l2_peak, "unit": "GB/s", "frac": l2_achieved / l2_peak,
                             "peak_source": "measured here: L2-resident 64 MiB read (sol_b200/csrc/probe.cu)",
                             "bytes": "lts__t_bytes.sum of the stored one-pass ncu capture"},
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "note": "per render call (megakernel + in-order sum pass)" if st.sample_chunk > 0
                                 else "per render call (one megakernel launch)"},
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d_bytes,
                    "d2h_bytes_per_step": int(3 * w * h * 4)},
            "gpu_launches": args.steps * st.launches,
            "schedule": ("split: one work item per pixel sample, a warp per sample of an 8x4 pixel tile, "
                         f"{st.sample_chunk}-sample chunks, in-order per-pixel sums (megakernel + sum pass)")
                        if st.sample_chunk > 0 else "per pixel: one lane per pixel for all its samples (megakernel)",
            "clocks": clocks.summary(),
            "wall_s_timed_region": wall,
            "scene": {"triangles": info.num_triangles, "bvh_inner_nodes": info.num_nodes,
                      "bvh_depth": info.bvh_depth, "sah_cost": info.sah_cost,
                      "device_mb": info.device_bytes / 2**20, "build_ms": info.build_ms},
        }
    if rank == 0 and world == 1 and not args.small and not args.no_configs:
        # The batch schedules on this one view, for comparison with the plain launch.
        line["batched"] = single_view_schedules(gscene, cfg, scene.camera, w, h, spp,
                                                1000.0 * kernel_s / args.steps, 5, 3)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_reference_mpaths(scene, cfg, w, h)
            except Exception as e:   # reported, not fatal
                line["cpu_baseline"] = {"value": None, "error": str(e)}
        if world == 1 and not args.no_configs and not args.small:
            # The other configurations, each with its own clocks, roofline and CPU baseline.
            import bench_workloads
            del gscene, pt, film, flush
            torch.cuda.empty_cache()
            line["configs"] = bench_workloads.sub_records(args, ClockSampler, load_peaks)
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.workload != "frame":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the CPU reference arm covers the frame workload"}))
            return 0
        if dist_env()[1] > 1:
            raise SystemExit("the views/adjoint/scenes workloads run on one GPU")
        import bench_workloads
        return bench_workloads.run(args, ClockSampler, load_peaks)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
