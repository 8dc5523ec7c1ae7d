"""The multi-rank path of bench.py on CPU: two gloo ranks (127.0.0.1).

Each rank renders its own sample range (bench.rank_sample_base) — here with
the CPU checker standing in for the GPU renderer — the ranges are disjoint,
the slowest rank's time is what reduce_max_over_ranks returns on every rank,
and the films summed over ranks equal one render of all ranks' samples."""
import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    import bench
    import oracle
    from sol_b200 import scenes
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    spp, warmup, steps = 2, 1, 2
    base = bench.rank_sample_base(rank, spp, warmup, steps)
    ranges = [None] * world
    dist.all_gather_object(ranges, (base, base + spp * (warmup + steps + 1)))
    scene, cfg = scenes.cornell_box(0), scenes.CORNELL_CONFIG
    film = oracle.render(scene, cfg, 16, 12, spp, sample_index=base)
    t = torch.from_numpy(film.copy())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    slowest = bench.reduce_max_over_ranks(float(rank + 1) * 0.5, world, device="cpu")
    if rank == 0:
        np.savez(os.path.join(out_dir, "r0.npz"), summed=t.numpy(), ranges=np.asarray(ranges), slowest=slowest)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_samples_and_reduce(tmp_path, built):
    import torch.multiprocessing as mp
    import oracle
    from sol_b200 import scenes
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r = np.load(tmp_path / "r0.npz")
    (a0, a1), (b0, b1) = r["ranges"]
    assert a1 <= b0 or b1 <= a0                       # disjoint sample ranges
    assert float(r["slowest"]) == 1.0                 # max over ranks, seen by rank 0
    scene, cfg = scenes.cornell_box(0), scenes.CORNELL_CONFIG
    ref = oracle.render(scene, cfg, 16, 12, 2, sample_index=int(a0))
    ref = oracle.render(scene, cfg, 16, 12, 2, sample_index=int(b0), film=ref)
    assert np.allclose(r["summed"], ref, rtol=1e-6, atol=1e-7)
