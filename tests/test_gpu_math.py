"""The device build of the shared pow_ against the host build, bit for bit.

core/math.h is compiled for the host (the CPU checker, SoL's shims) and for
sm_100a (every kernel); the films are bit-identical only if both give the same
bits.  The probe library evaluates pow_ with the kernels' compiler flags."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
from test_math import domains

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def test_device_pow_matches_host_bit_for_bit(built):
    import torch
    probe = C.CDLL(str(ROOT / "sol_b200" / "lib" / "libsol_probe.so"))
    probe.sol_probe_pow.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    probe.sol_probe_pow.restype = C.c_int
    xs, ys = zip(*domains(250_000, seed=7).values())
    edge_x = np.array([0.5, 1.0, 0.0, 0.0, np.inf, 1e-45, 1e-40, 0.999999, 3.0e38, 0.5], np.float32)
    edge_y = np.array([0.0, 7.0, 2.0, -2.0, 2.0, 0.5, 2.0, 1000.0, 2.0, 150.0], np.float32)
    x = np.concatenate(list(xs) + [edge_x])
    y = np.concatenate(list(ys) + [edge_y])
    host = oracle.pow_float(x, y)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    out = torch.empty_like(dx)
    assert probe.sol_probe_pow(dx.data_ptr(), dy.data_ptr(), out.data_ptr(), x.size) == 0
    dev = out.cpu().numpy()
    assert np.array_equal(dev.view(np.uint32), host.view(np.uint32)), \
        f"{np.count_nonzero(dev.view(np.uint32) != host.view(np.uint32))} of {x.size} differ"
