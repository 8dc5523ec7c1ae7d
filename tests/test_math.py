"""The shared pow_ (sol_b200/csrc/core/math.h), on the host.

SoL's Phong BSDF (src/bsdfs.cpp:102-104) and the cosine-power warps it calls
through proto take x^y with x a cosine in [0, 1] and y the Phong exponent or
1/(exponent + 1).  pow_ evaluates e^(y ln x) in double precision with tables
and short series; these tests hold its float result to the correctly rounded
value (x^y in double, rounded once to float) on those domains and a wide one,
check the special cases of C's pow for non-negative bases, and check that the
committed constant tables are the ones their generator computes.  The device
build of the same source is compared with this host build bit for bit in
tests/test_gpu_math.py."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle

ROOT = Path(__file__).resolve().parent.parent
N = 1_000_000


def _rounded(x, y):
    with np.errstate(all="ignore"):
        return (x.astype(np.float64) ** y.astype(np.float64)).astype(np.float32)


def domains(n=N, seed=1):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(0.0, np.log(1000.0), n))
    return {
        "cosine^exponent": (rng.random(n).astype(np.float32), ns.astype(np.float32)),
        "sample^(1/(exponent+1))": (rng.random(n).astype(np.float32), (1.0 / (ns + 1.0)).astype(np.float32)),
        "Cornell exponent 64": (rng.random(n).astype(np.float32), np.full(n, 64.0, np.float32)),
        "wide": (np.exp(rng.uniform(-80.0, 80.0, n)).astype(np.float32), rng.uniform(-3.0, 3.0, n).astype(np.float32)),
    }


@pytest.mark.parametrize("name", list(domains(8)))
def test_pow_is_correctly_rounded(built, name):
    x, y = domains()[name]
    got = oracle.pow_float(x, y)
    want = _rounded(x, y)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), \
        f"{np.count_nonzero(got != want)} of {x.size} differ"


def test_pow_special_cases(built):
    inf, nan = np.float32(np.inf), np.float32(np.nan)
    x = np.array([0.5, 1.0, 0.0, 0.0, 0.0, inf, inf, -0.5, nan, 0.5, 0.7, 1e-45, 1e-40, 3.0e38], np.float32)
    y = np.array([0.0, 123.0, 2.0, -2.0, 0.0, 2.0, -2.0, 2.0, 2.0, nan, 1000.0, 0.5, 2.0, 2.0], np.float32)
    got = oracle.pow_float(x, y)
    want = np.array([1.0, 1.0, 0.0, inf, 1.0, inf, 0.0, nan, nan, nan, _rounded(x[10:11], y[10:11])[0],
                     _rounded(x[11:12], y[11:12])[0], 0.0, inf], np.float32)
    same = (got == want) | (np.isnan(got) & np.isnan(want))
    assert same.all(), list(zip(x[~same], y[~same], got[~same], want[~same]))


def test_pow_tables_match_their_generator():
    gen = ROOT / "sol_b200" / "csrc" / "core" / "gen_pow_tables.py"
    assert subprocess.run([sys.executable, str(gen), "--check"]).returncode == 0
