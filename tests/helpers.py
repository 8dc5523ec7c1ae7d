"""Shared helpers for the tests."""
from __future__ import annotations

import numpy as np


def rel_diff(a: np.ndarray, b: np.ndarray, floor: float = 1e-6) -> np.ndarray:
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def per_pixel_parity(gpu: np.ndarray, ref: np.ndarray, tol: float = 1e-4):
    """Returns (fraction of pixels bit-identical, number of pixels above `tol` relative)."""
    exact = float(np.mean(np.all(gpu == ref, axis=0)))
    bad = int(np.sum(np.any(rel_diff(gpu, ref) > tol, axis=0)))
    return exact, bad


def random_rays(n: int, lo, hi, seed: int = 0) -> np.ndarray:
    """(n, 8) rays [org, tmin, dir, tmax] with origins in the box and random directions."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    org = lo + (hi - lo) * rng.random((n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = org
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = 3.4e38
    return rays
