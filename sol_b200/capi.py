"""ctypes binding of the C ABI in include/sol_gpu.h.

The library is loaded from `sol_b200/lib/libsol_gpu.so`, built in-tree by
`sol_b200/build.py`.  There is no fallback: if the library is missing the import
of this module fails with an explanation.  The declarations (structures, enum
values, signatures) live in `sol_b200.abi`, which loads nothing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .abi import *  # noqa: F401,F403  (the ABI's names are part of this module's interface)
from .abi import SIGNATURES

# SOL_B200_LIBRARY selects another build of the library (e.g. a tuning variant).
LIB_PATH = Path(os.environ.get("SOL_B200_LIBRARY") or Path(__file__).resolve().parent / "lib" / "libsol_gpu.so")


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m sol_b200.build` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class SolGpuError(RuntimeError):
    def __init__(self, code: int, what: str):
        msg = lib.sol_gpu_last_error().decode(errors="replace")
        super().__init__(f"{what} failed with status {code}: {msg}")
        self.code = code


def check(code: int, what: str) -> None:
    if code != OK:
        raise SolGpuError(code, what)
