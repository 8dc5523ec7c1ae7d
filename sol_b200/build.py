"""Builds the CUDA library `sol_b200/lib/libsol_gpu.so` in-tree with nvcc.

Device code is compiled for sm_100a only, with FMA contraction off and IEEE
division/square root, so that the shared math produces the same bits as the host
checker (explicit FMAs in the box tests are unaffected).  Host code is compiled
with -ffp-contract=off for the same reason.  The CUDA runtime is linked
statically, so the library only needs the driver at run time.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
BUILD_DIR = PKG / "_build"
LIB = LIB_DIR / "libsol_gpu.so"
PROBE_LIB = LIB_DIR / "libsol_probe.so"   # memory probes for the roofline (bench only)

CUDA_SOURCES = ["kernels/megakernel.cu", "kernels/trace.cu", "kernels/wavefront.cu", "kernels/adjoint.cu",
                "kernels/lbvh.cu", "noalloc.cu"]
HOST_SOURCES = ["capi.cpp", "batch.cpp", "job.cpp", "host/flatten.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_DEVICE = ARCH + ["-O3", "-lineinfo", "-std=c++20", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
                      "-Xptxas", "-v", "-Xcompiler", "-fPIC,-ffp-contract=off,-O3"]
HOST_FLAGS = ["-O3", "-std=c++20", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall", "-Wno-unknown-pragmas"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build sol_b200")
    return cand


def _inputs() -> list[Path]:
    files = [p for p in CSRC.rglob("*") if p.suffix in (".cu", ".cuh", ".h", ".cpp")]
    files.append(ROOT / "include" / "sol_gpu.h")
    files.append(Path(__file__))
    return files


def up_to_date() -> bool:
    if not LIB.exists() or not PROBE_LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _inputs())


def _run(cmd: list[str], log: Path | None = None) -> str:
    r = subprocess.run(cmd, capture_output=True, text=True)
    out = r.stdout + r.stderr
    if log is not None:
        log.write_text(" ".join(cmd) + "\n" + out)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{out}")
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the library if any source is newer than it; returns its path."""
    if not force and up_to_date():
        return LIB
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    inc = ["-I", str(CSRC), "-I", str(ROOT / "include")]
    jobs = []
    for src in CUDA_SOURCES:
        obj = BUILD_DIR / (Path(src).stem + ".o")
        cmd = [cc, "-c", str(CSRC / src), "-o", str(obj)] + NVCC_DEVICE + inc
        jobs.append((cmd, obj, BUILD_DIR / (Path(src).stem + ".ptxas.log")))
    for src in HOST_SOURCES:
        obj = BUILD_DIR / (Path(src).stem + ".o")
        cmd = ["g++", "-c", str(CSRC / src), "-o", str(obj), "-I/usr/local/cuda/include"] + HOST_FLAGS + \
              ["-I", str(CSRC), "-I", str(ROOT / "include")]
        jobs.append((cmd, obj, None))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        futs = [ex.submit(_run, cmd, log) for cmd, _, log in jobs]
        for f in futs:
            out = f.result()
            if verbose and out:
                print(out)
    link = [cc, "-shared", "-o", str(LIB)] + [str(o) for _, o, _ in jobs] + ARCH + \
           ["-Xcompiler", "-fopenmp", "-lgomp"]
    _run(link)
    _run([cc, "-shared", "-o", str(PROBE_LIB), str(CSRC / "probe.cu")] + NVCC_DEVICE + ["-Xcompiler", "-fPIC"])
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(path)
