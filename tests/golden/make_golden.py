"""Regenerates the golden fixtures in this directory from SoL's own code.

  pcg_kat.json      draws of SoL's PcgSampler (include/sol/samplers.h) for a few
                    seeds, in call order, from a program that includes SoL's
                    header unmodified and is compiled here with g++;
  render_*.npz      films rendered by SoL's own PathTracer (src/algorithms/path_tracer.cpp
                    and the classes it uses, built by oracle/Makefile against the
                    clean-room proto/par/bvh shims) on small seeded scenes.

Needs SoL's sources in $SOL_REF_DIR (by default the directory `reference`
beside the repository's root); run from the repo root:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
SOL = Path(os.environ.get("SOL_REF_DIR") or ROOT.parent / "reference")

PCG_SEEDS = [0, 1, 42, 0xDEADBEEF, 2**32 - 1, 123456789]
PCG_DRAWS = 64

KAT_PROGRAM = r"""
#include "sol/samplers.h"
#include <cstdio>
#include <cstdlib>
int main(int argc, char** argv) {
    for (int a = 2; a < argc; ++a) {
        unsigned long long seed = std::strtoull(argv[a], nullptr, 10);
        sol::PcgSampler s(seed);
        std::printf("%llu", seed);
        int n = std::atoi(argv[1]);
        for (int i = 0; i < n; ++i) { float f = s(); std::printf(" %a", f); }
        std::printf("\n");
    }
}
"""

# (name, scene factory, config, width, height, spp, sample_index)
RENDERS = [
    ("render_cornell_32x32_s4", "cornell", 32, 32, 4, 0),
    ("render_cornell_24x16_s3_i7", "cornell", 24, 16, 3, 7),
    ("render_cornell_textured_32x32_s2", "cornell_textured", 32, 32, 2, 0),
    ("render_spheres_48x27_s2", "spheres", 48, 27, 2, 0),
]


def scene_for(kind: str):
    from sol_b200 import scenes
    if kind == "cornell":
        return scenes.cornell_box(0), scenes.CORNELL_CONFIG
    if kind == "cornell_textured":
        return scenes.cornell_box(0, textured=True, tex_size=64), scenes.CORNELL_CONFIG
    if kind == "spheres":
        return scenes.sphere_field(8, seed=1, bands=17, segments=32), scenes.SPHERES_CONFIG
    raise ValueError(kind)


def make_pcg_kat() -> None:
    with tempfile.TemporaryDirectory() as tmp:
        src = Path(tmp) / "kat.cpp"
        exe = Path(tmp) / "kat"
        src.write_text(KAT_PROGRAM)
        subprocess.run(["g++", "-std=c++20", "-O2", f"-I{SOL / 'include'}", str(src), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe), str(PCG_DRAWS)] + [str(s) for s in PCG_SEEDS], check=True,
                             capture_output=True, text=True).stdout
    kat = {}
    for line in out.strip().splitlines():
        parts = line.split()
        kat[parts[0]] = parts[1:]
    (HERE / "pcg_kat.json").write_text(json.dumps({"generator": "sol::PcgSampler from include/sol/samplers.h",
                                                   "draws": kat}, indent=1) + "\n")


def make_renders() -> None:
    import oracle
    oracle.build(ref=True)
    for name, kind, w, h, spp, index in RENDERS:
        scene, cfg = scene_for(kind)
        film, _ = oracle.RefScene(scene).render(cfg, w, h, spp, sample_index=index)
        np.savez_compressed(HERE / f"{name}.npz", film=film, kind=kind, width=w, height=h, spp=spp,
                            sample_index=index)


if __name__ == "__main__":
    make_pcg_kat()
    make_renders()
    print("golden fixtures written to", HERE)
