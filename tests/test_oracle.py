"""The CPU checker against SoL's own code: PCG known-answer vectors from SoL's
samplers.h, golden films from SoL's PathTracer, and (where SoL's sources were
built here) a direct comparison with SoL's PathTracer."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import per_pixel_parity
from sol_b200 import scenes

GOLDEN = Path(__file__).resolve().parent / "golden"


def kat():
    return json.loads((GOLDEN / "pcg_kat.json").read_text())["draws"]


def test_pcg_matches_sol_samplers_kat(built):
    for seed, draws in kat().items():
        expect = np.array([float.fromhex(x) for x in draws], np.float32)
        got = oracle.pcg_floats(int(seed), len(draws))
        assert np.array_equal(got.view(np.uint32), expect.view(np.uint32)), seed


def test_scene_rng_matches_sol_samplers_kat():
    for seed, draws in kat().items():
        rng = scenes.Pcg(int(seed))
        got = np.array([rng() for _ in draws], np.float32)
        expect = np.array([float.fromhex(x) for x in draws], np.float32)
        assert np.array_equal(got, expect), seed


def test_pcg_seed_42_first_draws():
    # SoL's PcgSampler(42) in call order (from the probe of samplers.h).
    expect = np.array([0.131703794, 0.755355299, 0.583140016], np.float32)
    assert np.allclose(oracle.pcg_floats(42, 3), expect, rtol=0, atol=1e-9)


def test_pixel_seed_is_fnv1a_of_le_bytes(built):
    def fnv(vals):
        h = 2166136261
        for v in vals:
            for i in range(8):
                h ^= (v >> (8 * i)) & 0xFF
                h = (h * 16777619) & 0xFFFFFFFF
        return h
    fxy = np.array([[0, 0, 0], [1, 2, 3], [63, 1919, 1079], [2**40, 7, 9]], np.uint64)
    got = oracle.pixel_seeds(fxy)
    for (f, x, y), g in zip(fxy.tolist(), got.tolist()):
        assert g == fnv([x, y, f])


@pytest.mark.parametrize("path", sorted(GOLDEN.glob("render_*.npz")), ids=lambda p: p.stem)
def test_oracle_matches_sol_golden_films(built, path):
    import sys
    sys.path.insert(0, str(GOLDEN))
    from make_golden import scene_for
    g = np.load(path)
    scene, cfg = scene_for(str(g["kind"]))
    film = oracle.render(scene, cfg, int(g["width"]), int(g["height"]), int(g["spp"]), int(g["sample_index"]))
    exact, bad = per_pixel_parity(film, g["film"])
    assert bad == 0
    assert exact >= 0.99


@pytest.mark.skipif(not oracle.ref_available(), reason="SoL's sources are not built here")
def test_oracle_matches_sol_pathtracer_cornell(built):
    scene, cfg, *_ = scenes.cornell_frame()
    a = oracle.render(scene, cfg, 64, 64, 4)
    b, _ = oracle.RefScene(scene).render(cfg, 64, 64, 4)
    exact, bad = per_pixel_parity(a, b)
    assert bad == 0 and exact >= 0.999


@pytest.mark.skipif(not oracle.ref_available(), reason="SoL's sources are not built here")
def test_oracle_matches_sol_pathtracer_accumulation(built):
    """render(0, 2) then render(2, 3) on one film equals SoL doing the same."""
    scene, cfg, *_ = scenes.cornell_frame()
    a = oracle.render(scene, cfg, 16, 16, 2, 0)
    a = oracle.render(scene, cfg, 16, 16, 3, 2, film=a)
    ref = oracle.RefScene(scene)
    b, _ = ref.render(cfg, 16, 16, 2, 0)
    b, _ = ref.render(cfg, 16, 16, 3, 2, film=b)
    exact, bad = per_pixel_parity(a, b)
    assert bad == 0 and exact >= 0.99


@pytest.mark.skipif(not oracle.ref_available(), reason="SoL's sources were not built into oracle/_ref")
def test_reference_library_links_nothing_of_the_product():
    """The timed CPU reference (SoL's PathTracer in libsol_ref.so) must not map
    the product library: its dynamic section needs no libsol_gpu.so, and
    building a scene for it loads no CUDA library into the process."""
    import subprocess
    import sys
    out = subprocess.run(["readelf", "-d", str(oracle.REF_LIB)], capture_output=True, text=True, check=True).stdout
    needed = [l for l in out.splitlines() if "(NEEDED)" in l]
    assert needed and not any("sol_gpu" in l or "cuda" in l.lower() for l in needed), needed
    code = ("import sys; sys.path.insert(0, '.'); import oracle; from sol_b200 import scenes; "
            "s = scenes.cornell_box(0); r = oracle.RefScene(s); r.render(scenes.CORNELL_CONFIG, 8, 8, 1); "
            "maps = open('/proc/self/maps').read(); "
            "assert 'libsol_gpu' not in maps and 'libcuda' not in maps, 'product library mapped'; "
            "assert 'sol_b200.capi' not in sys.modules")
    subprocess.run([sys.executable, "-c", code], check=True, cwd=str(Path(__file__).resolve().parent.parent))
