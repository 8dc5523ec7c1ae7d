"""Regenerates tests/golden/sol_scenes/*.npz: SoL's four test scenes as this
library's loader reads them, with the film SoL renders from its own load.

For each of SoL's test scenes (test/data/cornell_box*.toml with their OBJ/MTL
files; modified Cornell boxes from Morgan McGuire's Computer Graphics Archive,
CC BY 3.0, as test/data/copyright.txt states -- "Created by Guedis Cardenas
and Morgan McGuire at Williams College, 2011") this script

  * loads the scene with sol_b200.loader.load_scene and with SoL's own
    sol::Scene::load (oracle/_ref), and checks that SoL's PathTracer renders
    both to the same film bit for bit;
  * stores the loaded tables (vertices, normals, texture coordinates,
    triangles, per-triangle BSDF and light, texture / BSDF / light tables,
    camera) and SoL's film of its own load: 64x64, samples 3..10 (8 spp),
    max path length 16, Russian roulette from bounce 3.

The GPU test (tests/test_gpu_loader.py) renders the stored scene on the
device and compares with the stored film, so it runs where SoL's tree is
absent.  Needs SoL's sources in $SOL_REF_DIR (default: the directory
`reference` beside the repository); run from the repository root:
    python tests/golden/make_sol_scenes.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

W = H = 64
SPP = 8
INDEX = 3
ASPECT = 1.0


def config():
    from sol_b200.scene import Config
    return Config(max_path_len=16, min_rr_path_len=3, min_survival_prob=0.05, max_survival_prob=0.75, ray_offset=1e-5)


def scene_to_arrays(s) -> dict:
    tables = {
        "textures": [[t.type, list(t.value), t.image, t.filter, t.border] for t in s.textures],
        "bsdfs": [[b.type, list(b.tex), b.a, b.b] for b in s.bsdfs],
        "lights": [[l.type, list(l.v0), list(l.v1), list(l.v2), l.intensity_tex, list(l.intensity)] for l in s.lights],
        "camera": [list(s.camera.eye), list(s.camera.dir), list(s.camera.up), s.camera.fov, s.camera.aspect],
    }
    return {"vertices": np.asarray(s.vertices, np.float32), "normals": np.asarray(s.normals, np.float32),
            "tex_coords": np.asarray(s.tex_coords, np.float32), "indices": np.asarray(s.indices, np.uint32),
            "tri_bsdf": np.asarray(s.tri_bsdf, np.int32), "tri_light": np.asarray(s.tri_light, np.int32),
            "tables": np.frombuffer(json.dumps(tables).encode(), np.uint8)}


def arrays_to_scene(d):
    """The Scene stored by scene_to_arrays (images: none in SoL's test scenes)."""
    from sol_b200.scene import Bsdf, Camera, Light, Scene, Texture
    t = json.loads(bytes(d["tables"]).decode())
    cam = t["camera"]
    return Scene(vertices=d["vertices"], normals=d["normals"], tex_coords=d["tex_coords"], indices=d["indices"],
                 tri_bsdf=d["tri_bsdf"], tri_light=d["tri_light"],
                 textures=[Texture(a, tuple(v), i, f, b) for a, v, i, f, b in t["textures"]],
                 bsdfs=[Bsdf(a, tuple(x), p, q) for a, x, p, q in t["bsdfs"]],
                 lights=[Light(a, tuple(v0), tuple(v1), tuple(v2), i, tuple(e)) for a, v0, v1, v2, i, e in t["lights"]],
                 images=[], camera=Camera(tuple(cam[0]), tuple(cam[1]), tuple(cam[2]), cam[3], cam[4]))


def main() -> None:
    import oracle
    from sol_b200 import loader
    oracle.build(ref=True)
    out = HERE / "sol_scenes"
    out.mkdir(exist_ok=True)
    for name in oracle.REFERENCE_SCENES:
        path = oracle.reference_scene(name)
        if path is None:
            raise SystemExit(f"SoL's test scene {name} is not present (set SOL_REF_DIR)")
        ours = loader.load_scene(str(path), ASPECT)
        assert not ours.images, "SoL's test scenes have no image textures"
        sol = oracle.RefScene.load(str(path), ASPECT)
        film, _ = sol.render(config(), W, H, SPP, sample_index=INDEX)
        again, _ = oracle.RefScene(ours).render(config(), W, H, SPP, sample_index=INDEX)
        assert np.array_equal(film, again), f"{name}: the two loads render differently"
        back = arrays_to_scene(scene_to_arrays(ours))
        again, _ = oracle.RefScene(back).render(config(), W, H, SPP, sample_index=INDEX)
        assert np.array_equal(film, again), f"{name}: the stored tables render differently"
        np.savez_compressed(out / f"{name}.npz", film=film, **scene_to_arrays(ours))
        print(name, ours.num_triangles, "triangles", (out / f"{name}.npz").stat().st_size, "bytes")


if __name__ == "__main__":
    main()
