"""Test infrastructure: CPU checkers for the GPU path tracer.  Not part of the product.

Two checkers, both over the flat scene of include/sol_gpu.h:
  * liboracle.so (oracle/_build/): pt_oracle.cpp, a C++ restatement of SoL's
    path tracer (src/algorithms/path_tracer.cpp and the classes it calls);
  * libsol_ref.so (oracle/_ref/): SoL's own sources compiled against the
    clean-room proto/par/bvh shims (oracle/Makefile), driven by ref_harness.cpp;
    it links nothing of the product;
  * libsol_dropin.so (oracle/_ref/): the GPU drop-in sol::GpuPathTracer over the
    scenes of libsol_ref.so (drop-in tests only; it loads the product library).

Only tests, the smoke check and bench.py's CPU-baseline leg use this package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libsol_ref.so"
DROPIN_LIB = HERE / "_ref" / "libsol_dropin.so"
# SoL's source tree (read only): $SOL_REF_DIR, by default the directory
# `reference` beside this repository's root (as oracle/Makefile assumes).
REF_SOURCES = Path(os.environ.get("SOL_REF_DIR") or HERE.parent.parent / "reference")

_oracle = None
_ref = None


def build(ref: bool = True) -> None:
    """Builds liboracle.so, and libsol_ref.so / libsol_dropin.so when SoL's
    sources are present."""
    targets = ["oracle"]
    if ref and (REF_SOURCES / "src" / "algorithms" / "path_tracer.cpp").exists():
        targets += ["ref", "dropin"]
    subprocess.run(["make", "-s", "-C", str(HERE), f"SOL_REF_DIR={REF_SOURCES}"] + targets, check=True)


def _bind_common():
    from sol_b200 import abi
    return abi


class CameraArgs(C.Structure):
    """OracleCamera: sol::PerspectiveCamera constructor arguments."""
    _fields_ = [("eye", C.c_float * 3), ("dir", C.c_float * 3), ("up", C.c_float * 3),
                ("fov", C.c_float), ("aspect", C.c_float)]


def camera_args(camera) -> CameraArgs:
    c = CameraArgs()
    c.eye[:] = camera.eye
    c.dir[:] = camera.dir
    c.up[:] = camera.up
    c.fov = camera.fov
    c.aspect = camera.aspect
    return c


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            build(ref=False)
        capi = _bind_common()
        lib = C.CDLL(str(ORACLE_LIB))
        f32p = C.POINTER(C.c_float)
        lib.oracle_render.argtypes = [C.POINTER(capi.SolGpuSceneDesc), C.POINTER(CameraArgs),
                                      C.POINTER(capi.SolGpuConfig), C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                      f32p, f32p, f32p, C.c_int]
        lib.oracle_render.restype = C.c_int
        lib.oracle_trace.argtypes = [C.POINTER(capi.SolGpuSceneDesc), C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
        lib.oracle_trace.restype = C.c_int
        lib.oracle_pcg_floats.argtypes = [C.c_uint64, C.c_uint32, f32p]
        lib.oracle_pcg_floats.restype = None
        lib.oracle_debug_path.argtypes = [C.POINTER(capi.SolGpuSceneDesc), C.POINTER(CameraArgs),
                                          C.POINTER(capi.SolGpuConfig), C.c_uint64, C.c_uint32, C.c_uint32,
                                          C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                          C.POINTER(C.c_float)]
        lib.oracle_debug_path.restype = C.c_uint32
        lib.oracle_pixel_seeds.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        lib.oracle_pow.argtypes = [f32p, f32p, C.c_uint32, f32p]
        lib.oracle_pow.restype = None
        lib.oracle_pixel_seeds.restype = None
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return REF_LIB.exists()


REFERENCE_SCENES = ("cornell_box", "cornell_box_glossy", "cornell_box_specular", "cornell_box_water")


def reference_scene(name: str):
    """Path of one of SoL's own test scene files (test/data/<name>.toml), or None
    where SoL's sources are not present."""
    p = REF_SOURCES / "test" / "data" / f"{name}.toml"
    return p if p.exists() else None


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} is not built (needs SoL's sources; see oracle/Makefile)")
        capi = _bind_common()
        lib = C.CDLL(str(REF_LIB))
        f32p = C.POINTER(C.c_float)
        lib.ref_scene_create.argtypes = [C.POINTER(capi.SolGpuSceneDesc), C.POINTER(CameraArgs)]
        lib.ref_scene_create.restype = C.c_void_p
        lib.ref_scene_destroy.argtypes = [C.c_void_p]
        lib.ref_scene_destroy.restype = None
        lib.ref_scene_set_camera.argtypes = [C.c_void_p, C.POINTER(CameraArgs)]
        lib.ref_scene_set_camera.restype = C.c_int
        lib.ref_scene_render.argtypes = [C.c_void_p, C.POINTER(capi.SolGpuConfig), C.c_uint64, C.c_uint32,
                                         C.c_uint32, C.c_uint32, f32p, f32p, f32p, C.c_int, C.POINTER(C.c_double)]
        lib.ref_scene_render.restype = C.c_int
        lib.ref_scene_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
        lib.ref_scene_trace.restype = C.c_int
        lib.ref_renderjob_render.argtypes = [C.c_void_p, C.POINTER(capi.SolGpuConfig), C.c_uint32, C.c_uint32,
                                             C.c_uint32, C.c_uint32, f32p, f32p, f32p, C.c_int]
        lib.ref_renderjob_render.restype = C.c_int
        lib.ref_last_error.argtypes = []
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_scene_load.argtypes = [C.c_char_p, C.c_float]
        lib.ref_scene_load.restype = C.c_void_p
        lib.ref_scene_counts.argtypes = [C.c_void_p] + [C.POINTER(C.c_uint32)] * 4
        lib.ref_scene_counts.restype = None
        _ref = lib
    return _ref


_dropin = None


def dropin_available() -> bool:
    return DROPIN_LIB.exists()


def dropin_lib() -> C.CDLL:
    """libsol_dropin.so (loads libsol_ref.so and the product library)."""
    global _dropin
    if _dropin is None:
        if not DROPIN_LIB.exists():
            raise FileNotFoundError(f"{DROPIN_LIB} is not built (needs SoL's sources; see oracle/Makefile)")
        capi = _bind_common()
        ref_lib()
        lib = C.CDLL(str(DROPIN_LIB))
        f32p = C.POINTER(C.c_float)
        lib.ref_adapter_render.argtypes = [C.c_void_p, C.POINTER(capi.SolGpuConfig), C.c_uint64, C.c_uint32,
                                           C.c_uint32, C.c_uint32, f32p, f32p, f32p, C.c_int, C.c_int, C.c_uint32]
        lib.ref_adapter_render.restype = C.c_int
        _dropin = lib
    return _dropin


def _film(w: int, h: int, film=None) -> np.ndarray:
    return np.zeros((3, h, w), np.float32) if film is None else np.ascontiguousarray(film, np.float32)


def _ptrs(film: np.ndarray):
    f32p = C.POINTER(C.c_float)
    return [film[c].ctypes.data_as(f32p) for c in range(3)]


def render(scene, config, width: int, height: int, spp: int, sample_index: int = 0, threads: int = 0,
           camera=None, film=None) -> np.ndarray:
    """Oracle render: returns the (3, h, w) film after adding `spp` samples per pixel."""
    desc = scene.desc()
    cam = camera_args(camera or scene.camera)
    cfg = config.to_c()
    out = _film(width, height, film)
    oracle_lib().oracle_render(desc.ptr, C.byref(cam), C.byref(cfg), sample_index, spp, width, height,
                               *_ptrs(out), threads)
    return out


def trace(scene, rays: np.ndarray, any_hit: bool) -> np.ndarray:
    """rays: (n, 8) float32 [org, tmin, dir, tmax] -> hits (n, 4) records (tri:int32, t, u, v)."""
    desc = scene.desc()
    rays = np.ascontiguousarray(rays, np.float32)
    hits = np.zeros((rays.shape[0], 4), np.float32)
    oracle_lib().oracle_trace(desc.ptr, rays.ctypes.data, rays.shape[0], int(any_hit), hits.ctypes.data)
    return hits


def debug_path(scene, config, frame: int, x: int, y: int, width: int, height: int, camera=None, cap: int = 64):
    """Rays of one (pixel, sample) path: (rays (n, 8), kinds (n,), hits (n, 4), colour (3,))."""
    desc = scene.desc()
    cam = camera_args(camera or scene.camera)
    cfg = config.to_c()
    rays = np.zeros((cap, 8), np.float32)
    kinds = np.zeros(cap, np.int32)
    hits = np.zeros((cap, 4), np.float32)
    col = (C.c_float * 3)()
    n = oracle_lib().oracle_debug_path(desc.ptr, C.byref(cam), C.byref(cfg), frame, x, y, width, height,
                                       rays.ctypes.data, kinds.ctypes.data, hits.ctypes.data, cap, col)
    n = min(n, cap)
    return rays[:n], kinds[:n], hits[:n], np.array(list(col), np.float32)


def pcg_floats(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    oracle_lib().oracle_pcg_floats(seed, n, out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def pixel_seeds(fxy: np.ndarray) -> np.ndarray:
    fxy = np.ascontiguousarray(fxy, np.uint64)
    out = np.zeros(fxy.shape[0], np.uint32)
    oracle_lib().oracle_pixel_seeds(fxy.ctypes.data, fxy.shape[0], out.ctypes.data)
    return out


def pow_float(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """The shared pow_ of core/math.h on the host, element-wise (float32)."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    out = np.zeros(x.shape[0], np.float32)
    f32p = C.POINTER(C.c_float)
    oracle_lib().oracle_pow(x.ctypes.data_as(f32p), y.ctypes.data_as(f32p), x.shape[0], out.ctypes.data_as(f32p))
    return out


class RefScene:
    """A sol::Scene built by SoL's own constructors, rendered by sol::PathTracer."""

    def __init__(self, scene, camera=None):
        self.lib = ref_lib()
        if scene is None:   # filled in by load()
            self.h = None
            return
        self._desc = scene.desc()
        cam = camera_args(camera or scene.camera)
        self.h = self.lib.ref_scene_create(self._desc.ptr, C.byref(cam))
        if not self.h:
            raise RuntimeError("ref_scene_create failed: " + self.lib.ref_last_error().decode())

    @classmethod
    def load(cls, path: str, aspect_ratio: float = 1.0) -> "RefScene":
        """A scene file loaded by SoL's own loader (sol::Scene::load)."""
        rs = cls(None)
        rs.h = rs.lib.ref_scene_load(str(path).encode(), aspect_ratio)
        if not rs.h:
            raise RuntimeError("sol::Scene::load failed: " + rs.lib.ref_last_error().decode())
        return rs

    def set_camera(self, camera) -> None:
        """Renders from now on through `camera` (a sol_b200.scene.Camera)."""
        cam = camera_args(camera)
        if self.lib.ref_scene_set_camera(self.h, C.byref(cam)) != 0:
            raise RuntimeError("ref_scene_set_camera failed: " + self.lib.ref_last_error().decode())

    def counts(self) -> dict:
        """Sizes of the scene's light, BSDF, texture and image tables."""
        v = [C.c_uint32() for _ in range(4)]
        self.lib.ref_scene_counts(self.h, *[C.byref(x) for x in v])
        return dict(zip(("lights", "bsdfs", "textures", "images"), (x.value for x in v)))

    def render(self, config, width, height, spp, sample_index=0, threads=0, film=None):
        """Returns (film, render_ms)."""
        out = _film(width, height, film)
        ms = C.c_double(0.0)
        cfg = config.to_c()
        rc = self.lib.ref_scene_render(self.h, C.byref(cfg), sample_index, spp, width, height, *_ptrs(out),
                                       threads, C.byref(ms))
        if rc != 0:
            raise RuntimeError("ref_scene_render failed: " + self.lib.ref_last_error().decode())
        return out, ms.value

    def render_gpu_dropin(self, config, width, height, spp, sample_index=0, device=0, render_job=False,
                          samples_per_frame=0, film=None):
        """The same sol::Scene rendered by sol::GpuPathTracer (the product's drop-in)."""
        out = _film(width, height, film)
        cfg = config.to_c()
        rc = dropin_lib().ref_adapter_render(self.h, C.byref(cfg), sample_index, spp, width, height, *_ptrs(out),
                                         device, int(render_job), samples_per_frame or spp)
        if rc != 0:
            raise RuntimeError("sol::GpuPathTracer failed: " + self.lib.ref_last_error().decode())
        return out

    def render_job(self, config, width, height, spp, samples_per_frame, threads=0, film=None):
        """sol::PathTracer driven by sol::RenderJob."""
        out = _film(width, height, film)
        cfg = config.to_c()
        self.lib.ref_renderjob_render(self.h, C.byref(cfg), spp, samples_per_frame, width, height, *_ptrs(out), threads)
        return out

    def trace(self, rays: np.ndarray, any_hit: bool) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros((rays.shape[0], 4), np.float32)
        self.lib.ref_scene_trace(self.h, rays.ctypes.data, rays.shape[0], int(any_hit), hits.ctypes.data)
        return hits

    def close(self):
        if self.h:
            self.lib.ref_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
