"""Python mirror of SoL's renderer interface over the C ABI.

  Image          sol::Image with three planar FP32 channels (include/sol/image.h)
  GpuScene       an uploaded scene (sol_gpu_scene_create / destroy)
  GpuPathTracer  sol::PathTracer's interface: render(image, sample_index,
                 sample_count) adds the samples into the image
                 (include/sol/renderer.h:34, src/algorithms/path_tracer.cpp:9-23)

Every call goes to the CUDA library; failures raise SolGpuError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .scene import Camera, Config, Scene


class Image:
    """sol::Image with 3 channels: planar float32 array of shape (3, height, width)."""

    def __init__(self, width: int, height: int):
        self.channels = np.zeros((3, height, width), np.float32)

    @property
    def width(self) -> int:
        return self.channels.shape[2]

    @property
    def height(self) -> int:
        return self.channels.shape[1]

    def clear(self, value: float = 0.0) -> None:       # src/image.cpp:13-16
        self.channels[...] = np.float32(value)

    def scale(self, value: float) -> None:             # src/image.cpp:18-23
        self.channels *= np.float32(value)

    def rgb_at(self, x: int, y: int):
        return tuple(float(self.channels[c, y, x]) for c in range(3))

    def save(self, path: str) -> None:
        """Image::save for OpenEXR (src/image.cpp:25-36, src/formats/exr.cpp:47-100):
        float channels named B, G, R.  Other formats are not written here."""
        if not str(path).lower().endswith(".exr"):
            raise ValueError("only .exr output is supported")
        from .film import save_exr
        save_exr(str(path), self.channels)

    @classmethod
    def load(cls, path: str) -> "Image":
        """Reads an EXR written by save() (R, G, B planes back in SoL's order)."""
        from .film import load_exr
        planes, names = load_exr(str(path))
        img = cls(planes.shape[2], planes.shape[1])
        for c, name in enumerate("RGB"):
            img.channels[c] = planes[names.index(name)]
        return img


class GpuScene:
    """A scene uploaded to one GPU. `bvh` optionally passes a prebuilt BVH (see scene.build_bvh)."""

    def __init__(self, scene: Scene, device: int = 0, bvh=None, gpu_bvh: bool = False):
        """`gpu_bvh`: build the hierarchy on the device (SOL_GPU_SCENE_GPU_BVH)."""
        self.scene = scene
        self.device = device
        desc = scene.desc(bvh)
        h = capi.ScenePtr()
        flags = capi.SCENE_GPU_BVH if gpu_bvh else 0
        capi.check(capi.lib.sol_gpu_scene_create_ex(desc.ptr, device, flags, C.byref(h)), "sol_gpu_scene_create_ex")
        self.handle = h

    def info(self) -> capi.SolGpuSceneInfo:
        out = capi.SolGpuSceneInfo()
        capi.check(capi.lib.sol_gpu_scene_info(self.handle, C.byref(out)), "sol_gpu_scene_info")
        return out

    def param_layout(self):
        """(count, per-texture offsets, per-image offsets) of the parameter vector."""
        n = C.c_uint64()
        capi.check(capi.lib.sol_gpu_param_layout(self.handle, C.byref(n), None, None), "sol_gpu_param_layout")
        nt, ni = max(1, len(self.scene.textures)), max(1, len(self.scene.images))
        to = (C.c_uint64 * nt)()
        io = (C.c_uint64 * ni)()
        capi.check(capi.lib.sol_gpu_param_layout(self.handle, C.byref(n), to, io), "sol_gpu_param_layout")
        return n.value, list(to)[:len(self.scene.textures)], list(io)[:len(self.scene.images)]

    def get_params(self) -> np.ndarray:
        n = self.param_layout()[0]
        out = np.zeros(n, np.float32)
        capi.check(capi.lib.sol_gpu_params_get(self.handle, out.ctypes.data_as(C.POINTER(C.c_float))),
                   "sol_gpu_params_get")
        return out

    def set_params(self, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, np.float32)
        if v.size != self.param_layout()[0]:
            raise ValueError("parameter vector has the wrong size")
        capi.check(capi.lib.sol_gpu_params_set(self.handle, v.ctypes.data_as(C.POINTER(C.c_float))),
                   "sol_gpu_params_set")

    def set_instrumented(self, on: bool) -> None:
        capi.check(capi.lib.sol_gpu_scene_set_instrumented(self.handle, int(on)), "sol_gpu_scene_set_instrumented")

    def set_schedule(self, schedule: int) -> None:
        """capi.SCHEDULE_AUTO / SCHEDULE_PER_PIXEL / SCHEDULE_SPLIT (same film bits)."""
        capi.check(capi.lib.sol_gpu_scene_set_schedule(self.handle, int(schedule)), "sol_gpu_scene_set_schedule")

    def set_scratch_limit(self, nbytes: int) -> None:
        """Bytes of split-schedule scratch a render may use (0: default); larger renders run in chunks."""
        capi.check(capi.lib.sol_gpu_scene_set_scratch_limit(self.handle, int(nbytes)), "sol_gpu_scene_set_scratch_limit")

    def set_traversal_limit(self, max_steps: int) -> None:
        """Self-check bound on one BVH traversal's loop steps (0: default); exceeding it fails the render."""
        capi.check(capi.lib.sol_gpu_scene_set_traversal_limit(self.handle, int(max_steps)),
                   "sol_gpu_scene_set_traversal_limit")

    def trace(self, rays_ptr: int, count: int, any_hit: bool, hits_ptr: int, stream: int = 0) -> None:
        """Device-pointer batch query (SolGpuRay in, SolGpuHit out)."""
        capi.check(capi.lib.sol_gpu_trace(self.handle, rays_ptr, count, int(any_hit), hits_ptr, stream), "sol_gpu_trace")

    def close(self) -> None:
        if getattr(self, "handle", None):
            capi.check(capi.lib.sol_gpu_scene_destroy(self.handle), "sol_gpu_scene_destroy")
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuPathTracer:
    """sol::PathTracer on the GPU: same constructor shape (scene, config)."""

    name = "PathTracer"

    def __init__(self, scene: GpuScene | Scene, config: Config | None = None, camera: Camera | None = None,
                 device: int = 0):
        self.scene = scene if isinstance(scene, GpuScene) else GpuScene(scene, device)
        self.config = config or Config()
        self.camera = camera or self.scene.scene.camera
        self._cam = self.camera.to_c()
        self._cfg = self.config.to_c()

    def render(self, image: Image, sample_index: int, sample_count: int = 1) -> None:
        """Adds samples [sample_index, sample_index + sample_count) of every pixel into `image`."""
        ch = image.channels
        if not ch.flags.c_contiguous or ch.dtype != np.float32:
            raise ValueError("image channels must be C-contiguous float32")
        f32p = C.POINTER(C.c_float)
        capi.check(capi.lib.sol_gpu_render(self.scene.handle, C.byref(self._cam), C.byref(self._cfg), sample_index,
                                           sample_count, image.width, image.height,
                                           ch[0].ctypes.data_as(f32p), ch[1].ctypes.data_as(f32p),
                                           ch[2].ctypes.data_as(f32p)), "sol_gpu_render")

    def render_device(self, film_ptr: int, width: int, height: int, sample_index: int, sample_count: int,
                      stream: int = 0) -> None:
        """Asynchronous render into a device film of 3*width*height floats (R, G, B planes)."""
        capi.check(capi.lib.sol_gpu_render_device(self.scene.handle, C.byref(self._cam), C.byref(self._cfg),
                                                  sample_index, sample_count, width, height, film_ptr, stream),
                   "sol_gpu_render_device")

    def adjoint(self, dl_dfilm_ptr: int, grad_ptr: int, width: int, height: int, sample_index: int,
                sample_count: int, stream: int = 0) -> None:
        """Path-replay adjoint: adds dL/d(params) into the device vector at `grad_ptr`."""
        capi.check(capi.lib.sol_gpu_adjoint(self.scene.handle, C.byref(self._cam), C.byref(self._cfg), sample_index,
                                            sample_count, width, height, dl_dfilm_ptr, grad_ptr, stream),
                   "sol_gpu_adjoint")

    def stats(self) -> capi.SolGpuRenderStats:
        out = capi.SolGpuRenderStats()
        capi.check(capi.lib.sol_gpu_render_stats(self.scene.handle, C.byref(out)), "sol_gpu_render_stats")
        return out


class GpuRenderJob:
    """sol::RenderJob on the GPU (include/sol/render_job.h): frames of
    `samples_per_frame` samples added into `output` on a background thread.
    start(frame_end) takes an optional callable(job) -> bool called after each
    frame with `output` up to date; False stops the job."""

    def __init__(self, renderer: "GpuPathTracer", output: Image):
        self.renderer = renderer
        self.output = output
        self.sample_count = 0
        self.samples_per_frame = 1
        self.handle = None
        self._cb = None
        self._frames = 0

    def start(self, frame_end=None) -> None:
        if self.handle:
            raise RuntimeError("job already started")
        ch = self.output.channels
        if not ch.flags.c_contiguous or ch.dtype != np.float32:
            raise ValueError("image channels must be C-contiguous float32")

        def trampoline(_user, frames):
            self._frames = int(frames)
            try:
                return 1 if frame_end is None or frame_end(self) else 0
            except Exception:
                return 0
        self._cb = capi.FrameEnd(trampoline)
        f32p = C.POINTER(C.c_float)
        h = capi.JobPtr()
        r = self.renderer
        capi.check(capi.lib.sol_gpu_job_start(r.scene.handle, C.byref(r._cam), C.byref(r._cfg), self.output.width,
                                              self.output.height, *[ch[c].ctypes.data_as(f32p) for c in range(3)],
                                              int(self.sample_count), int(self.samples_per_frame), self._cb, None,
                                              C.byref(h)), "sol_gpu_job_start")
        self.handle = h

    def wait(self, timeout_ms: int = 0) -> bool:
        if not self.handle:
            return True
        done = C.c_int(0)
        capi.check(capi.lib.sol_gpu_job_wait(self.handle, int(timeout_ms), C.byref(done)), "sol_gpu_job_wait")
        return bool(done.value)

    def cancel(self) -> None:
        if self.handle:
            capi.check(capi.lib.sol_gpu_job_cancel(self.handle), "sol_gpu_job_cancel")

    @property
    def frames(self) -> int:
        """Frames finished so far (inside frame_end: including the one just finished)."""
        if not self.handle:
            return self._frames
        n = C.c_uint64(0)
        capi.check(capi.lib.sol_gpu_job_frames(self.handle, C.byref(n)), "sol_gpu_job_frames")
        return max(n.value, self._frames)

    def close(self) -> None:
        if self.handle:
            capi.lib.sol_gpu_job_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def image_l2(film_ptr: int, target_ptr: int, count: int, film_scale: float, dl_dfilm_ptr: int, loss_ptr: int,
             stream: int = 0) -> None:
    """L2 loss kernel: adds sum (s*film - target)^2 into the device double at loss_ptr."""
    capi.check(capi.lib.sol_gpu_image_l2(film_ptr, target_ptr, count, film_scale, dl_dfilm_ptr or None, loss_ptr,
                                         stream), "sol_gpu_image_l2")


class BatchRenderer:
    """Many views (camera, film, sample range) over one or more GpuScenes in one
    wavefront launch (sol_gpu_batch_*).  Films are device pointers (3*w*h floats)."""

    def __init__(self, scenes, capacity: int = 0, block_size: int = 0, sort_threshold: int = 0,
                 host_loop: bool = False, schedule: int = capi.BATCH_WAVEFRONT, ray_order: int = 0):
        self.scenes = list(scenes)
        arr = (capi.ScenePtr * len(self.scenes))(*[s.handle for s in self.scenes])
        opts = capi.SolGpuBatchOptions(capacity, block_size, sort_threshold, int(host_loop), int(schedule),
                                       int(ray_order))
        h = capi.BatchPtr()
        capi.check(capi.lib.sol_gpu_batch_create(arr, len(self.scenes), C.byref(opts), C.byref(h)),
                   "sol_gpu_batch_create")
        self.handle = h

    @staticmethod
    def views(specs) -> "C.Array":
        """specs: iterable of (scene_index, Camera, width, height, sample_index, sample_count, film_ptr)."""
        specs = list(specs)
        arr = (capi.SolGpuView * max(1, len(specs)))()
        for k, (si, cam, w, h, index, count, film) in enumerate(specs):
            v = arr[k]
            v.scene = si
            v.camera = cam.to_c() if isinstance(cam, Camera) else cam
            v.width, v.height = w, h
            v.sample_index, v.sample_count = index, count
            v.film = film
        return arr, len(specs)

    def render(self, config: Config, views, stream: int = 0) -> None:
        arr, n = views
        cfg = config.to_c()
        capi.check(capi.lib.sol_gpu_batch_render(self.handle, C.byref(cfg), arr, n, stream), "sol_gpu_batch_render")

    def forward_adjoint(self, config: Config, specs, stream: int = 0) -> None:
        """Fused forward + L2-loss adjoint. specs: (scene_index, Camera, w, h, sample_index, sample_count,
        film_ptr, target_ptr, grad_ptr, loss_ptr) per view, all device pointers."""
        specs = list(specs)
        arr = (capi.SolGpuAdjointView * max(1, len(specs)))()
        for k, (si, cam, w, h, index, count, film, target, grad, loss) in enumerate(specs):
            a = arr[k]
            a.view.scene = si
            a.view.camera = cam.to_c() if isinstance(cam, Camera) else cam
            a.view.width, a.view.height = w, h
            a.view.sample_index, a.view.sample_count = index, count
            a.view.film, a.target, a.grad, a.loss = film, target, grad, loss
        cfg = config.to_c()
        capi.check(capi.lib.sol_gpu_batch_forward_adjoint(self.handle, C.byref(cfg), arr, len(specs), stream),
                   "sol_gpu_batch_forward_adjoint")

    def autotune(self, config: Config, views, cache_path: str | None = None) -> capi.SolGpuBatchOptions:
        arr, n = views
        cfg = config.to_c()
        out = capi.SolGpuBatchOptions()
        capi.check(capi.lib.sol_gpu_batch_autotune(self.handle, C.byref(cfg), arr, n,
                                                   cache_path.encode() if cache_path else None, C.byref(out)),
                   "sol_gpu_batch_autotune")
        return out

    def stats(self) -> capi.SolGpuRenderStats:
        out = capi.SolGpuRenderStats()
        capi.check(capi.lib.sol_gpu_batch_stats(self.handle, C.byref(out)), "sol_gpu_batch_stats")
        return out

    def set_scratch_limit(self, nbytes: int) -> None:
        """Wavefront scratch bytes per render (0: default); larger renders run in chunks of samples."""
        capi.check(capi.lib.sol_gpu_batch_set_scratch_limit(self.handle, int(nbytes)), "sol_gpu_batch_set_scratch_limit")

    def set_iteration_limit(self, max_iterations: int) -> None:
        """Self-check bound on the wavefront's bounce-loop iterations (0: default)."""
        capi.check(capi.lib.sol_gpu_batch_set_iteration_limit(self.handle, int(max_iterations)),
                   "sol_gpu_batch_set_iteration_limit")

    def close(self) -> None:
        if getattr(self, "handle", None):
            capi.check(capi.lib.sol_gpu_batch_destroy(self.handle), "sol_gpu_batch_destroy")
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
