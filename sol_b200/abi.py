"""ctypes declarations of the C ABI in include/sol_gpu.h: status codes, enum
values, structures and the signature table.

Importing this module loads no library, so scene descriptions can be built
(and handed to a CPU renderer) without the CUDA library; `sol_b200.capi` loads
the library and binds the signatures declared here.
"""
from __future__ import annotations

import ctypes as C


OK = 0
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_OUT_OF_MEMORY = -3
ERR_TIMEOUT = -4
ERR_QUEUE_OVERFLOW = -5
ERR_BAD_INDEX = -6
ERR_UNSUPPORTED = -7
ERR_CANCELLED = -8
SCHEDULE_AUTO, SCHEDULE_PER_PIXEL, SCHEDULE_SPLIT = 0, 1, 2
BATCH_WAVEFRONT, BATCH_MEGAKERNEL, BATCH_AUTO = 0, 1, 2
RAY_ORDER_DEFAULT, RAY_ORDER_QUEUE, RAY_ORDER_SORTED, RAY_ORDER_PACKED_SHADOWS = 0, 1, 2, 3
SCENE_GPU_BVH = 1

BSDF_DIFFUSE, BSDF_PHONG, BSDF_MIRROR, BSDF_GLASS, BSDF_INTERP = range(5)
TEX_CONSTANT, TEX_CONSTANT_COLOR, TEX_IMAGE = range(3)
FILTER_NEAREST, FILTER_BILINEAR = range(2)
BORDER_CLAMP, BORDER_REPEAT, BORDER_MIRROR = range(3)
LIGHT_POINT, LIGHT_TRIANGLE, LIGHT_SPHERE = range(3)

f32p = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)


class SolGpuTexture(C.Structure):
    _fields_ = [("type", C.c_int32), ("filter", C.c_int32), ("border", C.c_int32), ("image", C.c_int32),
                ("value", C.c_float * 3)]


class SolGpuImage(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("channels", f32p * 3)]


class SolGpuBsdf(C.Structure):
    _fields_ = [("type", C.c_int32), ("tex", C.c_int32 * 3), ("a", C.c_int32), ("b", C.c_int32)]


class SolGpuLight(C.Structure):
    _fields_ = [("type", C.c_int32), ("intensity_tex", C.c_int32), ("intensity", C.c_float * 3),
                ("v0", C.c_float * 3), ("v1", C.c_float * 3), ("v2", C.c_float * 3)]


class SolGpuBvhNode(C.Structure):
    _fields_ = [("lo", C.c_float * 3), ("hi", C.c_float * 3), ("first", C.c_uint32), ("count", C.c_uint32)]


class SolGpuSceneDesc(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("num_triangles", C.c_uint32),
                ("vertices", f32p), ("normals", f32p), ("tex_coords", f32p), ("indices", u32p),
                ("tri_bsdf", i32p), ("tri_light", i32p),
                ("num_bsdfs", C.c_uint32), ("bsdfs", C.POINTER(SolGpuBsdf)),
                ("num_textures", C.c_uint32), ("textures", C.POINTER(SolGpuTexture)),
                ("num_images", C.c_uint32), ("images", C.POINTER(SolGpuImage)),
                ("num_lights", C.c_uint32), ("lights", C.POINTER(SolGpuLight)),
                ("num_bvh_nodes", C.c_uint32), ("bvh_nodes", C.POINTER(SolGpuBvhNode)),
                ("bvh_prim_indices", u32p)]


class SolGpuCamera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("dir", C.c_float * 3), ("right", C.c_float * 3), ("up", C.c_float * 3)]


class SolGpuConfig(C.Structure):
    _fields_ = [("max_path_len", C.c_uint32), ("min_rr_path_len", C.c_uint32),
                ("min_survival_prob", C.c_float), ("max_survival_prob", C.c_float), ("ray_offset", C.c_float)]


class SolGpuRenderStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("nodes_visited", C.c_uint64), ("tris_tested", C.c_uint64), ("kernel_ms", C.c_float),
                ("launches", C.c_uint32), ("sample_chunk", C.c_uint32)]


class SolGpuSceneInfo(C.Structure):
    _fields_ = [("num_triangles", C.c_uint32), ("num_nodes", C.c_uint32), ("bvh_depth", C.c_uint32),
                ("sah_cost", C.c_float), ("device_bytes", C.c_uint64), ("build_ms", C.c_float)]


class SolGpuRay(C.Structure):
    _fields_ = [("org", C.c_float * 3), ("tmin", C.c_float), ("dir", C.c_float * 3), ("tmax", C.c_float)]


class SolGpuHit(C.Structure):
    _fields_ = [("tri", C.c_int32), ("t", C.c_float), ("u", C.c_float), ("v", C.c_float)]


class SolGpuView(C.Structure):
    _fields_ = [("scene", C.c_uint32), ("camera", SolGpuCamera), ("width", C.c_uint32), ("height", C.c_uint32),
                ("sample_index", C.c_uint64), ("sample_count", C.c_uint32), ("film", C.c_void_p)]


class SolGpuAdjointView(C.Structure):
    _fields_ = [("view", SolGpuView), ("target", C.c_void_p), ("grad", C.c_void_p), ("loss", C.c_void_p)]


class SolGpuBatchOptions(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("block_size", C.c_uint32), ("sort_threshold", C.c_uint32),
                ("host_loop", C.c_int32), ("schedule", C.c_int32), ("ray_order", C.c_int32)]


ScenePtr = C.c_void_p
BatchPtr = C.c_void_p
JobPtr = C.c_void_p
FrameEnd = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)

# (name, restype, argtypes) of every entry point declared in include/sol_gpu.h
SIGNATURES = [
    ("sol_gpu_last_error", C.c_char_p, []),
    ("sol_gpu_abi_version", C.c_int, []),
    ("sol_gpu_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("sol_gpu_scene_create", C.c_int, [C.POINTER(SolGpuSceneDesc), C.c_int, C.POINTER(ScenePtr)]),
    ("sol_gpu_scene_create_ex", C.c_int, [C.POINTER(SolGpuSceneDesc), C.c_int, C.c_uint32, C.POINTER(ScenePtr)]),
    ("sol_gpu_camera_perspective", C.c_int, [C.c_float * 3, C.c_float * 3, C.c_float * 3, C.c_float, C.c_float,
                                             C.POINTER(SolGpuCamera)]),
    ("sol_gpu_scene_destroy", C.c_int, [ScenePtr]),
    ("sol_gpu_scene_info", C.c_int, [ScenePtr, C.POINTER(SolGpuSceneInfo)]),
    ("sol_gpu_render", C.c_int, [ScenePtr, C.POINTER(SolGpuCamera), C.POINTER(SolGpuConfig), C.c_uint64, C.c_uint32,
                                 C.c_uint32, C.c_uint32, f32p, f32p, f32p]),
    ("sol_gpu_render_device", C.c_int, [ScenePtr, C.POINTER(SolGpuCamera), C.POINTER(SolGpuConfig), C.c_uint64,
                                        C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("sol_gpu_render_stats", C.c_int, [ScenePtr, C.POINTER(SolGpuRenderStats)]),
    ("sol_gpu_scene_set_instrumented", C.c_int, [ScenePtr, C.c_int]),
    ("sol_gpu_scene_set_schedule", C.c_int, [ScenePtr, C.c_int]),
    ("sol_gpu_scene_set_scratch_limit", C.c_int, [ScenePtr, C.c_uint64]),
    ("sol_gpu_scene_set_traversal_limit", C.c_int, [ScenePtr, C.c_uint32]),
    ("sol_gpu_trace", C.c_int, [ScenePtr, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]),
    ("sol_gpu_batch_create", C.c_int, [C.POINTER(ScenePtr), C.c_uint32, C.POINTER(SolGpuBatchOptions),
                                       C.POINTER(BatchPtr)]),
    ("sol_gpu_batch_destroy", C.c_int, [BatchPtr]),
    ("sol_gpu_batch_render", C.c_int, [BatchPtr, C.POINTER(SolGpuConfig), C.POINTER(SolGpuView), C.c_uint32,
                                       C.c_void_p]),
    ("sol_gpu_batch_stats", C.c_int, [BatchPtr, C.POINTER(SolGpuRenderStats)]),
    ("sol_gpu_batch_set_iteration_limit", C.c_int, [BatchPtr, C.c_uint64]),
    ("sol_gpu_batch_set_scratch_limit", C.c_int, [BatchPtr, C.c_uint64]),
    ("sol_gpu_batch_forward_adjoint", C.c_int, [BatchPtr, C.POINTER(SolGpuConfig), C.POINTER(SolGpuAdjointView),
                                                C.c_uint32, C.c_void_p]),
    ("sol_gpu_batch_forward_adjoint_noalloc", C.c_int, [C.POINTER(ScenePtr), C.c_uint32, C.POINTER(SolGpuConfig),
                                                        C.POINTER(SolGpuAdjointView), C.c_uint32, C.c_void_p]),
    ("sol_gpu_batch_autotune", C.c_int, [BatchPtr, C.POINTER(SolGpuConfig), C.POINTER(SolGpuView), C.c_uint32,
                                         C.c_char_p, C.POINTER(SolGpuBatchOptions)]),
    ("sol_gpu_param_layout", C.c_int, [ScenePtr, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("sol_gpu_params_get", C.c_int, [ScenePtr, f32p]),
    ("sol_gpu_params_set", C.c_int, [ScenePtr, f32p]),
    ("sol_gpu_adjoint", C.c_int, [ScenePtr, C.POINTER(SolGpuCamera), C.POINTER(SolGpuConfig), C.c_uint64, C.c_uint32,
                                  C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("sol_gpu_image_l2", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("sol_gpu_job_start", C.c_int, [ScenePtr, C.POINTER(SolGpuCamera), C.POINTER(SolGpuConfig), C.c_uint32, C.c_uint32,
                                     f32p, f32p, f32p, C.c_uint64, C.c_uint32, FrameEnd, C.c_void_p,
                                     C.POINTER(JobPtr)]),
    ("sol_gpu_job_wait", C.c_int, [JobPtr, C.c_uint32, C.POINTER(C.c_int)]),
    ("sol_gpu_job_cancel", C.c_int, [JobPtr]),
    ("sol_gpu_job_frames", C.c_int, [JobPtr, C.POINTER(C.c_uint64)]),
    ("sol_gpu_job_destroy", C.c_int, [JobPtr]),
    ("sol_gpu_build_bvh", C.c_int, [f32p, C.c_uint32, u32p, C.c_uint32, C.POINTER(SolGpuBvhNode), u32p, u32p]),
]


