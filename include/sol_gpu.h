/*
 * sol_gpu.h — C ABI of the B200 path tracer.
 *
 * This is the boundary between SoL's C++ renderer interface and the CUDA
 * kernels.  Everything crosses it as plain pointers, sizes and PODs; no C++ or
 * torch types appear.  Each entry point names the SoL interface it stands in
 * for (paths are relative to the SoL source tree).
 *
 * Conventions
 *  - Every function returns an int status: SOL_GPU_OK (0) or a negative
 *    SOL_GPU_ERR_* code.  sol_gpu_last_error() returns a message for the last
 *    failure on the calling thread.
 *  - Films are planar FP32 RGB, row-major, pixel (0,0) at the top-left, the
 *    layout of sol::Image's three channels (include/sol/image.h:27-28,97).
 *    Render calls ADD into the film (sol::Image::accumulate, image.h:54-60) and
 *    never clear it.
 *  - A scene handle is bound to the device it was created on; every call sets
 *    that device first, so handles may be used from any host thread (SoL's
 *    RenderJob renders on its own std::thread, src/render_job.cpp:25), but one
 *    handle must not be used by two threads at once.
 *  - Inputs are copied at creation; the caller keeps ownership of all arrays.
 */
#ifndef SOL_GPU_H
#define SOL_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOL_GPU_ABI_VERSION 3

/* Status codes */
#define SOL_GPU_OK                  0
#define SOL_GPU_ERR_INVALID_ARG    -1
#define SOL_GPU_ERR_CUDA           -2
#define SOL_GPU_ERR_OUT_OF_MEMORY  -3
#define SOL_GPU_ERR_TIMEOUT        -4
#define SOL_GPU_ERR_QUEUE_OVERFLOW -5
#define SOL_GPU_ERR_BAD_INDEX      -6
#define SOL_GPU_ERR_UNSUPPORTED    -7
#define SOL_GPU_ERR_CANCELLED      -8

/* BSDF kinds, in the order of sol::Bsdf::Tag (include/sol/bsdfs.h:30-36). */
#define SOL_GPU_BSDF_DIFFUSE 0
#define SOL_GPU_BSDF_PHONG   1
#define SOL_GPU_BSDF_MIRROR  2
#define SOL_GPU_BSDF_GLASS   3
#define SOL_GPU_BSDF_INTERP  4

/* Texture kinds (include/sol/textures.h:58-64) and image filter / border modes
 * (textures.h:17-53). */
#define SOL_GPU_TEX_CONSTANT       0   /* sol::ConstantTexture (scalar) */
#define SOL_GPU_TEX_CONSTANT_COLOR 1   /* sol::ConstantColorTexture */
#define SOL_GPU_TEX_IMAGE          2   /* sol::ImageTexture<Filter, Border> */
#define SOL_GPU_FILTER_NEAREST  0
#define SOL_GPU_FILTER_BILINEAR 1
#define SOL_GPU_BORDER_CLAMP  0
#define SOL_GPU_BORDER_REPEAT 1
#define SOL_GPU_BORDER_MIRROR 2

/* Light kinds, in the order of sol::Light::Tag (include/sol/lights.h:49-53). */
#define SOL_GPU_LIGHT_POINT    0
#define SOL_GPU_LIGHT_TRIANGLE 1   /* sol::UniformTriangleLight */
#define SOL_GPU_LIGHT_SPHERE   2   /* sol::UniformSphereLight */

/* A texture.  Scalar lookups of colour textures return their luminance
 * (sol::ColorTexture::sample, textures.h:97-99). */
typedef struct SolGpuTexture {
    int32_t type;      /* SOL_GPU_TEX_* */
    int32_t filter;    /* image: SOL_GPU_FILTER_* */
    int32_t border;    /* image: SOL_GPU_BORDER_* */
    int32_t image;     /* image: index into SolGpuSceneDesc.images */
    float value[3];    /* constant: value[0]; constant colour: r, g, b */
} SolGpuTexture;

/* An RGB image (sol::Image with three channels). */
typedef struct SolGpuImage {
    uint32_t width, height;
    const float* channels[3];   /* R, G, B planes of width*height floats */
} SolGpuImage;

/* A BSDF (include/sol/bsdfs.h:97-181). Texture slots by kind:
 *   diffuse: tex[0] = kd (colour)
 *   phong:   tex[0] = ks (colour), tex[1] = ns (scalar)
 *   mirror:  tex[0] = ks (colour)
 *   glass:   tex[0] = ks (colour), tex[1] = kt (colour), tex[2] = eta (scalar,
 *            the ratio outside/inside, i.e. 1/IOR as SoL's OBJ loader stores it)
 *   interp:  tex[0] = k (scalar), a/b = the two BSDFs (neither may be interp) */
typedef struct SolGpuBsdf {
    int32_t type;
    int32_t tex[3];
    int32_t a, b;
} SolGpuBsdf;

/* A light (include/sol/lights.h:91-138).
 *   point:    v0 = position, intensity = colour
 *   triangle: v0, v1, v2 = the emitting triangle (one-sided: it emits towards
 *             (v1 - v0) x (v2 - v0)), intensity_tex = colour texture
 *   sphere:   v0 = centre, v1[0] = radius, intensity_tex = colour texture */
typedef struct SolGpuLight {
    int32_t type;
    int32_t intensity_tex;
    float intensity[3];
    float v0[3], v1[3], v2[3];
} SolGpuLight;

/* One node of a prebuilt binary BVH, as SoL's TriangleMesh holds it after its
 * own build (src/triangle_mesh.cpp:119-146): node 0 is the root, an inner node
 * (count == 0) has its children at `first` and `first + 1`, a leaf covers
 * prim_indices[first .. first + count).  Leaves may hold at most 8 primitives. */
typedef struct SolGpuBvhNode {
    float lo[3], hi[3];
    uint32_t first;
    uint32_t count;
} SolGpuBvhNode;

/* Flat scene: the contents of one sol::Scene whose root is a TriangleMesh
 * (include/sol/scene.h:34-57, include/sol/triangle_mesh.h:18-24). */
typedef struct SolGpuSceneDesc {
    uint32_t num_vertices;
    uint32_t num_triangles;
    const float* vertices;       /* 3 * num_vertices */
    const float* normals;        /* 3 * num_vertices, shading normals */
    const float* tex_coords;     /* 2 * num_vertices */
    const uint32_t* indices;     /* 3 * num_triangles */
    const int32_t* tri_bsdf;     /* num_triangles; -1 = no BSDF (path ends there) */
    const int32_t* tri_light;    /* num_triangles; -1 = not emissive */
    uint32_t num_bsdfs;    const SolGpuBsdf* bsdfs;
    uint32_t num_textures; const SolGpuTexture* textures;
    uint32_t num_images;   const SolGpuImage* images;
    uint32_t num_lights;   const SolGpuLight* lights;   /* order = sol::Scene::lights */
    /* Optional prebuilt BVH; when num_bvh_nodes == 0 the library builds one
     * (full-sweep SAH + reinsertion, as src/triangle_mesh.cpp:142-144 does). */
    uint32_t num_bvh_nodes;
    const SolGpuBvhNode* bvh_nodes;
    const uint32_t* bvh_prim_indices;  /* num_triangles entries */
} SolGpuSceneDesc;

/* A constructed sol::PerspectiveCamera (include/sol/cameras.h:50-54): the eye,
 * the unit view direction, and the right / up vectors already scaled by the
 * half extents of the image plane.  Rays are generated as in
 * PerspectiveCamera::generate_ray (src/cameras.cpp:23-25). */
typedef struct SolGpuCamera {
    float eye[3];
    float dir[3];
    float right[3];
    float up[3];
} SolGpuCamera;

/* sol::PathTracer::Config (include/sol/algorithms/path_tracer.h:23-29). */
typedef struct SolGpuConfig {
    uint32_t max_path_len;
    uint32_t min_rr_path_len;
    float min_survival_prob;
    float max_survival_prob;
    float ray_offset;
} SolGpuConfig;

/* Counters of the last render on a scene handle. */
typedef struct SolGpuRenderStats {
    uint64_t paths;          /* camera paths traced */
    uint64_t rays;           /* closest-hit + any-hit rays */
    uint64_t shadow_rays;    /* any-hit rays */
    uint64_t nodes_visited;  /* BVH nodes fetched (instrumented renders only) */
    uint64_t tris_tested;    /* triangles tested (instrumented renders only) */
    float kernel_ms;         /* device time of the render kernel(s) */
    uint32_t launches;       /* kernels the render launched (sol_gpu_render_stats; 0 for batches) */
    uint32_t sample_chunk;   /* samples per chunk of the split schedule (0: per-pixel schedule or a batch) */
} SolGpuRenderStats;

/* Description of an uploaded scene. */
typedef struct SolGpuSceneInfo {
    uint32_t num_triangles;
    uint32_t num_nodes;       /* inner nodes of the device BVH */
    uint32_t bvh_depth;
    float sah_cost;
    uint64_t device_bytes;    /* node + triangle + shading arrays */
    float build_ms;           /* host BVH build + flatten */
} SolGpuSceneInfo;

/* A ray for sol_gpu_trace: origin, tmin, direction, tmax (8 floats). */
typedef struct SolGpuRay {
    float org[3]; float tmin;
    float dir[3]; float tmax;
} SolGpuRay;

/* Result of sol_gpu_trace: triangle index in the caller's numbering (-1 = miss),
 * distance and barycentrics (u weights vertex 1, v weights vertex 2). For any-hit
 * queries only `tri` is meaningful (>= 0: occluded). */
typedef struct SolGpuHit {
    int32_t tri;
    float t, u, v;
} SolGpuHit;

typedef struct SolGpuScene SolGpuScene;

/* Message for the last failing call on this thread ("" if none). */
const char* sol_gpu_last_error(void);

/* ABI version (SOL_GPU_ABI_VERSION). */
int sol_gpu_abi_version(void);

/* Number of CUDA devices visible to the library. */
int sol_gpu_device_count(int* count);

/* Builds (or takes) the BVH of a mesh scene and uploads it to `device`.
 * Replaces the device side of TriangleMesh::TriangleMesh + Scene ownership
 * (src/triangle_mesh.cpp:44-60, include/sol/scene.h:34-48). */
int sol_gpu_scene_create(const SolGpuSceneDesc* desc, int device, SolGpuScene** out);

/* Scene creation flags. */
#define SOL_GPU_SCENE_GPU_BVH 1u   /* build the BVH on the device (linear BVH, Karras 2012, with treelet
                                      restructuring, Karras and Aila 2013) instead of the host's SAH
                                      build: much faster for large meshes, a hierarchy of similar SAH
                                      cost; closest hits at exactly equal distances may resolve to
                                      another triangle than with the host build.  Ignored when the
                                      description carries a BVH or has fewer than 2 triangles. */

/* sol_gpu_scene_create with flags (SOL_GPU_SCENE_*); sol_gpu_scene_create is
 * this with flags = 0.  Fails with SOL_GPU_ERR_UNSUPPORTED when a device-built
 * hierarchy is deeper than the traversal stack (64). */
int sol_gpu_scene_create_ex(const SolGpuSceneDesc* desc, int device, uint32_t flags, SolGpuScene** out);

/* sol::PerspectiveCamera's constructor (src/cameras.cpp:5-21): `fov` is the
 * horizontal field of view in degrees, `aspect` = width / height. */
int sol_gpu_camera_perspective(const float eye[3], const float dir[3], const float up[3], float fov, float aspect,
                               SolGpuCamera* out);

/* Frees a scene and its device memory. */
int sol_gpu_scene_destroy(SolGpuScene* scene);

/* Sizes and build statistics of an uploaded scene. */
int sol_gpu_scene_info(const SolGpuScene* scene, SolGpuSceneInfo* out);

/* Renders samples [sample_index, sample_index + sample_count) of every pixel
 * and adds each pixel's sum into the host film channels, exactly as
 * sol::PathTracer::render does (src/algorithms/path_tracer.cpp:9-23 through
 * include/sol/renderer.h:34).  Blocking; host<->device copies included. */
int sol_gpu_render(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                   uint64_t sample_index, uint32_t sample_count,
                   uint32_t width, uint32_t height,
                   float* film_r, float* film_g, float* film_b);

/* Same as sol_gpu_render, but the film is a device buffer of 3*width*height
 * floats (R plane, G plane, B plane) and the call is asynchronous on `stream`
 * (a cudaStream_t; NULL = legacy default stream). */
int sol_gpu_render_device(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                          uint64_t sample_index, uint32_t sample_count,
                          uint32_t width, uint32_t height,
                          float* film_device, void* stream);

/* Counters of the last render on this handle (waits for it to finish). When
 * `instrumented` was set by sol_gpu_scene_set_instrumented, node and triangle
 * counts are filled in as well. */
int sol_gpu_render_stats(SolGpuScene* scene, SolGpuRenderStats* out);

/* Selects the counting variant of the render kernels (slower; for measuring
 * bytes per ray). */
int sol_gpu_scene_set_instrumented(SolGpuScene* scene, int instrumented);

/* Render schedules of sol_gpu_render / sol_gpu_render_device.  Both give the
 * same film bits.  PER_PIXEL: one lane renders all samples of a pixel.  SPLIT:
 * every (pixel, sample) is a work item, a warp taking one sample of an 8x4
 * pixel tile, and the samples are summed per pixel in order afterwards; it
 * uses scratch memory of 12 bytes per pixel and sample, at most 2 GiB (renders
 * needing more run in chunks of samples, with 12 more bytes per pixel for the
 * running sums), held by the scene handle, so renders through one handle must
 * be ordered, e.g. issued on one stream.  AUTO (the default) picks SPLIT for
 * every render of more than one sample (measured faster at every image size),
 * PER_PIXEL for single samples or when the scratch cannot be allocated. */
#define SOL_GPU_SCHEDULE_AUTO      0
#define SOL_GPU_SCHEDULE_PER_PIXEL 1
#define SOL_GPU_SCHEDULE_SPLIT     2
int sol_gpu_scene_set_schedule(SolGpuScene* scene, int schedule);

/* Limit on the split schedule's colour scratch for one render through this
 * handle, in bytes (0: the default, 2 GiB).  A render whose samples need more
 * runs in chunks of samples that fit; the film bits do not change.  No
 * counterpart in the reference (SoL renders on the host). */
int sol_gpu_scene_set_scratch_limit(SolGpuScene* scene, uint64_t bytes);

/* Self-check bound of the BVH traversal on this scene, for tests of the error
 * path (0 restores the default, 2 x (nodes + triangles) + 16 loop steps, which
 * no valid hierarchy reaches).  A ray whose traversal exceeds it is dropped,
 * the kernel records the fault instead of looping, and the render (or the
 * stats call after it) fails with SOL_GPU_ERR_BAD_INDEX; the next render
 * starts clean.  Applies to renders, traces and batches issued afterwards.
 * Replaces no SoL interface: SoL's traversal has no bound (it cannot fail). */
int sol_gpu_scene_set_traversal_limit(SolGpuScene* scene, uint32_t max_steps);

/* Closest-hit (any_hit == 0) or any-hit (any_hit != 0) queries for a batch of
 * device-resident rays, the device side of TriangleMesh::intersect_closest /
 * intersect_any (src/triangle_mesh.cpp:64-117).  Asynchronous on `stream`. */
int sol_gpu_trace(SolGpuScene* scene, const SolGpuRay* rays_device, uint32_t count, int any_hit,
                  SolGpuHit* hits_device, void* stream);

/* ---- Batched rendering: many views over one or more scenes ------------------
 *
 * The batch renderer traces all paths of all views of one call through a
 * persistent wavefront (generate / extend / shade / shadow stages over queues
 * in device memory, hits binned by BSDF kind) whose bounce loop runs inside one
 * CUDA graph.  Every view's film receives exactly what sol_gpu_render_device
 * would add for the same camera and sample range, bit for bit.  There is no
 * SoL counterpart (SoL renders one image per call); it batches
 * PathTracer::render (src/algorithms/path_tracer.cpp:9-23). */

/* One view of a batch. */
typedef struct SolGpuView {
    uint32_t scene;          /* index into the scenes given to sol_gpu_batch_create */
    SolGpuCamera camera;
    uint32_t width, height;
    uint64_t sample_index;
    uint32_t sample_count;
    float* film;             /* device film of 3*width*height floats (R, G, B planes); added into */
} SolGpuView;

/* Tuning of the batch renderer; zero fields take defaults. */
typedef struct SolGpuBatchOptions {
    uint32_t capacity;        /* path slots in flight (default: 4M; at most 64M and the work items;
                                 about 260 bytes of device memory per slot) */
    uint32_t block_size;      /* threads per block of the stages: 64, 128 or 256 (default 128) */
    uint32_t sort_threshold;  /* bin hits by BSDF kind when at least this many rays are queued
                                 (0 = always; 0xffffffff = never) */
    int32_t host_loop;        /* 1: bounce loop driven from the host instead of the graph */
    int32_t schedule;         /* SOL_GPU_BATCH_WAVEFRONT, _MEGAKERNEL or _AUTO (below) */
    int32_t ray_order;        /* SOL_GPU_RAY_ORDER_* (below); ABI version 3 */
} SolGpuBatchOptions;

/* Order in which the wavefront traces each bounce's rays.  QUEUE: as the
 * stages queued them (camera rays in 8x4 pixel tiles, bounce rays in their
 * parents' order, shadow rays in shading order -- material by material when
 * hits are binned).  PACKED_SHADOWS: the same, but shadow rays packed in the
 * order of the rays they were cast from (pixel neighbours stay neighbours
 * when shading is binned; one packing kernel per bounce).  SORTED:
 * counting-sorted first by scene, direction octant and the Morton cell of the
 * origin (14-bit key).  DEFAULT (0) is QUEUE; the autotuner chooses between
 * QUEUE and PACKED_SHADOWS (SORTED measured slower on every batch tried).
 * Films are the same bits in every order. */
#define SOL_GPU_RAY_ORDER_DEFAULT        0
#define SOL_GPU_RAY_ORDER_QUEUE          1
#define SOL_GPU_RAY_ORDER_SORTED         2
#define SOL_GPU_RAY_ORDER_PACKED_SHADOWS 3

/* Batch schedules.  WAVEFRONT: the queue-based wavefront (capacity, block size
 * and sort threshold apply).  MEGAKERNEL: one persistent megakernel launch over
 * all views, lanes claiming pixels of any view.  AUTO: sol_gpu_batch_autotune
 * times both and adopts the faster; before that, AUTO renders as WAVEFRONT.
 * Every schedule gives each film the bits sol_gpu_render_device gives it. */
#define SOL_GPU_BATCH_WAVEFRONT  0
#define SOL_GPU_BATCH_MEGAKERNEL 1
#define SOL_GPU_BATCH_AUTO       2

typedef struct SolGpuBatch SolGpuBatch;

/* Creates a batch renderer over `num_scenes` scenes (all on one device). */
int sol_gpu_batch_create(SolGpuScene* const* scenes, uint32_t num_scenes, const SolGpuBatchOptions* options,
                         SolGpuBatch** out);

/* Frees a batch renderer (the scenes stay alive). */
int sol_gpu_batch_destroy(SolGpuBatch* batch);

/* Renders every view's sample range into its film; asynchronous on `stream`. */
int sol_gpu_batch_render(SolGpuBatch* batch, const SolGpuConfig* config, const SolGpuView* views,
                         uint32_t num_views, void* stream);

/* Counters and device time of the last batch render (waits for it).  Fails
 * with SOL_GPU_ERR_TIMEOUT when the wavefront's bounce loop hit its iteration
 * bound, and with SOL_GPU_ERR_BAD_INDEX when a kernel self-check fired. */
int sol_gpu_batch_stats(SolGpuBatch* batch, SolGpuRenderStats* out);

/* Limit on the wavefront's scratch for one render of this batch, in bytes (0:
 * the default, 8 GiB): per-sample colours of every (view, sample, pixel) and,
 * when they do not fit, the pixel sums carried between chunks of samples that
 * fit.  The film bits do not change.  No counterpart in the reference. */
int sol_gpu_batch_set_scratch_limit(SolGpuBatch* batch, uint64_t bytes);

/* Self-check bound on the wavefront's bounce-loop iterations per render, for
 * tests of the error path (0 restores the default: every vertex of every
 * sample, plus one iteration per sample, which no render reaches).  A render
 * that reaches it stops, and sol_gpu_batch_stats reports SOL_GPU_ERR_TIMEOUT;
 * the next render starts clean.  No counterpart in SoL (RenderJob::wait's
 * timeout, src/render_job.cpp:42-55, bounds a host wait, not the loop). */
int sol_gpu_batch_set_iteration_limit(SolGpuBatch* batch, uint64_t max_iterations);

/* Times candidate options (capacity 2M-64M slots, each only if its pool fits in the
 * device's free memory with 1 GiB to spare; block size, binning threshold, ray
 * order; with schedule AUTO also the megakernel schedule) on up to four samples per pixel of the
 * given views, rendered into scratch films, adopts the fastest and returns it
 * in `chosen`.  With `cache_path` set, a previous
 * choice for the same device and batch shape is read from that file instead,
 * and new choices are appended to it. */
int sol_gpu_batch_autotune(SolGpuBatch* batch, const SolGpuConfig* config, const SolGpuView* views,
                           uint32_t num_views, const char* cache_path, SolGpuBatchOptions* chosen);

/* ---- Progressive rendering job ---------------------------------------------
 *
 * The GPU counterpart of sol::RenderJob (include/sol/render_job.h,
 * src/render_job.cpp:23-59): frames of samples rendered on a host thread into
 * a device copy of the caller's film, which is copied back into the caller's
 * planes after every frame.  Frames cover the sample ranges SoL's RenderJob
 * gives them (render_job.cpp:27-31), so with the same renderer the film
 * matches sol::RenderJob's bit for bit. */

typedef struct SolGpuJob SolGpuJob;

/* Called on the job's thread after each frame, once the host film holds the
 * image so far; `frames` counts the frames done.  Return 0 to stop the job. */
typedef int (*SolGpuFrameEnd)(void* user, uint64_t frames);

/* Starts rendering samples into film_r/g/b (host planes of width*height,
 * added into like sol_gpu_render); sample_count 0 renders until cancelled.
 * The film must stay valid and untouched by the caller until the job has
 * finished (sol_gpu_job_wait), except inside frame_end. */
int sol_gpu_job_start(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config, uint32_t width,
                      uint32_t height, float* film_r, float* film_g, float* film_b, uint64_t sample_count,
                      uint32_t samples_per_frame, SolGpuFrameEnd frame_end, void* user, SolGpuJob** out);

/* RenderJob::wait: waits for the job to end, at most timeout_ms milliseconds
 * (0 = no limit); *finished = 1 when it has ended.  Returns the status of the
 * job's renders once it has ended. */
int sol_gpu_job_wait(SolGpuJob* job, uint32_t timeout_ms, int* finished);

/* RenderJob::cancel: the job stops after the frame in flight. */
int sol_gpu_job_cancel(SolGpuJob* job);

/* Frames finished so far. */
int sol_gpu_job_frames(const SolGpuJob* job, uint64_t* frames);

/* Cancels, waits for the job and frees it. */
int sol_gpu_job_destroy(SolGpuJob* job);

/* ---- Differentiation --------------------------------------------------------
 *
 * Parameters are the scene's texture values: for each texture in order, a
 * constant texture's value (1 float) or a constant colour (3 floats), image
 * textures adding nothing there; then every image's texels (R, G, B planes of
 * width*height floats) in image order.  They cover SoL's diffuse albedos
 * (constant or image), Phong specular colours and exponents, mirror and glass
 * colours, glass ratios, interpolation weights and light emissions.  There is
 * no SoL counterpart: SoL has no differentiable rendering. */

/* Size of the parameter vector; optionally the offset of each texture's block
 * (image textures: their image's block) and of each image's block. */
int sol_gpu_param_layout(const SolGpuScene* scene, uint64_t* count, uint64_t* texture_offsets,
                         uint64_t* image_offsets);

/* Copies the current parameter values to / from a host vector of `count` floats.
 * Setting them changes what later renders and adjoints see. */
int sol_gpu_params_get(const SolGpuScene* scene, float* values);
int sol_gpu_params_set(SolGpuScene* scene, const float* values);

/* Path-replay adjoint: adds dL/d(parameters) into `grad` (device, `count`
 * floats) for the paths that sol_gpu_render_device traces with the same camera,
 * configuration and sample range, given dL/d(film) (device, 3*width*height:
 * R, G, B planes).  Paths are replayed from their seeds, not stored.
 * Derivatives reach every colour texture a path's value is linear in (diffuse
 * albedo, Phong, mirror and glass colours, emission), including the Russian
 * roulette probability's dependence on the path throughput.  Phong exponents
 * receive the derivative of the BSDF value with sampling detached (sampled
 * directions, pdfs and MIS weights held fixed): unbiased for the derivative of
 * the expected image, but not the per-sample derivative a finite difference
 * with common random numbers measures.  Glass ratios and interpolation weights
 * receive none.  Requires config->max_path_len <= 16.  Asynchronous. */
int sol_gpu_adjoint(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                    uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                    const float* dl_dfilm, float* grad, void* stream);

/* L2 image loss on the current device: adds sum_i (film_scale * film[i] - target[i])^2
 * into *loss (a device double) and, when dl_dfilm is not NULL, writes
 * dL/dfilm[i] = 2 film_scale (film_scale * film[i] - target[i]).  Asynchronous. */
int sol_gpu_image_l2(const float* film, const float* target, uint64_t count, float film_scale,
                     float* dl_dfilm, double* loss, void* stream);

/* One view of a fused forward + adjoint batch. */
typedef struct SolGpuAdjointView {
    SolGpuView view;       /* camera, size, sample range; the forward sums are added into view.film */
    const float* target;   /* device, 3*width*height: the loss is sum (sum/sample_count - target)^2 */
    float* grad;           /* device gradient of the view's scene parameters (added into) */
    double* loss;          /* device double (added into) */
} SolGpuAdjointView;

/* Forward render and L2-loss path-replay adjoint of every view, over the batch's
 * scenes, in one persistent launch: each pixel's samples are rendered (film
 * bits as sol_gpu_render_device), its loss and loss gradient formed, and the
 * same samples replayed backwards.  Requires config->max_path_len <= 16.
 * Asynchronous. */
int sol_gpu_batch_forward_adjoint(SolGpuBatch* batch, const SolGpuConfig* config, const SolGpuAdjointView* views,
                                  uint32_t num_views, void* stream);

/* The launch of sol_gpu_batch_forward_adjoint for callers that must not
 * allocate device memory while they render: a host that owns the device-memory
 * budget and forbids libraries to call cudaMalloc, or a loop that cannot
 * afford the device synchronisation of cudaFree.  No counterpart in the
 * reference (SoL renders on the CPU and has no device memory).
 *
 * It takes the scenes directly (no SolGpuBatch, whose creation allocates);
 * view.scene indexes `scenes`.  It allocates nothing: its scene table, view
 * table and counters live in a fixed 63,744-byte array inside the library, one
 * per GPU.  At most 64 scenes (all on one device) and 512 views per call;
 * larger calls fail with SOL_GPU_ERR_INVALID_ARG and say so in
 * sol_gpu_last_error.  Results are those of sol_gpu_batch_forward_adjoint:
 * films, gradients and losses are added into (the caller clears them); the
 * counters in the array are cleared by the call itself.  Calls share the
 * array, so calls that can overlap on the GPU (different streams without
 * ordering, different host threads) race: order them.  The first call on a
 * device looks up the array's address; make it before any stream capture.
 * The tables reach the array as kernel parameters of a small copy kernel (no
 * copy from pageable host memory).  With lazy module loading (the CUDA 12
 * default) the library's device image and the array become resident on a
 * device at the library's first launch there, or when the library is loaded
 * under CUDA_MODULE_LOADING=EAGER; the address is cached per device, so the
 * library must not be used after cudaDeviceReset in the same process.
 * Requires config->max_path_len <= 16.  Asynchronous. */
int sol_gpu_batch_forward_adjoint_noalloc(SolGpuScene* const* scenes, uint32_t num_scenes,
                                          const SolGpuConfig* config, const SolGpuAdjointView* views,
                                          uint32_t num_views, void* stream);

/* Host-only: builds the BVH that TriangleMesh builds for an indexed mesh
 * (src/triangle_mesh.cpp:119-146: triangle boxes and centroids, full-sweep SAH,
 * reinsertion), in the SolGpuBvhNode form that SolGpuSceneDesc accepts.
 * `*num_nodes` holds the capacity of `nodes_out` on entry and the node count on
 * return; with `nodes_out` or `prim_indices_out` NULL only the count is returned
 * (at most 2 * num_triangles - 1).  `prim_indices_out` receives num_triangles
 * entries. */
int sol_gpu_build_bvh(const float* vertices, uint32_t num_vertices, const uint32_t* indices,
                      uint32_t num_triangles, SolGpuBvhNode* nodes_out, uint32_t* num_nodes,
                      uint32_t* prim_indices_out);

#ifdef __cplusplus
}
#endif

#endif /* SOL_GPU_H */
