// C ABI of the B200 path tracer (include/sol_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sol_gpu.h"
#include "core/layout.h"
#include "host/flatten.h"
#include "host/handles.h"
#include "kernels/lbvh.h"
#include "kernels/adjoint.h"
#include "kernels/kernels.h"

using namespace sol_b200;

namespace sol_b200 {

namespace {
thread_local std::string g_last_error;
}  // namespace

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

const char* last_error() { return g_last_error.c_str(); }

int cuda_fail(cudaError_t e, const char* what) {
    int code = e == cudaErrorMemoryAllocation ? SOL_GPU_ERR_OUT_OF_MEMORY : SOL_GPU_ERR_CUDA;
    return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

DConfig to_config(const SolGpuConfig& c) {
    DConfig d;
    d.max_path_len = c.max_path_len;
    d.min_rr_path_len = c.min_rr_path_len;
    d.min_survival_prob = c.min_survival_prob;
    d.max_survival_prob = c.max_survival_prob;
    d.ray_offset = c.ray_offset;
    return d;
}

int check_fault(SolGpuScene* s) {
    unsigned int f = 0;
    cudaError_t e = cudaMemcpy(&f, s->fault, sizeof(f), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "fault read");
    if (f == 0) return SOL_GPU_OK;
    cudaMemset(s->fault, 0, sizeof(unsigned int));
    std::string msg = "a kernel self-check failed:";
    if (f & kFaultTraversalSteps) msg += " traversal exceeded its step bound or stack;";
    if (f & kFaultNodeIndex) msg += " BVH node index out of range;";
    if (f & kFaultTriIndex) msg += " triangle index out of range;";
    if (f & kFaultPathLoop) msg += " render loop exceeded its bound;";
    if (f & kFaultClaimLoop) msg += " pixel claim loop exceeded its bound;";
    return fail(SOL_GPU_ERR_BAD_INDEX, msg);
}

DCamera to_camera(const SolGpuCamera& c) {
    DCamera d;
    for (int k = 0; k < 3; ++k) { d.eye[k] = c.eye[k]; d.dir[k] = c.dir[k]; d.right[k] = c.right[k]; d.up[k] = c.up[k]; }
    return d;
}

}  // namespace sol_b200

namespace {

template <typename T>
cudaError_t upload(T** dst, const std::vector<T>& src) {
    size_t bytes = std::max<size_t>(sizeof(T), src.size() * sizeof(T));
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), bytes);
    if (e != cudaSuccess) return e;
    if (!src.empty()) e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

void release(SolGpuScene* s) {
    if (!s) return;
    DeviceGuard g(s->device);
    cudaFree(s->nodes); cudaFree(s->tris); cudaFree(s->shade); cudaFree(s->bsdfs);
    cudaFree(s->textures); cudaFree(s->images); cudaFree(s->texels); cudaFree(s->lights);
    cudaFree(s->counters); cudaFree(s->film_tmp); cudaFree(s->split_scratch); cudaFree(s->adj_texels4); cudaFree(s->param_offsets); cudaFree(s->fault);
    if (s->film_host) cudaFreeHost(s->film_host);
    if (s->ev_start) cudaEventDestroy(s->ev_start);
    if (s->ev_stop) cudaEventDestroy(s->ev_stop);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int check_render_args(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                      uint32_t width, uint32_t height) {
    if (!scene || !camera || !config) return fail(SOL_GPU_ERR_INVALID_ARG, "scene, camera and config must not be NULL");
    if (width == 0 || height == 0) return fail(SOL_GPU_ERR_INVALID_ARG, "image size must be positive");
    if ((uint64_t)((width + 7) / 8) * ((height + 3) / 4) * 32 > 0xffffffffull)
        return fail(SOL_GPU_ERR_INVALID_ARG, "image too large");
    return SOL_GPU_OK;
}

int render_into(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                float* film, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(scene->counters, 0, sizeof(DeviceCounters), stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    SceneView v = scene->view;
    // The full-occupancy build for renders of many paths per resident lane,
    // the 12-block build (fewer spills per path) for smaller ones.
    const bool basic = scene->basic_shading;
    const int per_sm_full = megakernel_blocks_per_sm(scene->instrumented, true, basic);
    if (per_sm_full <= 0) return fail(SOL_GPU_ERR_CUDA, "megakernel occupancy query failed");
    const uint64_t paths = (uint64_t)width * height * sample_count;
    const bool full = paths >= kMegakernelFullPathsPerLane * (uint64_t)per_sm_full * scene->num_sms * kMegakernelBlock;
    const int per_sm = full ? per_sm_full : megakernel_blocks_per_sm(scene->instrumented, false, basic);
    if (per_sm <= 0) return fail(SOL_GPU_ERR_CUDA, "megakernel occupancy query failed");
    const int grid = per_sm * scene->num_sms;
    const DCamera cam = to_camera(*camera);
    // Split schedule (one work item per pixel sample, measured faster than the
    // per-pixel schedule on small and full-size frames alike) for every render
    // of more than one sample, in chunks of samples whose colours fit in the
    // scratch limit; the per-pixel schedule for single samples, on request, or
    // when not even one sample's colours fit.
    const uint64_t pixels = (uint64_t)width * height;
    const uint64_t sample_items = (uint64_t)((width + 7) / 8) * ((height + 3) / 4) * 32;
    const uint64_t sample_floats = 3 * pixels;
    const uint64_t limit = scene->scratch_limit ? scene->scratch_limit : (uint64_t)kSplitScratchMaxBytes;
    const uint64_t chunk = std::min<uint64_t>({(uint64_t)sample_count, limit / (sample_floats * sizeof(float)),
                                               0x7fffffffull / sample_items});
    if (scene->schedule == SOL_GPU_SCHEDULE_SPLIT && chunk == 0)
        return fail(SOL_GPU_ERR_UNSUPPORTED, "the split schedule needs more than " + std::to_string(limit) +
                                             " bytes of scratch for one sample of this image");
    bool split = chunk > 0 && (scene->schedule == SOL_GPU_SCHEDULE_SPLIT ||
                               (scene->schedule == SOL_GPU_SCHEDULE_AUTO && sample_count > 1));
    const size_t scratch_floats = split ? (size_t)(chunk * sample_floats) : 0;
    const size_t running_floats = split && chunk < sample_count ? (size_t)sample_floats : 0;
    if (split && scene->split_floats < scratch_floats + running_floats) {
        cudaFree(scene->split_scratch);
        scene->split_scratch = nullptr;
        scene->split_floats = 0;
        e = cudaMalloc(reinterpret_cast<void**>(&scene->split_scratch),
                       (scratch_floats + running_floats) * sizeof(float));
        if (e == cudaSuccess) {
            scene->split_floats = scratch_floats + running_floats;
        } else if (scene->schedule == SOL_GPU_SCHEDULE_AUTO) {
            cudaGetLastError();   // no room for the scratch: render per pixel instead
            split = false;
        } else {
            return cuda_fail(e, "cudaMalloc split scratch");
        }
    }
    cudaEventRecord(scene->ev_start, stream);
    if (split)
        e = launch_megakernel_split(v, cam, to_config(*config), sample_index, sample_count, width, height, film,
                                    scene->split_scratch, running_floats ? scene->split_scratch + scratch_floats : nullptr,
                                    (uint32_t)chunk, scene->counters, scene->instrumented, full, basic, grid,
                                    stream, scene->l2);
    else
        e = launch_megakernel(v, cam, to_config(*config), sample_index, sample_count, width, height, film,
                              scene->counters, scene->instrumented, full, basic, grid, stream, scene->l2);
    if (e != cudaSuccess) return cuda_fail(e, "megakernel launch");
    cudaEventRecord(scene->ev_stop, stream);
    scene->rendered = true;
    scene->last_chunk = split ? (uint32_t)chunk : 0u;
    scene->last_launches = split ? 2u * (uint32_t)((sample_count + chunk - 1) / chunk) : 1u;
    return SOL_GPU_OK;
}

}  // namespace

extern "C" {

const char* sol_gpu_last_error(void) { return sol_b200::last_error(); }

int sol_gpu_abi_version(void) { return SOL_GPU_ABI_VERSION; }

int sol_gpu_device_count(int* count) {
    if (!count) return fail(SOL_GPU_ERR_INVALID_ARG, "count must not be NULL");
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) { *count = 0; return cuda_fail(e, "cudaGetDeviceCount"); }
    return SOL_GPU_OK;
}

int sol_gpu_scene_create(const SolGpuSceneDesc* desc, int device, SolGpuScene** out) {
    return sol_gpu_scene_create_ex(desc, device, 0u, out);
}

int sol_gpu_scene_create_ex(const SolGpuSceneDesc* desc, int device, uint32_t flags, SolGpuScene** out) {
    if (!desc || !out) return fail(SOL_GPU_ERR_INVALID_ARG, "desc and out must not be NULL");
    *out = nullptr;
    const bool gpu_bvh = (flags & SOL_GPU_SCENE_GPU_BVH) && desc->num_bvh_nodes == 0 && desc->num_triangles >= 2;
    FlatScene flat;
    std::string err;
    if (!flatten_scene(*desc, flat, err, !gpu_bvh)) return fail(SOL_GPU_ERR_INVALID_ARG, err);

    DeviceGuard guard(device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    auto* s = new SolGpuScene();
    s->device = device;
    cudaError_t e = cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_start);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_stop);
    float gpu_build_ms = 0.0f;
    if (gpu_bvh && e == cudaSuccess) {
        // Build the hierarchy on the device from the mesh arrays.
        const uint32_t nv = desc->num_vertices, nt = desc->num_triangles;
        float *d_v = nullptr, *d_n = nullptr, *d_uv = nullptr;
        uint32_t* d_i = nullptr;
        int32_t *d_b = nullptr, *d_l = nullptr;
        auto up = [&](void** dst, const void* src, size_t bytes) {
            if (e != cudaSuccess) return;
            e = cudaMalloc(dst, bytes ? bytes : 1);
            if (e == cudaSuccess && bytes) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
        };
        cudaEvent_t b0, b1;
        cudaEventCreate(&b0);
        cudaEventCreate(&b1);
        cudaEventRecord(b0, s->stream);
        up(reinterpret_cast<void**>(&d_v), desc->vertices, sizeof(float) * 3 * nv);
        up(reinterpret_cast<void**>(&d_n), desc->normals, sizeof(float) * 3 * nv);
        up(reinterpret_cast<void**>(&d_uv), desc->tex_coords, sizeof(float) * 2 * nv);
        up(reinterpret_cast<void**>(&d_i), desc->indices, sizeof(uint32_t) * 3 * nt);
        up(reinterpret_cast<void**>(&d_b), desc->tri_bsdf, sizeof(int32_t) * nt);
        up(reinterpret_cast<void**>(&d_l), desc->tri_light, sizeof(int32_t) * nt);
        LbvhResult r;
        if (e == cudaSuccess) e = build_lbvh(d_v, d_i, d_n, d_uv, d_b, d_l, nt, s->stream, &r);
        cudaEventRecord(b1, s->stream);
        cudaEventSynchronize(b1);
        cudaEventElapsedTime(&gpu_build_ms, b0, b1);
        cudaEventDestroy(b0);
        cudaEventDestroy(b1);
        cudaFree(d_v); cudaFree(d_n); cudaFree(d_uv); cudaFree(d_i); cudaFree(d_b); cudaFree(d_l);
        if (e == cudaSuccess) {
            s->nodes = r.nodes;
            s->tris = r.tris;
            s->shade = r.shade;
            flat.depth = r.depth;
            flat.sah_cost = r.sah_cost;
            flat.top_nodes = 0;
            flat.nodes.assign(r.num_nodes, DNode{});   // sizes only: the arrays are already on the device
            if (r.depth > (uint32_t)kTraversalStack) {
                release(s);
                return fail(SOL_GPU_ERR_UNSUPPORTED, "GPU BVH depth " + std::to_string(r.depth) +
                                                     " exceeds the traversal stack (64); use the host builder");
            }
        }
    }
    if (!gpu_bvh) {
        if (e == cudaSuccess) e = upload(&s->nodes, flat.nodes);
        if (e == cudaSuccess) e = upload(&s->tris, flat.tris);
        if (e == cudaSuccess) e = upload(&s->shade, flat.shade);
    }
    if (e == cudaSuccess) e = upload(&s->bsdfs, flat.bsdfs);
    if (e == cudaSuccess) e = upload(&s->textures, flat.textures);
    if (e == cudaSuccess) e = upload(&s->images, flat.images);
    if (e == cudaSuccess) e = upload(&s->texels, flat.texels);
    if (e == cudaSuccess) e = upload(&s->lights, flat.lights);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s->counters), sizeof(DeviceCounters));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s->fault), sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(s->fault, 0, sizeof(unsigned int));
    // Parameter layout: constants in texture order, then the images' texel blocks.
    s->host_textures = flat.textures;
    s->host_images = flat.images;
    s->texel_count = flat.texels.size();
    uint64_t off = 0;
    s->texture_offsets.assign(flat.textures.size(), 0);
    for (size_t i = 0; i < flat.textures.size(); ++i) {
        const int kind = flat.textures[i].kind;
        if (kind == SOL_GPU_TEX_CONSTANT) { s->texture_offsets[i] = off; off += 1; }
        else if (kind == SOL_GPU_TEX_CONSTANT_COLOR) { s->texture_offsets[i] = off; off += 3; }
    }
    s->constants_count = off;
    for (const DImage& im : flat.images) { s->image_offsets.push_back(off + im.offset); }
    off += flat.texels.size();
    s->param_count = off;
    for (size_t i = 0; i < flat.textures.size(); ++i)
        if (flat.textures[i].kind == SOL_GPU_TEX_IMAGE) s->texture_offsets[i] = s->image_offsets[flat.textures[i].image];
    {
        std::vector<unsigned long long> offs(s->texture_offsets.begin(), s->texture_offsets.end());
        if (e == cudaSuccess) e = upload(&s->param_offsets, offs);
    }
    if (e != cudaSuccess) { int rc = cuda_fail(e, "scene upload"); release(s); return rc; }

    s->view.nodes = s->nodes;
    s->view.tris = s->tris;
    s->view.shade = s->shade;
    s->view.bsdfs = s->bsdfs;
    s->view.textures = s->textures;
    s->view.images = s->images;
    s->view.texels = s->texels;
    s->view.lights = s->lights;
    s->view.num_lights = (uint32_t)flat.lights.size();
    s->view.num_tris = desc->num_triangles;
    s->view.param_offsets = s->param_offsets;
    s->view.num_nodes = (uint32_t)flat.nodes.size();
    const size_t num_tris = gpu_bvh ? desc->num_triangles : flat.tris.size();
    s->default_max_steps = (uint32_t)std::min<uint64_t>(2ull * (flat.nodes.size() + num_tris) + 16ull, 0xffffffffull);
    s->view.max_steps = s->default_max_steps;
    s->view.fault = s->fault;
    s->basic_shading =
        std::none_of(flat.textures.begin(), flat.textures.end(),
                     [](const DTexture& t) { return t.kind == SOL_GPU_TEX_IMAGE; }) &&
        std::none_of(flat.bsdfs.begin(), flat.bsdfs.end(), [](const DBsdf& b) { return b.kind == SOL_GPU_BSDF_INTERP; });

    s->info.num_triangles = desc->num_triangles;
    s->info.num_nodes = (uint32_t)flat.nodes.size();
    s->info.bvh_depth = flat.depth;
    s->info.sah_cost = flat.sah_cost;
    s->info.device_bytes = flat.nodes.size() * sizeof(DNode) + num_tris * (sizeof(DTri) + sizeof(DTriShade));
    s->info.build_ms = (float)flat.build_ms + gpu_build_ms;
#if SOL_L2_PERSIST
    // Keep the upper BVH levels (stored first) in L2: raise this process's
    // persisting-L2 carve-out up to the device maximum if the range needs it,
    // and let the render launches mark that range as persisting.
    {
        int max_persist = 0;
        if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, s->device) == cudaSuccess &&
            max_persist > 0) {
            const size_t want = std::min<size_t>((size_t)flat.top_nodes * sizeof(DNode), (size_t)max_persist);
            size_t have = 0;
            cudaDeviceGetLimit(&have, cudaLimitPersistingL2CacheSize);
            if (want > have) cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want);
            cudaDeviceGetLimit(&have, cudaLimitPersistingL2CacheSize);
            const size_t bytes = (size_t)flat.top_nodes * sizeof(DNode);
            if (have > 0 && bytes > 0) {
                s->l2.base = s->nodes;
                s->l2.bytes = bytes;
                s->l2.hit_ratio = (float)std::min(1.0, (double)have / (double)bytes);
            }
        }
        cudaGetLastError();   // a device without persisting L2 simply runs without the window
    }
#endif
    *out = s;
    return SOL_GPU_OK;
}

int sol_gpu_camera_perspective(const float eye[3], const float dir[3], const float up[3], float fov, float aspect,
                               SolGpuCamera* out) {
    if (!eye || !dir || !up || !out) return fail(SOL_GPU_ERR_INVALID_ARG, "camera arguments must not be NULL");
    *out = perspective_camera(eye, dir, up, fov, aspect);
    return SOL_GPU_OK;
}

int sol_gpu_scene_destroy(SolGpuScene* scene) {
    if (!scene) return fail(SOL_GPU_ERR_INVALID_ARG, "scene must not be NULL");
    {
        DeviceGuard g(scene->device);
        if (scene->stream) cudaStreamSynchronize(scene->stream);
    }
    release(scene);
    return SOL_GPU_OK;
}

int sol_gpu_scene_info(const SolGpuScene* scene, SolGpuSceneInfo* out) {
    if (!scene || !out) return fail(SOL_GPU_ERR_INVALID_ARG, "scene and out must not be NULL");
    *out = scene->info;
    return SOL_GPU_OK;
}

int sol_gpu_scene_set_instrumented(SolGpuScene* scene, int instrumented) {
    if (!scene) return fail(SOL_GPU_ERR_INVALID_ARG, "scene must not be NULL");
    scene->instrumented = instrumented != 0;
    return SOL_GPU_OK;
}

int sol_gpu_scene_set_schedule(SolGpuScene* scene, int schedule) {
    if (!scene) return fail(SOL_GPU_ERR_INVALID_ARG, "scene must not be NULL");
    if (schedule < SOL_GPU_SCHEDULE_AUTO || schedule > SOL_GPU_SCHEDULE_SPLIT)
        return fail(SOL_GPU_ERR_INVALID_ARG, "unknown schedule");
    scene->schedule = schedule;
    return SOL_GPU_OK;
}

int sol_gpu_scene_set_scratch_limit(SolGpuScene* scene, uint64_t bytes) {
    if (!scene) return fail(SOL_GPU_ERR_INVALID_ARG, "scene must not be NULL");
    scene->scratch_limit = bytes;
    return SOL_GPU_OK;
}

int sol_gpu_scene_set_traversal_limit(SolGpuScene* scene, uint32_t max_steps) {
    if (!scene) return fail(SOL_GPU_ERR_INVALID_ARG, "scene must not be NULL");
    scene->view.max_steps = max_steps ? max_steps : scene->default_max_steps;
    return SOL_GPU_OK;
}

int sol_gpu_render_device(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                          uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                          float* film_device, void* stream) {
    int rc = check_render_args(scene, camera, config, width, height);
    if (rc != SOL_GPU_OK) return rc;
    if (!film_device) return fail(SOL_GPU_ERR_INVALID_ARG, "film must not be NULL");
    DeviceGuard guard(scene->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    return render_into(scene, camera, config, sample_index, sample_count, width, height, film_device,
                       static_cast<cudaStream_t>(stream));
}

int sol_gpu_render(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                   uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                   float* film_r, float* film_g, float* film_b) {
    int rc = check_render_args(scene, camera, config, width, height);
    if (rc != SOL_GPU_OK) return rc;
    if (!film_r || !film_g || !film_b) return fail(SOL_GPU_ERR_INVALID_ARG, "film channels must not be NULL");
    DeviceGuard guard(scene->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    const size_t plane = (size_t)width * height;
    const size_t floats = 3 * plane;
    cudaError_t e = cudaSuccess;
    if (scene->film_tmp_floats < floats) {
        cudaFree(scene->film_tmp);
        scene->film_tmp = nullptr;
        scene->film_tmp_floats = 0;
        e = cudaMalloc(reinterpret_cast<void**>(&scene->film_tmp), floats * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc film");
        scene->film_tmp_floats = floats;
    }
    if (scene->film_host_floats < floats) {
        if (scene->film_host) cudaFreeHost(scene->film_host);
        scene->film_host = nullptr;
        scene->film_host_floats = 0;
        e = cudaMallocHost(reinterpret_cast<void**>(&scene->film_host), floats * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost film");
        scene->film_host_floats = floats;
    }
    e = cudaMemsetAsync(scene->film_tmp, 0, floats * sizeof(float), scene->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync film");
    rc = render_into(scene, camera, config, sample_index, sample_count, width, height, scene->film_tmp, scene->stream);
    if (rc != SOL_GPU_OK) return rc;
    e = cudaMemcpyAsync(scene->film_host, scene->film_tmp, floats * sizeof(float), cudaMemcpyDeviceToHost, scene->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(scene->stream);
    if (e != cudaSuccess) return cuda_fail(e, "render");
    rc = check_fault(scene);
    if (rc != SOL_GPU_OK) return rc;
    // Image::accumulate: one add per pixel and channel (include/sol/image.h:54-60).
    const float* src = scene->film_host;
    float* dst[3] = {film_r, film_g, film_b};
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)plane; ++i)
        for (int c = 0; c < 3; ++c) dst[c][i] += src[c * plane + i];
    return SOL_GPU_OK;
}

int sol_gpu_render_stats(SolGpuScene* scene, SolGpuRenderStats* out) {
    if (!scene || !out) return fail(SOL_GPU_ERR_INVALID_ARG, "scene and out must not be NULL");
    std::memset(out, 0, sizeof(*out));
    if (!scene->rendered) return SOL_GPU_OK;
    DeviceGuard guard(scene->device);
    cudaError_t e = cudaEventSynchronize(scene->ev_stop);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventSynchronize");
    DeviceCounters c;
    e = cudaMemcpy(&c, scene->counters, sizeof(c), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy counters");
    out->paths = c.paths;
    out->rays = c.rays;
    out->shadow_rays = c.shadow_rays;
    out->nodes_visited = c.nodes;
    out->tris_tested = c.tris;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, scene->ev_start, scene->ev_stop) == cudaSuccess) out->kernel_ms = ms;
    out->launches = scene->last_launches;
    out->sample_chunk = scene->last_chunk;
    return check_fault(scene);
}

int sol_gpu_trace(SolGpuScene* scene, const SolGpuRay* rays_device, uint32_t count, int any_hit,
                  SolGpuHit* hits_device, void* stream) {
    if (!scene || (count > 0 && (!rays_device || !hits_device)))
        return fail(SOL_GPU_ERR_INVALID_ARG, "scene, rays and hits must not be NULL");
    DeviceGuard guard(scene->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    if (scene->view.num_tris == 0) {
        // No geometry: every query misses.
        cudaError_t e = cudaMemsetAsync(hits_device, 0xff, sizeof(SolGpuHit) * count, static_cast<cudaStream_t>(stream));
        return e == cudaSuccess ? SOL_GPU_OK : cuda_fail(e, "cudaMemsetAsync");
    }
    cudaError_t e = launch_trace(scene->view, rays_device, count, any_hit != 0, hits_device,
                                 static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? SOL_GPU_OK : cuda_fail(e, "trace launch");
}

int sol_gpu_param_layout(const SolGpuScene* scene, uint64_t* count, uint64_t* texture_offsets,
                         uint64_t* image_offsets) {
    if (!scene || !count) return fail(SOL_GPU_ERR_INVALID_ARG, "scene and count must not be NULL");
    *count = scene->param_count;
    if (texture_offsets) std::copy(scene->texture_offsets.begin(), scene->texture_offsets.end(), texture_offsets);
    if (image_offsets) std::copy(scene->image_offsets.begin(), scene->image_offsets.end(), image_offsets);
    return SOL_GPU_OK;
}

int sol_gpu_params_get(const SolGpuScene* scene, float* values) {
    if (!scene || !values) return fail(SOL_GPU_ERR_INVALID_ARG, "scene and values must not be NULL");
    for (size_t i = 0; i < scene->host_textures.size(); ++i) {
        const DTexture& t = scene->host_textures[i];
        if (t.kind == SOL_GPU_TEX_CONSTANT) values[scene->texture_offsets[i]] = t.v[0];
        else if (t.kind == SOL_GPU_TEX_CONSTANT_COLOR)
            for (int c = 0; c < 3; ++c) values[scene->texture_offsets[i] + c] = t.v[c];
    }
    if (scene->texel_count == 0) return SOL_GPU_OK;
    DeviceGuard guard(scene->device);
    cudaError_t e = cudaMemcpy(values + scene->constants_count, scene->texels, sizeof(float) * scene->texel_count,
                               cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? SOL_GPU_OK : cuda_fail(e, "params get");
}

int sol_gpu_params_set(SolGpuScene* scene, const float* values) {
    if (!scene || !values) return fail(SOL_GPU_ERR_INVALID_ARG, "scene and values must not be NULL");
    for (size_t i = 0; i < scene->host_textures.size(); ++i) {
        DTexture& t = scene->host_textures[i];
        if (t.kind == SOL_GPU_TEX_CONSTANT) t.v[0] = values[scene->texture_offsets[i]];
        else if (t.kind == SOL_GPU_TEX_CONSTANT_COLOR)
            for (int c = 0; c < 3; ++c) t.v[c] = values[scene->texture_offsets[i] + c];
    }
    DeviceGuard guard(scene->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    cudaError_t e = cudaStreamSynchronize(scene->stream);
    if (e == cudaSuccess && !scene->host_textures.empty())
        e = cudaMemcpy(scene->textures, scene->host_textures.data(), sizeof(DTexture) * scene->host_textures.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess && scene->texel_count > 0)
        e = cudaMemcpy(scene->texels, values + scene->constants_count, sizeof(float) * scene->texel_count,
                       cudaMemcpyHostToDevice);
    return e == cudaSuccess ? SOL_GPU_OK : cuda_fail(e, "params set");
}

int sol_gpu_adjoint(SolGpuScene* scene, const SolGpuCamera* camera, const SolGpuConfig* config,
                    uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                    const float* dl_dfilm, float* grad, void* stream) {
    int rc = check_render_args(scene, camera, config, width, height);
    if (rc != SOL_GPU_OK) return rc;
    if (!dl_dfilm || !grad) return fail(SOL_GPU_ERR_INVALID_ARG, "dl_dfilm and grad must not be NULL");
    if (config->max_path_len > (uint32_t)kAdjointMaxDepth)
        return fail(SOL_GPU_ERR_UNSUPPORTED, "the adjoint replays paths of at most 16 vertices");
    DeviceGuard guard(scene->device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(scene->counters, 0, sizeof(DeviceCounters), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    const uint32_t n_shared = (uint32_t)std::min<uint64_t>(scene->constants_count, kAdjointMaxSharedParams);
    const int per_sm = adjoint_blocks_per_sm(n_shared);
    if (per_sm <= 0) return fail(SOL_GPU_ERR_CUDA, "adjoint occupancy query failed");
    // Spread a pixel's samples over several lanes when the image alone would
    // not give every resident lane a few items.
    const uint64_t lanes = (uint64_t)per_sm * scene->num_sms * kAdjointBlock;
    const uint64_t total = (uint64_t)((width + 7) / 8) * ((height + 3) / 4) * 32;
    // One sample per item when the item count allows; otherwise enough chunks
    // for four items per resident lane.
    uint64_t chunks = (uint64_t)sample_count;
    if (total * chunks > 0x7fffffffull)
        chunks = std::min<uint64_t>(sample_count, std::max<uint64_t>(1, (4 * lanes + total - 1) / total));
    chunks = std::max<uint64_t>(1, std::min<uint64_t>(chunks, 0x7fffffffull / total));
    const uint32_t chunk = (uint32_t)((sample_count + chunks - 1) / chunks);
    cudaEventRecord(scene->ev_start, st);
    const uint64_t num_texels = scene->texel_count / 3;
    if (num_texels > scene->adj_texels4_count) {
        cudaFree(scene->adj_texels4);
        scene->adj_texels4 = nullptr;
        scene->adj_texels4_count = 0;
        e = cudaMalloc(reinterpret_cast<void**>(&scene->adj_texels4), sizeof(float4) * num_texels);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc texel gradient scratch");
        scene->adj_texels4_count = num_texels;
    }
    e = launch_adjoint(scene->view, to_camera(*camera), to_config(*config), sample_index, sample_count, chunk, width,
                       height, dl_dfilm, grad, n_shared, scene->adj_texels4, num_texels,
                       (uint32_t)scene->host_images.size(), scene->constants_count, scene->counters,
                       per_sm * scene->num_sms, st);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint launch");
    cudaEventRecord(scene->ev_stop, st);
    scene->rendered = true;
    return SOL_GPU_OK;
}

int sol_gpu_image_l2(const float* film, const float* target, uint64_t count, float film_scale, float* dl_dfilm,
                     double* loss, void* stream) {
    if (!film || !target || !loss) return fail(SOL_GPU_ERR_INVALID_ARG, "film, target and loss must not be NULL");
    if (count == 0) return SOL_GPU_OK;
    int grid = (int)std::min<uint64_t>((count + 255) / 256, 4096);
    cudaError_t e = launch_l2_loss(film, target, count, film_scale, dl_dfilm, loss, grid, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? SOL_GPU_OK : cuda_fail(e, "loss launch");
}

int sol_gpu_build_bvh(const float* vertices, uint32_t num_vertices, const uint32_t* indices, uint32_t num_triangles,
                      SolGpuBvhNode* nodes_out, uint32_t* num_nodes, uint32_t* prim_indices_out) {
    if (!num_nodes) return fail(SOL_GPU_ERR_INVALID_ARG, "num_nodes must not be NULL");
    if (num_triangles > 0 && (!vertices || !indices)) return fail(SOL_GPU_ERR_INVALID_ARG, "mesh arrays must not be NULL");
    for (size_t i = 0; i < 3 * (size_t)num_triangles; ++i)
        if (indices[i] >= num_vertices) return fail(SOL_GPU_ERR_INVALID_ARG, "vertex index out of range");
    if (num_triangles == 0) { *num_nodes = 0; return SOL_GPU_OK; }
    bvh::Bvh tree = build_mesh_bvh(vertices, indices, num_triangles);
    const uint32_t capacity = *num_nodes;
    *num_nodes = (uint32_t)tree.nodes.size();
    if (!nodes_out || !prim_indices_out) return SOL_GPU_OK;   // size query
    if (capacity < tree.nodes.size()) return fail(SOL_GPU_ERR_INVALID_ARG, "node buffer too small");
    for (size_t i = 0; i < tree.nodes.size(); ++i) {
        const bvh::Node& n = tree.nodes[i];
        for (int k = 0; k < 3; ++k) { nodes_out[i].lo[k] = n.box.lo[k]; nodes_out[i].hi[k] = n.box.hi[k]; }
        nodes_out[i].first = n.first;
        nodes_out[i].count = n.count;
    }
    std::memcpy(prim_indices_out, tree.prim_indices.data(), sizeof(uint32_t) * num_triangles);
    return SOL_GPU_OK;
}

}  // extern "C"
