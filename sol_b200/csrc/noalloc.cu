// Allocation-free entry point: the fused forward + adjoint launch of
// sol_gpu_batch_forward_adjoint, with its scratch memory in a fixed array that
// is part of the library image instead of memory obtained from cudaMalloc.
//
// Who needs this: callers that must not allocate device memory while they
// render.  A host application that owns the device-memory budget (a plugin
// host with its own allocator, which forbids libraries from calling cudaMalloc
// behind its back) and an optimisation loop that cannot afford the device-wide
// synchronisation cudaFree implies both fall in this group.  Such a caller
// creates its scenes up front and passes films, targets, gradients and loss
// words it allocated itself; sol_gpu_batch_forward_adjoint instead needs a
// SolGpuBatch, whose creation and first use allocate.
//
// The scratch holds the per-call scene table, the per-call view table and the
// launch counters: at most 64 scenes and 512 views, 63,744 bytes in all, which
// every GPU that loads the library keeps until the process exits.  What must
// start at zero: the launch counters, which each call clears itself on its
// stream before the launch; the caller's films, gradients and loss words are
// added into, exactly as with sol_gpu_batch_forward_adjoint.  Every call
// reuses the same array, so two calls that can overlap on the GPU (on two
// streams with no ordering between them, or from two host threads) race on
// it; the caller must order them.  The first call on a device looks the
// array's device address up (cudaGetSymbolAddress); make that first call
// before any stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/sol_gpu.h"
#include "host/handles.h"
#include "kernels/adjoint.h"

namespace sol_b200 {

namespace {

constexpr uint32_t kNoAllocMaxScenes = 64;
constexpr uint32_t kNoAllocMaxViews = 512;

constexpr size_t align256_(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kScenesOffset = 0;
constexpr size_t kViewsOffset = align256_(sizeof(SceneView) * kNoAllocMaxScenes);
constexpr size_t kCountersOffset = kViewsOffset + align256_(sizeof(AdjView) * kNoAllocMaxViews);
constexpr size_t kNoAllocScratchBytes = kCountersOffset + align256_(sizeof(DeviceCounters));
static_assert(kNoAllocScratchBytes <= 64 * 1024, "scratch stays under 64 KiB");

/// The scratch array itself.  In host code this name is only a stand-in for the
/// device object; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

/// Device address of the scratch array on the current device, looked up once
/// per device (the first call on a device does this; make that first call before
/// any stream capture).
int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return fail(SOL_GPU_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[device];
    return SOL_GPU_OK;
}

}  // namespace

}  // namespace sol_b200

using namespace sol_b200;

extern "C" int sol_gpu_batch_forward_adjoint_noalloc(SolGpuScene* const* scenes, uint32_t num_scenes,
                                                      const SolGpuConfig* config, const SolGpuAdjointView* views,
                                                      uint32_t num_views, void* stream) {
    if (!scenes || num_scenes == 0 || !config || (num_views > 0 && !views))
        return fail(SOL_GPU_ERR_INVALID_ARG, "scenes, config and views must not be NULL");
    if (num_scenes > kNoAllocMaxScenes)
        return fail(SOL_GPU_ERR_INVALID_ARG, "the allocation-free entry point takes at most 64 scenes per call");
    if (num_views > kNoAllocMaxViews)
        return fail(SOL_GPU_ERR_INVALID_ARG, "the allocation-free entry point takes at most 512 views per call");
    if (config->max_path_len > (uint32_t)kAdjointMaxDepth)
        return fail(SOL_GPU_ERR_UNSUPPORTED, "the adjoint replays paths of at most 16 vertices");
    const int device = scenes[0] ? scenes[0]->device : -1;
    for (uint32_t i = 0; i < num_scenes; ++i) {
        if (!scenes[i]) return fail(SOL_GPU_ERR_INVALID_ARG, "scene must not be NULL");
        if (scenes[i]->device != device) return fail(SOL_GPU_ERR_INVALID_ARG, "all scenes must be on one device");
    }
    // The tables are built on the host stack (63 KB) and copied in; a copy from
    // pageable memory is staged before cudaMemcpyAsync returns, so the stack may
    // unwind afterwards.
    SceneView scene_table[kNoAllocMaxScenes];
    AdjView view_table[kNoAllocMaxViews];
    uint64_t items = 0;
    for (uint32_t i = 0; i < num_scenes; ++i) scene_table[i] = scenes[i]->view;
    for (uint32_t i = 0; i < num_views; ++i) {
        const SolGpuAdjointView& a = views[i];
        if (a.view.scene >= num_scenes) return fail(SOL_GPU_ERR_INVALID_ARG, "view scene index out of range");
        if (a.view.width == 0 || a.view.height == 0 || a.view.sample_count == 0)
            return fail(SOL_GPU_ERR_INVALID_ARG, "view size and sample count must be positive");
        if (!a.view.film || !a.target || !a.grad || !a.loss) return fail(SOL_GPU_ERR_INVALID_ARG, "view buffers must not be NULL");
        AdjView& w = view_table[i];
        w.cam = to_camera(a.view.camera);
        w.scene = a.view.scene;
        w.width = a.view.width;
        w.height = a.view.height;
        w.sample_count = a.view.sample_count;
        w.sample_index = a.view.sample_index;
        w.film = a.view.film;
        w.target = a.target;
        w.grad = a.grad;
        w.loss = a.loss;
        w.item_begin = (uint32_t)items;
        w.group = fused_group(a.view.sample_count);
        items += fused_items(a.view.width, a.view.height, a.view.sample_count);
        if (items > 0xffffffffull) return fail(SOL_GPU_ERR_INVALID_ARG, "batch too large");
    }
    DeviceGuard guard(device);
    if (guard.err != cudaSuccess) return cuda_fail(guard.err, "cudaSetDevice");
    unsigned char* scratch = nullptr;
    int rc = scratch_address(device, &scratch);
    if (rc != SOL_GPU_OK) return rc;
    if (num_views == 0) return SOL_GPU_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SceneView* d_scenes = reinterpret_cast<SceneView*>(scratch + kScenesOffset);
    AdjView* d_views = reinterpret_cast<AdjView*>(scratch + kViewsOffset);
    DeviceCounters* d_ctr = reinterpret_cast<DeviceCounters*>(scratch + kCountersOffset);
    cudaError_t e = cudaMemcpyAsync(d_scenes, scene_table, sizeof(SceneView) * num_scenes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_views, view_table, sizeof(AdjView) * num_views, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_ctr, 0, sizeof(DeviceCounters), st);
    if (e != cudaSuccess) return cuda_fail(e, "scratch upload");
    int num_sms = 0;
    e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    const int per_sm = fused_blocks_per_sm();
    if (per_sm <= 0) return fail(SOL_GPU_ERR_CUDA, "fused kernel occupancy query failed");
    e = launch_fused_forward_adjoint(d_views, num_views, (uint32_t)items, d_scenes, to_config(*config), d_ctr,
                                     per_sm * num_sms, st);
    return e == cudaSuccess ? SOL_GPU_OK : cuda_fail(e, "fused forward/adjoint launch");
}
