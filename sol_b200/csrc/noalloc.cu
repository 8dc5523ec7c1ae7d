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
//
// The tables are built on the host and reach the array as kernel parameters:
// a small copy kernel takes up to 30 KiB of them by value per launch and
// stores them, so no host-to-device copy from pageable memory is involved
// (the launch itself snapshots its parameters).
//
// With lazy module loading (the CUDA 12 default) the library's device image,
// and with it the array, becomes resident on a device at the library's first
// launch there (with CUDA_MODULE_LOADING=EAGER, when the library is loaded).
// The cached address is that of the current CUDA context of the device: after
// cudaDeviceReset the library must not be used in the same process.
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

/// One piece of the host-built scratch image, passed to the copy kernel by value.
constexpr uint32_t kUploadChunkBytes = 30 * 1024;
struct UploadChunk {
    uint32_t offset;   // byte offset in the scratch array (multiple of 16)
    uint32_t bytes;    // multiple of 16, at most kUploadChunkBytes
    uint32_t pad[2];
    uint4 data[kUploadChunkBytes / 16];
};
static_assert(sizeof(UploadChunk) <= 32764, "kernel parameters are limited to 32,764 bytes");

/// Stores one chunk of the tables into the scratch array.
__global__ void __launch_bounds__(256) upload_chunk(const __grid_constant__ UploadChunk c, unsigned char* dst) {
    uint4* out = reinterpret_cast<uint4*>(dst + c.offset);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.bytes / 16; i += gridDim.x * blockDim.x)
        out[i] = c.data[i];
}

/// Copies bytes [offset, offset + bytes) of the host image `src` (laid out as
/// the scratch array) into the array at `dst`, one kernel launch per chunk.
cudaError_t upload(const unsigned char* src, size_t offset, size_t bytes, unsigned char* dst, cudaStream_t stream) {
    bytes = (bytes + 15) & ~(size_t)15;
    UploadChunk c;
    for (size_t at = 0; at < bytes; at += kUploadChunkBytes) {
        const size_t n = bytes - at < kUploadChunkBytes ? bytes - at : kUploadChunkBytes;
        c.offset = (uint32_t)(offset + at);
        c.bytes = (uint32_t)n;
        std::memcpy(c.data, src + offset + at, n);
        const int blocks = (int)((n / 16 + 255) / 256);
        upload_chunk<<<blocks, 256, 0, stream>>>(c, dst);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

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
    // The tables are built on the host stack in the layout of the scratch array
    // (63 KB, counters zero) and stored into it by upload(), whose launches take
    // them by value: the stack may unwind as soon as this call returns.
    alignas(16) unsigned char image[kNoAllocScratchBytes];
    std::memset(image + kCountersOffset, 0, sizeof(DeviceCounters));
    SceneView* scene_table = reinterpret_cast<SceneView*>(image + kScenesOffset);
    AdjView* view_table = reinterpret_cast<AdjView*>(image + kViewsOffset);
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
    cudaError_t e = upload(image, kScenesOffset, sizeof(SceneView) * num_scenes, scratch, st);
    if (e == cudaSuccess) e = upload(image, kViewsOffset, sizeof(AdjView) * num_views, scratch, st);
    if (e == cudaSuccess) e = upload(image, kCountersOffset, sizeof(DeviceCounters), scratch, st);
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
