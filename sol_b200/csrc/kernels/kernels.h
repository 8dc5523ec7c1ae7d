// Host-side launchers of the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../core/layout.h"
#include "../../../include/sol_gpu.h"

namespace sol_b200 {

#ifndef SOL_MEGAKERNEL_BLOCK
#define SOL_MEGAKERNEL_BLOCK 128
#endif
#ifndef SOL_MEGAKERNEL_MIN_BLOCKS
#define SOL_MEGAKERNEL_MIN_BLOCKS 12  // 40 registers: the lean split kernel measured fastest here (16: 32 registers, 1.2 % slower)
#endif
#ifndef SOL_MEGAKERNEL_VIEWS_MIN_BLOCKS
#define SOL_MEGAKERNEL_VIEWS_MIN_BLOCKS 12   // the multi-view megakernel: 40 registers (measured faster than 16 and 10)
#endif
#ifndef SOL_MEGAKERNEL_SMALL_MIN_BLOCKS
#define SOL_MEGAKERNEL_SMALL_MIN_BLOCKS 12   // 40 registers: renders of a few paths per lane, where spills cost more
#endif
#ifndef SOL_MEGAKERNEL_SPLIT_LEAN
#define SOL_MEGAKERNEL_SPLIT_LEAN 1   // 1: the split schedule's lean kernel (pt_megakernel_lean)
#endif
#ifndef SOL_LEAN_REGEN_MIN
// The split schedule's lean kernel: idle lanes of a warp claim new work items
// together once at least this many are idle (0: the warp claims only when all
// 32 paths have ended).  Measured (frame / Cornell Mpaths/s): 0 -> 2455 /
// 604, 8 -> 2593 / 654, 12 -> 2617 / 652, 16 -> 2635 / 645, 20 -> 2636 / 650,
// 24 -> 2636 / 648, 32 -> 2419 / 589.
#define SOL_LEAN_REGEN_MIN 20
#endif
#ifndef SOL_MEGAKERNEL_SHARED_STACK
#define SOL_MEGAKERNEL_SHARED_STACK 0   // 1: first traversal-stack entries in shared memory (measured 5% slower)
#endif
/// Threads per block of the megakernel, and the resident blocks per SM its
/// register allocation must allow (the compile-time occupancy target).
constexpr int kMegakernelBlock = SOL_MEGAKERNEL_BLOCK;
constexpr int kMegakernelMinBlocks = SOL_MEGAKERNEL_MIN_BLOCKS;
constexpr int kMegakernelSmallMinBlocks = SOL_MEGAKERNEL_SMALL_MIN_BLOCKS;
constexpr int kMegakernelViewsMinBlocks = SOL_MEGAKERNEL_VIEWS_MIN_BLOCKS;
/// K1 renders with at least this many paths per resident lane of the
/// full-occupancy build use it; smaller renders use the 12-block build.
constexpr uint64_t kMegakernelFullPathsPerLane = 8;
constexpr int kTraceBlock = 128;
#ifndef SOL_SPLIT_SCRATCH_MAX_MB
#define SOL_SPLIT_SCRATCH_MAX_MB 2048
#endif
/// Largest per-sample colour scratch a split-schedule render may use (renders
/// needing more run their samples in chunks that fit).
constexpr size_t kSplitScratchMaxBytes = size_t(SOL_SPLIT_SCRATCH_MAX_MB) << 20;

#ifndef SOL_L2_PERSIST
#define SOL_L2_PERSIST 0   // 1: L2 access-policy window over the upper BVH levels (measured no gain: L2 already keeps them)
#endif

/// A range of device memory that a launch asks L2 to keep (persisting lines):
/// the upper BVH levels, stored first in the node array.  bytes == 0: none.
struct L2Window {
    const void* base = nullptr;
    size_t bytes = 0;
    float hit_ratio = 1.0f;
};

/// Resident blocks per SM of the megakernel (for sizing its persistent grid);
/// `full`: the full-occupancy build (kMegakernelMinBlocks), else the
/// kMegakernelSmallMinBlocks build; `basic`: the build without image textures
/// and Interp BSDFs, for scenes that have neither (SolGpuScene::basic_shading).
int megakernel_blocks_per_sm(bool instrumented, bool full, bool basic);

/// K1: renders samples [sample_index, sample_index + sample_count) of every
/// pixel and adds each pixel's sum into `film` (3 planes of width*height).
/// `counters` must be zeroed before the launch.
cudaError_t launch_megakernel(const SceneView& s, const DCamera& cam, const DConfig& cfg,
                              uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                              float* film, DeviceCounters* counters, bool instrumented, bool full, bool basic,
                              int grid, cudaStream_t stream, const L2Window& l2 = {});

/// K1 in the split schedule: every (pixel, sample) is its own work item, taken
/// sample-major so that a warp runs one sample of an 8x4 pixel tile.  Samples
/// run in chunks of `chunk`: the path colours of a chunk go to `scratch` (chunk
/// x 3 planes of width*height) and are added in sample order to each pixel's
/// running sum (`running`, 3 planes; unused when one chunk holds every
/// sample), which goes into `film` after the last chunk.  Same result bits as
/// launch_megakernel.  `counters` must be zeroed before the call.
cudaError_t launch_megakernel_split(const SceneView& s, const DCamera& cam, const DConfig& cfg,
                                    uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                                    float* film, float* scratch, float* running, uint32_t chunk,
                                    DeviceCounters* counters, bool instrumented, bool full, bool basic, int grid,
                                    cudaStream_t stream, const L2Window& l2 = {});

struct WfView;

/// Scenes a multi-view megakernel launch takes as a kernel parameter.
constexpr uint32_t kViewsTableScenes = 32;
struct SceneTable {
    SceneView v[kViewsTableScenes];
};

/// Resident blocks per SM of the multi-view megakernel.
int megakernel_views_blocks_per_sm();

/// K1b: the megakernel over many views (see WfView) of the scenes in `scenes`;
/// each view's film receives the bits launch_megakernel would give it.
/// `counters` must be zeroed before the launch; kernel self-check failures
/// are ORed into `*fault`.
/// `scenes` is the device copy of the batch's scene views and `host_scenes`
/// the same `num_scenes` views on the host: up to kViewsTableScenes of them go
/// to the kernel by value (SceneTable), more are read from `scenes`.  `basic`:
/// every scene has basic shading (no image textures, no Interp BSDFs).
cudaError_t launch_megakernel_views(const WfView* views, uint32_t num_views, uint32_t total_items, uint32_t max_spp,
                                    const SceneView* scenes, const SceneView* host_scenes, uint32_t num_scenes,
                                    bool basic, const DConfig& cfg, DeviceCounters* counters, unsigned int* fault,
                                    int grid, cudaStream_t stream, const L2Window& l2 = {});

/// Sum pass of the split views of launch_megakernel_views (see WfView::split).
cudaError_t launch_sum_samples_views(const WfView* views, uint32_t num_views, uint64_t total_floats,
                                     cudaStream_t stream);

/// Sum pass of the wavefront's views (item-ordered float4 scratch, see
/// WfView): one thread per pixel of the views laid end to end from
/// WfView::sum_begin (`total_pixels` in all).
cudaError_t launch_sum_items_views(const WfView* views, uint32_t num_views, uint64_t total_pixels, cudaStream_t stream);

/// K9: closest-hit or any-hit queries for a batch of rays.
cudaError_t launch_trace(const SceneView& s, const SolGpuRay* rays, uint32_t count, bool any_hit,
                         SolGpuHit* hits, cudaStream_t stream);

/// Launches `kernel` with an L2 access-policy window (persisting hits on
/// l2.base .. + l2.bytes, streaming misses) when l2.bytes > 0, otherwise plainly.
template <typename... KArgs, typename... Args>
cudaError_t launch_l2(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t stream,
                      const L2Window& l2, Args&&... args) {
    cudaLaunchConfig_t c{};
    c.gridDim = dim3((unsigned)grid);
    c.blockDim = dim3((unsigned)block);
    c.dynamicSmemBytes = smem;
    c.stream = stream;
    cudaLaunchAttribute attr[1];
    if (l2.bytes > 0) {
        attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[0].val.accessPolicyWindow.base_ptr = const_cast<void*>(l2.base);
        attr[0].val.accessPolicyWindow.num_bytes = l2.bytes;
        attr[0].val.accessPolicyWindow.hitRatio = l2.hit_ratio;
        attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        c.attrs = attr;
        c.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&c, kernel, std::forward<Args>(args)...);
}

}  // namespace sol_b200
