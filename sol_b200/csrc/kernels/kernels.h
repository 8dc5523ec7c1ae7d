// Host-side launchers of the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../core/layout.h"
#include "../../../include/sol_gpu.h"

namespace sol_b200 {

#ifndef SOL_MEGAKERNEL_BLOCK
#define SOL_MEGAKERNEL_BLOCK 128
#endif
#ifndef SOL_MEGAKERNEL_MIN_BLOCKS
#define SOL_MEGAKERNEL_MIN_BLOCKS 12  // 40 registers: measured fastest despite spills (latency-bound traversal)
#endif
#ifndef SOL_MEGAKERNEL_SHARED_STACK
#define SOL_MEGAKERNEL_SHARED_STACK 0   // 1: first traversal-stack entries in shared memory (measured 5% slower)
#endif
/// Threads per block of the megakernel, and the resident blocks per SM its
/// register allocation must allow (the compile-time occupancy target).
constexpr int kMegakernelBlock = SOL_MEGAKERNEL_BLOCK;
constexpr int kMegakernelMinBlocks = SOL_MEGAKERNEL_MIN_BLOCKS;
constexpr int kTraceBlock = 128;
/// Largest per-sample colour scratch a split-schedule render may use.
constexpr size_t kSplitScratchMaxBytes = size_t(256) << 20;

/// Resident blocks per SM of the megakernel (for sizing its persistent grid).
int megakernel_blocks_per_sm(bool instrumented);

/// K1: renders samples [sample_index, sample_index + sample_count) of every
/// pixel and adds each pixel's sum into `film` (3 planes of width*height).
/// `counters` must be zeroed before the launch.
cudaError_t launch_megakernel(const SceneView& s, const DCamera& cam, const DConfig& cfg,
                              uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                              float* film, DeviceCounters* counters, bool instrumented, int grid,
                              cudaStream_t stream);

/// K1 in the split schedule for small images: every (pixel, sample) is its own
/// work item; the path colours go to `scratch` (sample_count x 3 planes of
/// width*height) and are then added into `film` in sample order.  Same result
/// bits as launch_megakernel.  `counters` must be zeroed before the launch.
cudaError_t launch_megakernel_split(const SceneView& s, const DCamera& cam, const DConfig& cfg,
                                    uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                                    float* film, float* scratch, DeviceCounters* counters, bool instrumented, int grid,
                                    cudaStream_t stream);

struct WfView;

/// Resident blocks per SM of the multi-view megakernel.
int megakernel_views_blocks_per_sm();

/// K1b: the megakernel over many views (see WfView) of the scenes in `scenes`;
/// each view's film receives the bits launch_megakernel would give it.
/// `counters` must be zeroed before the launch; kernel self-check failures
/// are ORed into `*fault`.
cudaError_t launch_megakernel_views(const WfView* views, uint32_t num_views, uint32_t total_items, uint32_t max_spp,
                                    const SceneView* scenes, const DConfig& cfg, DeviceCounters* counters,
                                    unsigned int* fault, int grid, cudaStream_t stream);

/// Sum pass of the split views of launch_megakernel_views (see WfView::split).
cudaError_t launch_sum_samples_views(const WfView* views, uint32_t num_views, uint64_t total_floats,
                                     cudaStream_t stream);

/// K9: closest-hit or any-hit queries for a batch of rays.
cudaError_t launch_trace(const SceneView& s, const SolGpuRay* rays, uint32_t count, bool any_hit,
                         SolGpuHit* hits, cudaStream_t stream);

}  // namespace sol_b200
