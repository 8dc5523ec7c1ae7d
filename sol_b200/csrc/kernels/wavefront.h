// Device-side structures of the batched wavefront renderer (host and device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../core/layout.h"

namespace sol_b200 {

/// Hit bins: one per BSDF kind (SOL_GPU_BSDF_*), the last for hits without a BSDF
/// (and for everything when binning is off).
constexpr int kWfBins = 6;

#ifndef SOL_WF_REFILL_BELOW
#define SOL_WF_REFILL_BELOW 20
#endif
/// A traversal warp pauses to give idle lanes new rays once fewer than this
/// many of its 32 lanes are still traversing (32 + 1 would refill after every
/// leaf, 1 never before the warp drains).
constexpr int kWfRefillBelow = SOL_WF_REFILL_BELOW;

#ifndef SOL_WF_TRACE_MIN_BLOCKS
#define SOL_WF_TRACE_MIN_BLOCKS 5
#endif
/// Resident 256-thread blocks per SM the traversal stages' registers must allow.
constexpr int kWfTraceMinBlocks = SOL_WF_TRACE_MIN_BLOCKS;

/// One view of a batch: a constructed camera, its film and sample range.
struct WfView {
    float eye[3], dir[3], right[3], up[3];
    uint32_t scene;          // index into the batch's scenes
    uint32_t width, height;
    uint32_t sample_count;
    uint64_t sample_index;
    float* film;             // device film, 3 planes of width*height, +=
    uint32_t item_begin;     // first work item of this view (8x4 pixel tiles, 32 items each)
    uint32_t tiles_x;
    // Multi-view megakernel only: split views have one work item per (sample,
    // pixel) and write each sample's colour to `scratch` (sample_count x 3
    // planes); `sum_begin` is the view's first float in the sum pass.
    uint32_t split;
    float* scratch;
    uint64_t sum_begin;
};

struct WfCounters {
    uint32_t extend[2];
    uint32_t regen[2];
    uint32_t bins[kWfBins];
    uint32_t shadow;
    uint32_t fetch_extend;   // rays taken from the extend / shadow queue by the traversal stages
    uint32_t fetch_shadow;
    uint32_t next_item;
    uint32_t iter;
    uint32_t more;
    unsigned long long paths, rays, shadow_rays;
    uint32_t error;
};

/// Everything the stages read, in device memory at a fixed address so that a
/// captured graph can be replayed for new batches.
struct WfParams {
    uint32_t capacity;
    uint32_t sort_threshold;
    uint32_t num_views;
    uint32_t total_items;
    unsigned long long max_iterations;   // self-check bound on bounce-loop iterations
    int refill_below;        // a traversal warp refills its idle lanes when fewer than this many are busy
    DConfig cfg;
    const WfView* views;
    const SceneView* scenes;
    WfCounters* ctr;
    float4* ray_o;       // org, tmin
    float4* ray_d;       // dir, pdf_prev
    float4* thru;        // throughput, path_len
    float4* color;       // radiance of the current path
    unsigned long long* rng;
    uint4* pix;          // view, x, y, sample number (view = 0xffffffff: idle)
    float4* sum;         // the pixel's sum so far
    float4* sh_o;
    float4* sh_d;
    float4* pending;     // light-sample contribution, w = 1 when the path ends after it
    float2* hit;         // triangle slot (int bits), t
    uint32_t* q_extend[2];
    uint32_t* q_regen[2];
    uint32_t* q_bins;    // kWfBins * capacity
    uint32_t* q_shadow;
};

/// Grid and block of each stage: generate, extend, shade, shadow.
struct WfLaunch {
    int grid[4];
    int block[4];
};

int wavefront_blocks_per_sm(int stage, int block);
cudaError_t launch_wf_init(const WfParams* params, uint32_t capacity, cudaStream_t stream);
cudaError_t launch_wf_iteration(const WfParams* params, const WfLaunch& launch, cudaGraphConditionalHandle handle,
                                int use_handle, cudaStream_t stream);

}  // namespace sol_b200
