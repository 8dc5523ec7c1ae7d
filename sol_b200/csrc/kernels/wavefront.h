// Device-side structures of the batched renderers (host and device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../core/layout.h"

namespace sol_b200 {

/// Hit bins: one per BSDF kind (SOL_GPU_BSDF_*), the last for misses and hits
/// without a BSDF (and for everything when binning is off).
constexpr int kWfBins = 6;

#ifndef SOL_WF_REFILL_BELOW
#define SOL_WF_REFILL_BELOW 20
#endif
/// A traversal warp pauses to give idle lanes new rays once fewer than this
/// many of its 32 lanes are still traversing (32 + 1 would refill after every
/// leaf, 1 never before the warp drains).
constexpr int kWfRefillBelow = SOL_WF_REFILL_BELOW;

#ifndef SOL_WF_TRACE_MIN_BLOCKS
#define SOL_WF_TRACE_MIN_BLOCKS 6
#endif
/// Resident 256-thread blocks per SM the traversal stages' registers must allow.
constexpr int kWfTraceMinBlocks = SOL_WF_TRACE_MIN_BLOCKS;

#ifndef SOL_WF_SHADE_MIN_BLOCKS
#define SOL_WF_SHADE_MIN_BLOCKS 3
#endif
/// Resident 256-thread blocks per SM the shading stage's registers must allow.
constexpr int kWfShadeMinBlocks = SOL_WF_SHADE_MIN_BLOCKS;

#ifndef SOL_WF_SHADE_RESTART
#define SOL_WF_SHADE_RESTART 1
#endif
/// 1: a path that ends in the shade stage with no shadow ray pending (a miss,
/// the path length, roulette, a failed BSDF sample) restarts its slot right
/// there -- colour out, next work item, camera ray into the next extend queue
/// -- instead of going through the ended list and the next generate stage.

#ifndef SOL_WF_GEN_SMEM_VIEWS
#define SOL_WF_GEN_SMEM_VIEWS 1
#endif
/// The generate stage copies view tables of up to this many views into shared
/// memory (SOL_WF_GEN_SMEM_VIEWS=0: reads them from global memory).
constexpr uint32_t kGenSmemViews = 64;

#ifndef SOL_WF_SHARED_STACK
#define SOL_WF_SHARED_STACK 0
#endif
/// 1: the traversal stages keep the first kSharedStackDepth entries of each
/// lane's stack in shared memory (dynamic, sized by the block), the rest in
/// local memory; 0: the whole stack in local memory (measured 3 % faster on
/// the 64-view batch: the L1 it leaves caches the stack and the upper nodes).
constexpr bool kWfSharedStack = SOL_WF_SHARED_STACK != 0;

/// Scenes one wavefront batch may hold: they travel with every stage launch as
/// a kernel parameter, and a ray carries its scene's index in the bits above
/// its slot number.
constexpr uint32_t kWfMaxScenes = 64;
constexpr uint32_t kWfSlotBits = 26;
constexpr uint32_t kWfSlotMask = (1u << kWfSlotBits) - 1u;
/// Largest pool (slots in flight) of the wavefront.
constexpr uint32_t kWfMaxCapacity = 1u << kWfSlotBits;

struct WfSceneTable {
    SceneView v[kWfMaxScenes];
};

/// Ray reordering (SolGpuBatchOptions::ray_order = SOL_GPU_RAY_ORDER_SORTED):
/// before each traversal stage the queue is counting-sorted by a key of
/// kWfSortBits bits -- the ray's scene, the octant of its direction and the
/// Morton cell of its origin in the scene's bounds -- so that neighbouring
/// lanes start in the same part of the hierarchy.  Measured slower than the
/// queue's own order (64 views: 725 against 789 Mpaths/s; 32 scenes: 1823
/// against 2221): the cells are coarse and the scatter shuffles rays inside a
/// cell, losing the pixel tiles' coherence; off by default.
constexpr int kWfSortBits = 14;
constexpr uint32_t kWfSortBins = 1u << kWfSortBits;

/// One view of a batch: a constructed camera, its film and sample range.
/// Work items are 8x4 pixel tiles of 32 items each; split views (every
/// wavefront view, and the multi-view megakernel's views of more than one
/// sample) have one item per (sample, pixel), taken sample-major, and write
/// each path's colour to `scratch`, which the sum pass adds per pixel in sample
/// order.  The multi-view megakernel's scratch is sample_count x 3 planes of
/// the image; the wavefront's is one float4 per work item, in item order (the
/// items in flight are a contiguous range, so their colours land in a few MB
/// that L2 keeps until every 32-byte sector is complete).
struct WfView {
    float eye[3], dir[3], right[3], up[3];
    uint32_t scene;          // index into the batch's scenes
    uint32_t width, height;
    uint32_t sample_count;   // samples of this launch
    uint64_t sample_index;   // first sample of this launch
    float* film;             // device film, 3 planes of width*height, +=
    uint32_t item_begin;     // first work item of this view
    uint32_t tiles_x;
    uint32_t split;
    float* scratch;
    uint64_t sum_begin;      // the view's first float in the sum pass
    // Samples of a view rendered over several launches (the wavefront's sample
    // chunks): the pixel sums carried from chunk to chunk, or null.
    float* running;
    uint32_t first_chunk;    // the sum starts from 0 (else from `running`)
    uint32_t last_chunk;     // the sum goes into the film (else into `running`)
};

static_assert(sizeof(WfView) % 16 == 0, "the generate stage copies views as 16-byte words");

struct WfCounters {
    uint32_t extend[2];      // rays queued for the closest-hit stage, by parity
    uint32_t ended[2];       // slots whose path ended, by parity
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
///
/// Path state lives per slot; rays travel in queues by value (origin and
/// direction, the slot and scene in the direction's w), so the traversal
/// stages read their input and write their output in queue order.
struct WfParams {
    uint32_t capacity;
    uint32_t sort_threshold;
    uint32_t num_views;
    uint32_t total_items;
    unsigned long long max_iterations;   // self-check bound on bounce-loop iterations
    int refill_below;        // a traversal warp refills its idle lanes when fewer than this many are busy
    uint32_t keep_counts;    // 1: add this launch's paths and rays to the counters instead of restarting them
    uint32_t ray_sort;       // 1: reorder each ray queue before it is traced (see kWfSortBits)
    uint32_t shadow_packed;  // 1: shadow rays staged at their extend position, packed in extend order
    uint32_t scene_bits;     // bits of the sort key taken by the scene index
    const float4* scene_box; // per scene: lower corner, upper corner (2 float4)
    uint32_t* sort_key;      // per queue position: the ray's key (scratch of the reordering)
    uint32_t* sort_bins;     // kWfSortBins counts, then kWfSortBins offsets
    float4* alt[3];          // spare queue arrays: reordered rays land here and swap places with the queue's
    DConfig cfg;
    const WfView* views;
    WfCounters* ctr;
    // per slot
    float4* thru;            // throughput, pdf_prev
    float4* color;           // radiance gathered so far, path_len (bits)
    unsigned long long* rng;
    uint2* item;             // the slot's work item: view, item within the view (view = idle: none)
    // per queue position
    float4* ray_o[2];        // extend queue by parity: origin, tmin
    float4* ray_d[2];        //                         direction, slot | scene << kWfSlotBits (bits)
    float4* hit;             // closest hit of extend position i: triangle slot (int bits, -1: miss), t, u, v
    uint32_t* q_bins;        // kWfBins * capacity extend positions
    float4* sh_o;            // shadow queue: origin, slot | scene << kWfSlotBits (bits)
    float4* sh_d;            //               direction, 1 when the path ends after it
    float4* sh_c;            //               unoccluded contribution
    uint32_t* q_ended[2];    // ended slots by parity
};

/// Grid and block of each stage: generate, extend, shade, shadow.
struct WfLaunch {
    int grid[4];
    int block[4];
    int sms;                 // multiprocessors of the device (grids of the reordering kernels)
};

int wavefront_blocks_per_sm(int stage, int block);
cudaError_t launch_wf_init(const WfParams* params, uint32_t capacity, cudaStream_t stream);
/// One bounce of the wavefront: generate, extend, shade, shadow, advance.
/// `basic`: every scene has basic shading (shade's build without image
/// textures and Interp BSDFs).
/// `ray_sort`: reorder the extend and shadow queues before they are traced
/// (WfParams::ray_sort must agree); `packed_shadows`: pack the shadow queue in
/// extend order (WfParams::shadow_packed must agree).  `params` is in device memory; the
/// reordering swaps queue arrays in it.
cudaError_t launch_wf_iteration(WfParams* params, const WfSceneTable& scenes, bool basic, bool ray_sort,
                                bool packed_shadows, const WfLaunch& launch, cudaGraphConditionalHandle handle,
                                int use_handle, cudaStream_t stream);
/// Lets the reordering's histogram kernel use kWfSortBins * 4 bytes of shared memory (current device).
cudaError_t allow_sort_smem();

}  // namespace sol_b200
