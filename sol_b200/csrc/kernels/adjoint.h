// Launchers of the adjoint (K7) and loss (K8) kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../core/layout.h"

namespace sol_b200 {

#ifndef SOL_ADJOINT_MIN_BLOCKS
#define SOL_ADJOINT_MIN_BLOCKS 16  // resident blocks per SM the register allocation must allow (32 registers; measured fastest)
#endif
constexpr int kAdjointBlock = 128;
constexpr int kAdjointMinBlocks = SOL_ADJOINT_MIN_BLOCKS;
/// Longest path the adjoint replays (vertex records per lane).
constexpr int kAdjointMaxDepth = 16;

/// One view of a fused forward + adjoint batch.
struct AdjView {
    DCamera cam;
    uint32_t scene;
    uint32_t width, height;
    uint32_t sample_count;
    uint64_t sample_index;
    float* film;            // forward sums are added into
    const float* target;    // the loss compares (sum / sample_count) with it
    float* grad;            // the scene's parameter gradient, added into
    double* loss;           // added into
    uint32_t item_begin;    // first work item of the view (fused_items per view, in order)
    uint32_t group;         // lanes per pixel (fused_group of sample_count)
};

/// Lanes per pixel of the fused kernel for a view of `spp` samples: the
/// smallest power of two >= spp, at most 32.
inline uint32_t fused_group(uint32_t spp) {
    uint32_t g = 1;
    while (g < spp && g < 32) g <<= 1;
    return g;
}

/// Work items (one warp each) of a width x height view in the fused kernel:
/// 8x4-pixel tiles, 32 / g pixels per item.
inline uint64_t fused_items(uint32_t width, uint32_t height, uint32_t spp) {
    return (uint64_t)((width + 7) / 8) * ((height + 3) / 4) * fused_group(spp);
}

/// Most constant-texture values whose gradients a block gathers in shared memory.
constexpr uint32_t kAdjointMaxSharedParams = 2048;   // 8 KB per block, so 16 blocks fit an SM

int adjoint_blocks_per_sm(uint32_t n_shared);
int fused_blocks_per_sm();

/// Forward render + L2-loss adjoint of every view in one persistent launch.
cudaError_t launch_fused_forward_adjoint(const AdjView* views, uint32_t num_views, uint32_t total_items,
                                         const SceneView* scenes, const DConfig& cfg, DeviceCounters* counters, int grid,
                                         cudaStream_t stream);

/// Adds dL/d(parameters) of the paths of samples [sample_index, + sample_count)
/// of every pixel into `grad`, given dL/dfilm (3 planes of width*height).  Each
/// work item replays `chunk` consecutive samples of one pixel; the first
/// `n_shared` parameters (at most kAdjointMaxSharedParams, all of them constant
/// textures) are gathered per block in shared memory.
/// With `texels4` (num_texels float4, one per image texel in arena order) the
/// image-texel gradients are gathered there with vector reductions and added
/// into `grad` afterwards (parameter first_texel_param + image offset + ...).
cudaError_t launch_adjoint(const SceneView& s, const DCamera& cam, const DConfig& cfg, uint64_t sample_index,
                           uint32_t sample_count, uint32_t chunk, uint32_t width, uint32_t height,
                           const float* dl_dfilm, float* grad, uint32_t n_shared, float4* texels4, uint64_t num_texels,
                           uint32_t num_images, uint64_t first_texel_param, DeviceCounters* counters, int grid,
                           cudaStream_t stream);

/// Adds sum (scale * film - target)^2 into *loss and writes dL/dfilm (optional).
cudaError_t launch_l2_loss(const float* film, const float* target, uint64_t n, float scale, float* dl_dfilm,
                           double* loss, int grid, cudaStream_t stream);

}  // namespace sol_b200
