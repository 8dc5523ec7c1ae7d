// Launchers of the adjoint (K7) and loss (K8) kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../core/layout.h"

namespace sol_b200 {

constexpr int kAdjointBlock = 128;
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
    uint32_t item_begin;    // first work item (8x4 tiles, 32 items each)
};

int adjoint_blocks_per_sm();
int fused_blocks_per_sm();

/// Forward render + L2-loss adjoint of every view in one persistent launch.
cudaError_t launch_fused_forward_adjoint(const AdjView* views, uint32_t num_views, uint32_t total_items,
                                         const SceneView* scenes, const DConfig& cfg, DeviceCounters* counters, int grid,
                                         cudaStream_t stream);

/// Adds dL/d(parameters) of the paths of samples [sample_index, + sample_count)
/// of every pixel into `grad`, given dL/dfilm (3 planes of width*height).
cudaError_t launch_adjoint(const SceneView& s, const DCamera& cam, const DConfig& cfg, uint64_t sample_index,
                           uint32_t sample_count, uint32_t width, uint32_t height, const float* dl_dfilm, float* grad,
                           DeviceCounters* counters, int grid, cudaStream_t stream);

/// Adds sum (scale * film - target)^2 into *loss and writes dL/dfilm (optional).
cudaError_t launch_l2_loss(const float* film, const float* target, uint64_t n, float scale, float* dl_dfilm,
                           double* loss, int grid, cudaStream_t stream);

}  // namespace sol_b200
