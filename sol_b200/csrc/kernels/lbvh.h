// GPU linear-BVH construction (kernels/lbvh.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../core/layout.h"

namespace sol_b200 {

/// Device arrays of a built hierarchy, owned by the caller afterwards.
struct LbvhResult {
    DNode* nodes = nullptr;        // num_nodes entries, node 0 the root (unused entries zeroed)
    DTri* tris = nullptr;          // num_triangles, leaf order
    DTriShade* shade = nullptr;    // num_triangles, leaf order
    uint32_t num_nodes = 0;
    uint32_t depth = 0;            // node levels including the leaf level
    float sah_cost = 0.0f;         // SAH cost (traversal 1, triangle 1) normalised by the root's area
};

/// Builds the hierarchy on the device from device arrays (vertices 3*nv floats,
/// indices 3*nt, normals 3*nv, uvs 2*nv, per-triangle BSDF and light ids).
/// Needs at least 2 triangles.  Synchronises `stream` before returning.
cudaError_t build_lbvh(const float* vertices, const uint32_t* indices, const float* normals, const float* uvs,
                       const int32_t* tri_bsdf, const int32_t* tri_light, uint32_t num_triangles,
                       cudaStream_t stream, LbvhResult* out);

}  // namespace sol_b200
