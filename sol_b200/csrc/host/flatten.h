// Scene validation and flattening into the device layout (host only).
#pragma once

#include <string>
#include <vector>

#include "../core/layout.h"
#include "../../../include/sol_gpu.h"
#include "bvh_builder.h"

namespace sol_b200 {

/// Inner nodes of the upper BVH levels stored first, level by level, so that
/// one contiguous range of the node array can be kept resident in L2: whole
/// levels are taken while they fit in this many nodes (64 B each, 16 MiB).
constexpr uint32_t kTopNodesMax = 1u << 18;

struct FlatScene {
    std::vector<DNode> nodes;
    std::vector<DTri> tris;
    std::vector<DTriShade> shade;
    std::vector<DBsdf> bsdfs;
    std::vector<DTexture> textures;
    std::vector<DImage> images;
    std::vector<float> texels;
    std::vector<DLight> lights;
    uint32_t depth = 0;
    uint32_t top_nodes = 0;   // nodes of the upper levels, stored first (breadth first)
    float sah_cost = 0.0f;
    double build_ms = 0.0;
};

/// Builds the BVH SoL's TriangleMesh builds for a mesh (src/triangle_mesh.cpp:119-146):
/// triangle boxes and centroids, full-sweep SAH, then reinsertion.
bvh::Bvh build_mesh_bvh(const float* vertices, const uint32_t* indices, size_t num_triangles);

/// Validates `desc` and produces the device layout. Returns false with a message
/// in `err` on invalid input.
/// With host_bvh == false the BVH, triangle and shading arrays are left empty
/// (the caller builds them on the device).
bool flatten_scene(const SolGpuSceneDesc& desc, FlatScene& out, std::string& err, bool host_bvh = true);

/// PerspectiveCamera's constructor (src/cameras.cpp:5-21).
SolGpuCamera perspective_camera(const float eye[3], const float dir[3], const float up[3], float fov, float aspect);

}  // namespace sol_b200
