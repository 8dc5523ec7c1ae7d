// Device layout of an uploaded scene (shared by the host flattener and kernels).
//
//  nodes   : BVH2, one 64-byte record per inner node holding the boxes of both
//            children and their references, read as four 16-byte vectors.
//  tris    : one 48-byte record per triangle in BVH leaf order, the three
//            vertices for the watertight test; the w lanes carry the caller's
//            triangle index, the BSDF and the light of the triangle.
//  shade   : one 80-byte record per triangle in the same order: vertex normals,
//            texture coordinates, the face normal (computed from the leaf-order
//            vertices by the shared math) and the BSDF and light of the
//            triangle, everything a closest hit's surface needs besides the
//            barycentrics, fetched once per closest hit.
//  bsdfs, textures, images, lights: small tables; image texels are planar.
#pragma once

#include <stdint.h>

namespace sol_b200 {

/// Child reference of a BVH2 node: >= 0 is an inner node index; < 0 is a leaf,
/// ~ref = (first_triangle << 3) | (count - 1), so leaves hold 1..8 triangles.
constexpr int32_t kLeafMaxTris = 8;
constexpr int32_t kStackSentinel = (int32_t)0x80000000;   // never a valid reference
constexpr uint32_t kMaxTriangles = (1u << 28) - 2;
constexpr int kTraversalStack = 64;                        // >= BVH depth - 1

struct alignas(16) DNode {
    float b0[4];    // c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y
    float b1[4];    // c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y
    float b2[4];    // c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z
    int32_t ref[4]; // c0, c1, (unused), (unused)
};
static_assert(sizeof(DNode) == 64, "node layout");

struct alignas(16) DTri {
    float v0[3]; uint32_t prim;   // caller's triangle index
    float v1[3]; int32_t bsdf;    // -1: none
    float v2[3]; int32_t light;   // -1: not emissive
};
static_assert(sizeof(DTri) == 48, "triangle layout");

struct alignas(16) DTriShade {
    float n0[3]; float uv0x;
    float n1[3]; float uv0y;
    float n2[3]; float uv1x;
    float uv1y, uv2x, uv2y; int32_t bsdf;   // -1: none
    float fn[3]; int32_t light;             // face normal normalize((v1 - v0) x (v2 - v0)); light, -1: none
};
static_assert(sizeof(DTriShade) == 80, "shading layout");

/// Bsdf::Type (include/sol/bsdfs.h:39-43).
enum : int32_t { kTypeDiffuse = 0, kTypeGlossy = 1, kTypeSpecular = 2 };

struct DBsdf {
    int32_t kind;       // SOL_GPU_BSDF_*
    int32_t tex[3];
    int32_t a, b;       // interp operands
    int32_t type;       // kType*
    int32_t pad;
};

struct DTexture {
    int32_t kind;       // SOL_GPU_TEX_*
    int32_t filter, border, image;
    float v[3];
    int32_t pad;
};

struct DImage {
    uint64_t offset;    // first texel of the R plane in the texel arena
    uint32_t width, height;
};

struct DLight {
    int32_t kind;       // SOL_GPU_LIGHT_*
    int32_t tex;        // intensity texture (area lights)
    float inv_area;
    float radius;
    float v0[3]; float pad0;
    float v1[3]; float pad1;
    float v2[3]; float pad2;
    float n[3];  float pad3;     // triangle normal
    float intensity[3]; float pad4;
};

/// PerspectiveCamera after its constructor (src/cameras.cpp:5-21): right and
/// up are already scaled by the half-extents of the image plane.
struct DCamera {
    float eye[3], dir[3], right[3], up[3];
};

struct DConfig {
    uint32_t max_path_len;
    uint32_t min_rr_path_len;
    float min_survival_prob;
    float max_survival_prob;
    float ray_offset;
};

struct SceneView {
    const DNode* nodes;
    const DTri* tris;
    const DTriShade* shade;
    const DBsdf* bsdfs;
    const DTexture* textures;
    const DImage* images;
    const float* texels;
    const DLight* lights;
    uint32_t num_lights;
    uint32_t num_tris;
    const unsigned long long* param_offsets;   // per texture, into the parameter vector
    uint32_t num_nodes;
    uint32_t max_steps;      // bound on traversal loop iterations (a tree never needs more)
    unsigned int* fault;     // device word; kernels OR kFault* bits into it instead of looping or reading out of bounds
};

/// Bits a kernel records in SceneView::fault when a self-check fails.
enum : unsigned int {
    kFaultTraversalSteps = 1u,   // a traversal exceeded max_steps
    kFaultNodeIndex = 2u,        // a node reference outside the node array
    kFaultTriIndex = 4u,         // a triangle slot outside the triangle array
    kFaultPathLoop = 8u,         // a render loop exceeded its iteration bound
    kFaultClaimLoop = 16u,       // the pixel-claim loop exceeded its iteration bound
};

/// Per-launch counters and status, zeroed before each launch.
struct DeviceCounters {
    unsigned long long paths;
    unsigned long long rays;
    unsigned long long shadow_rays;
    unsigned long long nodes;
    unsigned long long tris;
    uint32_t next_item;
    uint32_t error;
};

}  // namespace sol_b200
