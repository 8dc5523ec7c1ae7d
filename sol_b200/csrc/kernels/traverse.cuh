// BVH2 traversal on the device: the GPU statement of
// TriangleMesh::intersect_closest / intersect_any (src/triangle_mesh.cpp:64-117),
// which SoL runs through bvh v2's SingleRayTraverser.
//
// Layout: every inner node is 64 bytes holding both child boxes, fetched as four
// 128-bit read-only loads; triangles are 48 bytes (three 128-bit loads).  The
// traversal is the stack-based "while-while" loop of Aila & Laine ("Understanding
// the Efficiency of Ray Traversal on GPUs", HPG 2009): descend inner nodes
// nearest-child first, pushing the farther child, until a leaf is reached; then
// test the leaf's triangles.  Box tests compute (bound - origin) / direction and
// widen the exit distance by kSlabWiden so that they are conservative; they are
// the same operations as the host traversal's, so both visit children in the same
// order and resolve equal-distance hits alike.  The triangle test is the shared
// watertight test, so a hit found here is bit-identical to the one the host finds.
#pragma once

#include "../core/layout.h"
#include "../core/math.h"

namespace sol_b200 {

struct TraversalCounters {
    uint32_t nodes;
    uint32_t tris;
};

__device__ __forceinline__ float4 ldg4(const void* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

/// Traversal stack in local memory.
struct LocalStack {
    int v[kTraversalStack];
    __device__ __forceinline__ void put(int i, int x) { v[i] = x; }
    __device__ __forceinline__ int get(int i) const { return v[i]; }
};

#ifndef SOL_SHARED_STACK_DEPTH
#define SOL_SHARED_STACK_DEPTH 16
#endif
/// Entries of the traversal stack kept in shared memory by SharedStack.
constexpr int kSharedStackDepth = SOL_SHARED_STACK_DEPTH;

/// Traversal stack whose first kSharedStackDepth entries live in shared memory,
/// laid out entry-major ([entry][thread] for kThreads threads, so a warp's
/// accesses at any mix of depths fall in distinct banks); deeper entries, which
/// few rays reach, go to local memory.  `column` is the thread's first entry:
/// shared_array + threadIdx.x.
template <int kThreads>
struct SharedStack {
    int* column;
    int deep[kTraversalStack - kSharedStackDepth];
    __device__ __forceinline__ void put(int i, int x) {
        if (i < kSharedStackDepth) column[i * kThreads] = x;
        else deep[i - kSharedStackDepth] = x;
    }
    __device__ __forceinline__ int get(int i) const {
        return i < kSharedStackDepth ? column[i * kThreads] : deep[i - kSharedStackDepth];
    }
};

/// SharedStack with the thread stride given at run time (the block size), for
/// kernels launched with several block sizes: `column` = a dynamic shared
/// array of kSharedStackDepth * blockDim.x ints + threadIdx.x.
struct SharedStackDyn {
    int* column;
    int stride;
    int deep[kTraversalStack - kSharedStackDepth];
    __device__ __forceinline__ void put(int i, int x) {
        if (i < kSharedStackDepth) column[i * stride] = x;
        else deep[i - kSharedStackDepth] = x;
    }
    __device__ __forceinline__ int get(int i) const {
        return i < kSharedStackDepth ? column[i * stride] : deep[i - kSharedStackDepth];
    }
};

__device__ __forceinline__ Vec3 tri_vertex(float4 a) { return vec3(a.x, a.y, a.z); }

__device__ __forceinline__ float fminf3(float a, float b, float c) { return fminf(fminf(a, b), c); }
__device__ __forceinline__ float fmaxf3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }

/// Entry and (widened) exit distances of a ray against both child boxes of a
/// node: a = c0.x and c0.y bounds, b = c1.x and c1.y bounds, c = both z bounds.
/// (bound - org) * (1/dir) takes two correctly rounded operations per plane, so
/// the widened exit distance stays conservative even for grazing rays (the
/// product-with-offset form loses |org / dir| ulps to cancellation).
__device__ __forceinline__ void child_slabs(float4 a, float4 b, float4 c, Vec3 org, Vec3 idir, float tmin,
                                            float tmax, float& n0, float& f0, float& n1, float& f1) {
    const float t0lx = (a.x - org.x) * idir.x, t0hx = (a.y - org.x) * idir.x;
    const float t0ly = (a.z - org.y) * idir.y, t0hy = (a.w - org.y) * idir.y;
    const float t0lz = (c.x - org.z) * idir.z, t0hz = (c.y - org.z) * idir.z;
    const float t1lx = (b.x - org.x) * idir.x, t1hx = (b.y - org.x) * idir.x;
    const float t1ly = (b.z - org.y) * idir.y, t1hy = (b.w - org.y) * idir.y;
    const float t1lz = (c.z - org.z) * idir.z, t1hz = (c.w - org.z) * idir.z;
    n0 = fmaxf3(fminf(t0lx, t0hx), fminf(t0ly, t0hy), fmaxf(fminf(t0lz, t0hz), tmin));
    f0 = fminf3(fmaxf(t0lx, t0hx), fmaxf(t0ly, t0hy), fminf(fmaxf(t0lz, t0hz), tmax)) * kSlabWiden;
    n1 = fmaxf3(fminf(t1lx, t1hx), fminf(t1ly, t1hy), fmaxf(fminf(t1lz, t1hz), tmin));
    f1 = fminf3(fmaxf(t1lx, t1hx), fmaxf(t1ly, t1hy), fminf(fmaxf(t1lz, t1hz), tmax)) * kSlabWiden;
}

/// BVH traversal of one ray as a resumable state: start() sets it up, run()
/// advances it.  For kAnyHit the first triangle hit inside (tmin, tmax) is
/// kept; otherwise the closest one, with `tmax` shrunk to its distance.  `hit`
/// is the triangle's position in leaf order, or -1.
///
/// With kYield, run() may return early, after a leaf, when fewer than
/// `min_active` lanes of the warp are still traversing: the caller gives the
/// lanes whose rays are done new rays and calls run() again, which continues
/// exactly where it stopped (dynamic ray fetch; Aila & Laine, "Understanding
/// the Efficiency of Ray Traversal on GPUs", HPG 2009).  Stopping changes
/// nothing in the order nodes and triangles are visited, so the result is the
/// same as an uninterrupted traversal.
///
/// Self-checks: at most `max_steps` steps, node and triangle references checked
/// against the array sizes and the stack against its capacity; a failed check
/// ORs a kFault* bit into `*fault` and ends the traversal with no hit.
template <bool kAnyHit, bool kCount, bool kYield>
struct Traversal {
    Vec3 org, dir, idir;
    RayShear rs;
    float tmin, tmax;
    int node, sp, hit;
    float hu, hv;   // barycentrics of the closest hit (kAnyHit: unused)
    uint32_t steps;

    template <class Stack>
    __device__ __forceinline__ void start(Vec3 o, Vec3 d, float t0, float t1, bool active, Stack& stack) {
        org = o;
        dir = d;
        tmin = t0;
        tmax = t1;
        idir = safe_inverse(d);
        rs = make_shear(o, d);
        sp = 0;
        hit = -1;
        hu = hv = 0.0f;
        steps = 0;
        node = active ? 0 : kStackSentinel;
        stack.put(sp++, kStackSentinel);
    }

    __device__ __forceinline__ bool fail(unsigned int* fault, unsigned int bit) {
        atomicOr(fault, bit);
        hit = -1;
        node = kStackSentinel;
        return true;
    }

    /// Advances the traversal; true when it has finished.
    template <class Stack>
    __device__ __forceinline__ bool run(const DNode* __restrict__ nodes, const DTri* __restrict__ tris,
                                        TraversalCounters& ctr, uint32_t num_nodes, uint32_t num_tris,
                                        uint32_t max_steps, unsigned int* fault, Stack& stack, int min_active) {
        while (node != kStackSentinel) {
            // Descend inner nodes until a leaf (or the end) is reached.
            while (node >= 0) {
                if (++steps > max_steps) return fail(fault, kFaultTraversalSteps);
                if ((uint32_t)node >= num_nodes) return fail(fault, kFaultNodeIndex);
                const DNode* n = nodes + node;
                const float4 a = ldg4(n->b0);
                const float4 b = ldg4(n->b1);
                const float4 c = ldg4(n->b2);
                const int4 r = __ldg(reinterpret_cast<const int4*>(n->ref));
                if (kCount) ctr.nodes++;
                float n0, f0, n1, f1;
                child_slabs(a, b, c, org, idir, tmin, tmax, n0, f0, n1, f1);
                const bool h0 = n0 <= f0, h1 = n1 <= f1;
                if (h0 && h1) {
                    int near = r.x, far = r.y;
                    if (n1 < n0) { near = r.y; far = r.x; }
                    if (sp >= kTraversalStack) return fail(fault, kFaultTraversalSteps);
                    stack.put(sp++, far);
                    node = near;
                } else if (h0) {
                    node = r.x;
                } else if (h1) {
                    node = r.y;
                } else {
                    if (sp <= 0) return fail(fault, kFaultTraversalSteps);
                    node = stack.get(--sp);
                }
            }
            if (node == kStackSentinel) break;
            // Leaf: ~node = (first << 3) | (count - 1)
            const uint32_t v = ~(uint32_t)node;
            const uint32_t first = v >> 3, count = (v & 7u) + 1u;
            if (first + count > num_tris) return fail(fault, kFaultTriIndex);
            if (++steps > max_steps) return fail(fault, kFaultTraversalSteps);
            for (uint32_t i = first; i < first + count; ++i) {
                const DTri* tp = tris + i;
                const float4 p0 = ldg4(tp->v0), p1 = ldg4(tp->v1), p2 = ldg4(tp->v2);
                if (kCount) ctr.tris++;
                float t, u, w;
                if (intersect_triangle(rs, tri_vertex(p0), tri_vertex(p1), tri_vertex(p2), tmin, tmax, &t, &u, &w)) {
                    hit = (int)i;
                    tmax = t;
                    if (kAnyHit) break;
                    hu = u;
                    hv = w;
                }
            }
            if (kAnyHit && hit >= 0) return true;
            if (sp <= 0) return fail(fault, kFaultTraversalSteps);
            node = stack.get(--sp);
            if (kYield && node != kStackSentinel && __popc(__activemask()) < min_active) return false;
        }
        return true;
    }
};

/// Traverses the BVH for one ray to completion (see Traversal).  Returns the
/// hit triangle's position in leaf order, or -1; `tmax` becomes the hit
/// distance.  `active == false` lanes return -1 at once.
template <bool kAnyHit, bool kCount, class Stack>
__device__ __forceinline__ int traverse_bounded(const DNode* __restrict__ nodes, const DTri* __restrict__ tris,
                                        Vec3 org, Vec3 dir, float tmin, float& tmax, bool active,
                                        TraversalCounters& ctr, uint32_t num_nodes, uint32_t num_tris,
                                        uint32_t max_steps, unsigned int* fault, Stack& stack) {
    Traversal<kAnyHit, kCount, false> tr;
    tr.start(org, dir, tmin, tmax, active, stack);
    tr.run(nodes, tris, ctr, num_nodes, num_tris, max_steps, fault, stack, 0);
    tmax = tr.tmax;
    return tr.hit;
}

/// Closest-hit traverse_bounded over a scene view that also returns the hit's
/// barycentrics (u, v) as the triangle test computed them.
template <bool kCount, class Stack>
__device__ __forceinline__ int traverse_closest_uv(const SceneView& s, Vec3 org, Vec3 dir, float tmin, float& tmax,
                                                   float& u, float& v, TraversalCounters& ctr, Stack& stack) {
    Traversal<false, kCount, false> tr;
    tr.start(org, dir, tmin, tmax, s.num_tris > 0, stack);
    tr.run(s.nodes, s.tris, ctr, s.num_nodes, s.num_tris, s.max_steps, s.fault, stack, 0);
    tmax = tr.tmax;
    u = tr.hu;
    v = tr.hv;
    return tr.hit;
}

/// traverse_bounded over the arrays and limits of a scene view, with the given stack.
template <bool kAnyHit, bool kCount, class Stack>
__device__ __forceinline__ int traverse(const SceneView& s, Vec3 org, Vec3 dir, float tmin, float& tmax,
                                        TraversalCounters& ctr, Stack& stack) {
    return traverse_bounded<kAnyHit, kCount>(s.nodes, s.tris, org, dir, tmin, tmax, s.num_tris > 0, ctr, s.num_nodes,
                                             s.num_tris, s.max_steps, s.fault, stack);
}

/// traverse with a stack in local memory.
template <bool kAnyHit, bool kCount>
__device__ __forceinline__ int traverse(const SceneView& s, Vec3 org, Vec3 dir, float tmin, float& tmax,
                                        TraversalCounters& ctr) {
    LocalStack stack;
    return traverse<kAnyHit, kCount>(s, org, dir, tmin, tmax, ctr, stack);
}

}  // namespace sol_b200
