// K9: batched closest-hit / any-hit queries, the device side of
// TriangleMesh::intersect_closest and TriangleMesh::intersect_any
// (src/triangle_mesh.cpp:64-117) for raw rays.  One thread per ray; used to
// check hit identities against the host checker and to time traversal alone.
#include <cuda_runtime.h>

#include "kernels.h"
#include "traverse.cuh"

namespace sol_b200 {

namespace {

template <bool kAnyHit>
__global__ void __launch_bounds__(kTraceBlock)
trace_rays(SceneView s, const SolGpuRay* __restrict__ rays, uint32_t count, SolGpuHit* __restrict__ hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4 a = __ldg(reinterpret_cast<const float4*>(rays + i));
    const float4 b = __ldg(reinterpret_cast<const float4*>(rays + i) + 1);
    const Vec3 org = vec3(a.x, a.y, a.z), dir = vec3(b.x, b.y, b.z);
    float tmax = b.w;
    TraversalCounters tc{0u, 0u};
    const int slot = traverse<kAnyHit, false>(s, org, dir, a.w, tmax, tc);
    SolGpuHit h;
    h.tri = -1; h.t = 0.0f; h.u = 0.0f; h.v = 0.0f;
    if (slot >= 0) {
        const DTri* tp = s.tris + slot;
        const float4 p0 = ldg4(tp->v0), p1 = ldg4(tp->v1), p2 = ldg4(tp->v2);
        h.tri = (int32_t)__float_as_uint(p0.w);
        h.t = tmax;
        if (!kAnyHit) {
            float tt;
            intersect_triangle(make_shear(org, dir), tri_vertex(p0), tri_vertex(p1), tri_vertex(p2),
                               a.w, kFloatMax, &tt, &h.u, &h.v);
        }
    }
    hits[i] = h;
}

}  // namespace

cudaError_t launch_trace(const SceneView& s, const SolGpuRay* rays, uint32_t count, bool any_hit,
                         SolGpuHit* hits, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    const uint32_t grid = (count + kTraceBlock - 1) / kTraceBlock;
    if (any_hit) trace_rays<true><<<grid, kTraceBlock, 0, stream>>>(s, rays, count, hits);
    else trace_rays<false><<<grid, kTraceBlock, 0, stream>>>(s, rays, count, hits);
    return cudaGetLastError();
}

}  // namespace sol_b200
