// Test infrastructure (oracle): single-ray stack traversal with the interface
// SoL uses: traverse<IsAnyHit>(ray, bvh, leaf_fn).  Near child first by slab
// entry distance; box tests are widened like the GPU's so both are conservative.
#pragma once

#include <optional>
#include <type_traits>

#include "bvh/bvh.h"
#include "proto/ray.h"

namespace bvh {

template <typename B>
struct SingleRayTraverser {
    static bool slab(const sol_b200::bvh::BBox& b, const proto::Rayf& r, const sol_b200::Vec3& idir, float* tnear) {
        float t0x = (b.lo[0] - r.org[0]) * idir.x, t1x = (b.hi[0] - r.org[0]) * idir.x;
        float t0y = (b.lo[1] - r.org[1]) * idir.y, t1y = (b.hi[1] - r.org[1]) * idir.y;
        float t0z = (b.lo[2] - r.org[2]) * idir.z, t1z = (b.hi[2] - r.org[2]) * idir.z;
        float n = std::max(std::max(std::min(t0x, t1x), std::min(t0y, t1y)), std::max(std::min(t0z, t1z), r.tmin));
        float f = std::min(std::min(std::max(t0x, t1x), std::max(t0y, t1y)), std::min(std::max(t0z, t1z), r.tmax)) * sol_b200::kSlabWiden;
        *tnear = n;
        return n <= f;
    }

    template <bool IsAnyHit, typename F>
    static auto traverse(proto::Rayf& ray, const B& bvh, F&& leaf_fn) {
        using Result = std::invoke_result_t<F, proto::Rayf&, const typename B::Node&>;
        Result best{};
        if (bvh.nodes.empty()) return best;
        const sol_b200::Vec3 idir = sol_b200::safe_inverse(proto::to_m(ray.dir));
        size_t stack[128];
        int sp = 0;
        float tn;
        if (!slab(bvh.nodes[0].box, ray, idir, &tn)) return best;
        stack[sp++] = 0;
        while (sp > 0) {
            const auto& n = bvh.nodes[stack[--sp]];
            if (n.is_leaf()) {
                auto r = leaf_fn(ray, n);
                if (r) {
                    best = r;
                    if constexpr (IsAnyHit) return best;
                }
                continue;
            }
            float n0, n1;
            bool h0 = slab(bvh.nodes[n.first_index].box, ray, idir, &n0);
            bool h1 = slab(bvh.nodes[n.first_index + 1].box, ray, idir, &n1);
            if (h0 && h1) {
                size_t near = n.first_index, far = n.first_index + 1;
                if (n1 < n0) std::swap(near, far);
                stack[sp++] = far;
                stack[sp++] = near;
            } else if (h0) {
                stack[sp++] = n.first_index;
            } else if (h1) {
                stack[sp++] = n.first_index + 1;
            }
        }
        return best;
    }
};

} // namespace bvh
