// Test infrastructure (oracle): clean-room stand-in for bvh v2's Bvh<float> as
// SoL uses it (src/triangle_mesh.cpp:27-28,65-117,119-146).  The tree itself is
// the product's host builder output (sol_b200::bvh), so that SoL's TriangleMesh
// and the GPU path traverse the same hierarchy.
#pragma once

#include <cstddef>
#include <vector>

#include "host/bvh_builder.h"

namespace bvh {

template <typename T>
struct Bvh {
    struct Node {
        size_t first_index;
        size_t prim_count;
        sol_b200::bvh::BBox box;
        bool is_leaf() const { return prim_count != 0; }
    };
    std::vector<Node> nodes;
    std::vector<size_t> prim_indices;

    template <typename Executor>
    std::vector<size_t> parents(Executor&) const {
        std::vector<size_t> p(nodes.size(), 0);
        for (size_t i = 0; i < nodes.size(); ++i)
            if (!nodes[i].is_leaf()) { p[nodes[i].first_index] = i; p[nodes[i].first_index + 1] = i; }
        return p;
    }

    static Bvh from(const sol_b200::bvh::Bvh& b) {
        Bvh r;
        r.nodes.resize(b.nodes.size());
        for (size_t i = 0; i < b.nodes.size(); ++i)
            r.nodes[i] = Node{b.nodes[i].first, b.nodes[i].count, b.nodes[i].box};
        r.prim_indices.assign(b.prim_indices.begin(), b.prim_indices.end());
        return r;
    }
    sol_b200::bvh::Bvh to_builder() const {
        sol_b200::bvh::Bvh b;
        b.nodes.resize(nodes.size());
        for (size_t i = 0; i < nodes.size(); ++i) {
            b.nodes[i].box = nodes[i].box;
            b.nodes[i].first = (uint32_t)nodes[i].first_index;
            b.nodes[i].count = (uint32_t)nodes[i].prim_count;
        }
        b.prim_indices.assign(prim_indices.begin(), prim_indices.end());
        return b;
    }
};

} // namespace bvh
