// Host BVH construction: full-sweep SAH top-down builder plus an insertion-based
// reinsertion optimizer.
//
// SoL builds its mesh BVH with bvh v2's SweepSahBuilder and then runs
// SequentialReinsertionOptimizer over it (src/triangle_mesh.cpp:119-146).  bvh v2
// is an external library that is not vendored with SoL, so this file provides the
// two steps from their published descriptions:
//  * top-down construction choosing, at every node, the split with the lowest
//    surface-area-heuristic cost among all object partitions along the centroid
//    order of each axis (MacDonald & Booth 1990; Wald, Boulos, Shirley 2007);
//  * reinsertion optimization: repeatedly detach the subtrees whose bounding
//    boxes have the largest area and re-insert each at the position found by a
//    branch-and-bound search that minimises the induced SAH cost (Bittner, Hapala,
//    Havran: "Fast Insertion-Based Optimization of Bounding Volume Hierarchies",
//    CGF 2013; Meister & Bittner 2018).
//
// The tree is binary.  Node 0 is the root; the two children of an inner node sit
// at consecutive indices `first` and `first + 1`; a leaf covers `count` entries
// of `prim_indices` starting at `first`.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>
#include <queue>
#include <vector>

namespace sol_b200::bvh {

struct BBox {
    float lo[3], hi[3];
    static BBox empty() {
        BBox b;
        for (int k = 0; k < 3; ++k) { b.lo[k] = std::numeric_limits<float>::infinity(); b.hi[k] = -std::numeric_limits<float>::infinity(); }
        return b;
    }
    void extend(const BBox& o) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], o.lo[k]); hi[k] = std::max(hi[k], o.hi[k]); }
    }
    void extend(const float p[3]) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    /// Half of the surface area (the factor 2 cancels in every SAH ratio).
    float half_area() const {
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (!(dx >= 0.0f && dy >= 0.0f && dz >= 0.0f)) return 0.0f;
        return dx * dy + dy * dz + dz * dx;
    }
    static BBox merge(const BBox& a, const BBox& b) { BBox r = a; r.extend(b); return r; }
};

struct Node {
    BBox box;
    uint32_t first = 0;   ///< inner: left child index (right = first + 1); leaf: first prim slot
    uint32_t count = 0;   ///< leaf: primitive count (> 0); inner: 0
    bool is_leaf() const { return count != 0; }
};

struct Bvh {
    std::vector<Node> nodes;
    std::vector<uint32_t> prim_indices;

    /// SAH cost normalised by the root area, with the given traversal and
    /// intersection costs (inner nodes counted once, leaves by their size).
    double sah_cost(double c_trav = 1.0, double c_isect = 1.0) const {
        if (nodes.empty()) return 0.0;
        double root = nodes[0].box.half_area();
        if (root <= 0.0) return 0.0;
        double cost = 0.0;
        for (auto& n : nodes) {
            double a = n.box.half_area();
            cost += n.is_leaf() ? a * c_isect * n.count : a * c_trav;
        }
        return cost / root;
    }

    /// Parent index of every node (root's parent = itself), for slots in use.
    std::vector<uint32_t> parents() const {
        std::vector<uint32_t> p(nodes.size(), 0);
        std::vector<uint32_t> stack{0};
        while (!stack.empty()) {
            uint32_t i = stack.back(); stack.pop_back();
            if (!nodes[i].is_leaf()) {
                p[nodes[i].first] = i; p[nodes[i].first + 1] = i;
                stack.push_back(nodes[i].first); stack.push_back(nodes[i].first + 1);
            }
        }
        return p;
    }

    uint32_t depth() const {
        uint32_t best = 0;
        std::vector<std::pair<uint32_t, uint32_t>> stack{{0, 1}};
        while (!stack.empty()) {
            auto [i, d] = stack.back(); stack.pop_back();
            best = std::max(best, d);
            if (!nodes[i].is_leaf()) { stack.push_back({nodes[i].first, d + 1}); stack.push_back({nodes[i].first + 1, d + 1}); }
        }
        return best;
    }
};

struct BuildConfig {
    uint32_t min_leaf_size = 1;
    uint32_t max_leaf_size = 8;     ///< also the GPU leaf encoding limit
    float traversal_cost = 1.0f;    ///< relative to one primitive intersection
    uint32_t parallel_threshold = 1u << 14;
};

namespace detail {

struct SweepBuilder {
    const BBox* bboxes;
    const float* centers;           // 3 floats per primitive
    BuildConfig cfg;
    std::vector<uint32_t> order[3]; // primitives sorted by centre along each axis, per node range
    std::vector<uint8_t> goes_left;
    std::vector<uint32_t> scratch;  // partition buffer (per thread ranges are disjoint)
    std::vector<float> right_cost;  // suffix areas (indexed by range position)
    Bvh* out;
    std::atomic<uint32_t> next_node{1};

    struct Task { uint32_t node, begin, end; };

    // Returns true when the node became a leaf.
    bool split(const Task& t, uint32_t& mid) {
        const uint32_t n = t.end - t.begin;
        BBox box = BBox::empty();
        for (uint32_t i = t.begin; i < t.end; ++i) box.extend(bboxes[order[0][i]]);
        out->nodes[t.node].box = box;
        if (n <= cfg.min_leaf_size) return true;

        float best_cost = std::numeric_limits<float>::infinity();
        int best_axis = -1;
        uint32_t best_pos = 0;
        for (int axis = 0; axis < 3; ++axis) {
            const uint32_t* ord = order[axis].data();
            // Right-to-left sweep: area of the suffix [i, end)
            BBox acc = BBox::empty();
            for (uint32_t i = t.end - 1; i > t.begin; --i) {
                acc.extend(bboxes[ord[i]]);
                right_cost[i] = acc.half_area() * (float)(t.end - i);
            }
            acc = BBox::empty();
            for (uint32_t i = t.begin; i < t.end - 1; ++i) {
                acc.extend(bboxes[ord[i]]);
                float c = acc.half_area() * (float)(i + 1 - t.begin) + right_cost[i + 1];
                if (c < best_cost) { best_cost = c; best_axis = axis; best_pos = i + 1; }
            }
        }
        float node_area = box.half_area();
        float leaf_cost = node_area * (float)n;
        float split_cost = node_area * cfg.traversal_cost + best_cost;
        if (best_axis < 0 || (n <= cfg.max_leaf_size && leaf_cost <= split_cost)) {
            if (n <= cfg.max_leaf_size) return true;
        }
        if (best_axis < 0) { best_axis = 0; best_pos = t.begin + n / 2; }
        // Mark the primitives of the left side, then stably partition the other axes.
        for (uint32_t i = t.begin; i < t.end; ++i) goes_left[order[best_axis][i]] = i < best_pos ? 1 : 0;
        for (int axis = 0; axis < 3; ++axis) {
            if (axis == best_axis) continue;
            uint32_t* ord = order[axis].data();
            uint32_t l = t.begin, r = best_pos;
            for (uint32_t i = t.begin; i < t.end; ++i) {
                uint32_t p = ord[i];
                if (goes_left[p]) scratch[l++] = p; else scratch[r++] = p;
            }
            std::memcpy(ord + t.begin, scratch.data() + t.begin, sizeof(uint32_t) * n);
        }
        mid = best_pos;
        return false;
    }

    void build_range(Task root) {
        std::vector<Task> stack{root};
        while (!stack.empty()) {
            Task t = stack.back(); stack.pop_back();
            uint32_t mid = 0;
            if (split(t, mid)) {
                Node& nd = out->nodes[t.node];
                nd.first = t.begin;
                nd.count = t.end - t.begin;
                continue;
            }
            // The node array is preallocated (a binary tree over n primitives has
            // at most 2n - 1 nodes), so slots are claimed with one atomic add.
            uint32_t left = next_node.fetch_add(2, std::memory_order_relaxed);
            out->nodes[t.node].first = left;
            out->nodes[t.node].count = 0;
            Task lt{left, t.begin, mid}, rt{left + 1, mid, t.end};
            bool big = (t.end - t.begin) >= cfg.parallel_threshold;
            if (big) {
                #pragma omp task firstprivate(rt)
                build_range(rt);
                stack.push_back(lt);
            } else {
                stack.push_back(rt);
                stack.push_back(lt);
            }
        }
    }
};

}  // namespace detail

/// Full-sweep SAH build over `n` primitives with the given bounding boxes and
/// centres (3 floats each).  Deterministic: ties in centre order are broken by
/// primitive index, and node numbering does not depend on thread timing because
/// nodes are renumbered depth-first at the end.
inline Bvh build_sweep_sah(const BBox* bboxes, const float* centers, size_t n, const BuildConfig& cfg = {}) {
    Bvh bvh;
    if (n == 0) return bvh;
    detail::SweepBuilder b;
    b.bboxes = bboxes; b.centers = centers; b.cfg = cfg; b.out = &bvh;
    for (int axis = 0; axis < 3; ++axis) {
        b.order[axis].resize(n);
        std::iota(b.order[axis].begin(), b.order[axis].end(), 0u);
        auto& ord = b.order[axis];
        std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) {
            float cx = centers[3 * x + axis], cy = centers[3 * y + axis];
            return cx < cy || (cx == cy && x < y);
        });
    }
    b.goes_left.assign(n, 0);
    b.scratch.assign(n, 0);
    b.right_cost.assign(n + 1, 0.0f);
    bvh.nodes.assign(2 * n, Node{});
    // right_cost is indexed by range position and ranges of concurrent tasks are disjoint.
    #pragma omp parallel
    #pragma omp single
    b.build_range({0, 0, (uint32_t)n});
    bvh.nodes.resize(b.next_node.load());
    bvh.prim_indices = std::move(b.order[0]);

    // Renumber nodes depth-first (left subtree first) so that the result does not
    // depend on task scheduling and siblings stay adjacent.
    std::vector<Node> renum;
    renum.reserve(bvh.nodes.size());
    renum.push_back(bvh.nodes[0]);
    std::vector<std::pair<uint32_t, uint32_t>> stack{{0, 0}};  // (old index, new index)
    while (!stack.empty()) {
        auto [oi, ni] = stack.back(); stack.pop_back();
        const Node& on = bvh.nodes[oi];
        if (on.is_leaf()) continue;
        uint32_t nl = (uint32_t)renum.size();
        renum.push_back(bvh.nodes[on.first]);
        renum.push_back(bvh.nodes[on.first + 1]);
        renum[ni].first = nl;
        stack.push_back({on.first + 1, nl + 1});
        stack.push_back({on.first, nl});
    }
    bvh.nodes = std::move(renum);
    return bvh;
}

/// Reinsertion optimizer over a binary BVH whose siblings are adjacent.
/// Each step detaches a subtree (its sibling takes the parent's slot), searches
/// the remaining tree for the insertion point with the lowest induced area
/// (branch and bound over a priority queue), and inserts it there when that
/// lowers the total area, otherwise back where it was.
class ReinsertionOptimizer {
public:
    struct Config {
        float batch_ratio = 0.05f;     ///< fraction of nodes tried per pass
        uint32_t max_passes = 4;
        double min_relative_gain = 1e-4;
    };

    explicit ReinsertionOptimizer(Bvh& bvh) : bvh_(bvh) {}

    /// Runs passes until one improves the SAH cost by less than the threshold.
    /// Returns the number of subtrees that moved.
    size_t optimize() { return optimize(Config{}); }
    size_t optimize(const Config& cfg) {
        if (bvh_.nodes.size() < 7) return 0;
        parents_ = bvh_.parents();
        size_t applied = 0;
        double cost = bvh_.sah_cost();
        const uint32_t n = (uint32_t)bvh_.nodes.size();
        for (uint32_t pass = 0; pass < cfg.max_passes; ++pass) {
            id_at_.resize(n); slot_of_.resize(n);
            for (uint32_t i = 0; i < n; ++i) { id_at_[i] = i; slot_of_[i] = i; }
            std::vector<uint32_t> cand;
            cand.reserve(n);
            for (uint32_t i = 1; i < n; ++i) if (parents_[i] != 0) cand.push_back(i);
            size_t k = std::min(cand.size(), std::max<size_t>(1, (size_t)(cfg.batch_ratio * (double)n)));
            std::partial_sort(cand.begin(), cand.begin() + (long)k, cand.end(), [&](uint32_t a, uint32_t b) {
                float aa = bvh_.nodes[a].box.half_area(), ab = bvh_.nodes[b].box.half_area();
                return aa > ab || (aa == ab && a < b);
            });
            cand.resize(k);
            for (uint32_t id : cand) {
                uint32_t slot = slot_of_[id];
                if (slot == 0 || parents_[slot] == 0) continue;
                if (reinsert(slot)) ++applied;
            }
            double new_cost = bvh_.sah_cost();
            double gain = cost > 0.0 ? (cost - new_cost) / cost : 0.0;
            cost = new_cost;
            if (gain < cfg.min_relative_gain) break;
        }
        return applied;
    }

private:
    Bvh& bvh_;
    std::vector<uint32_t> parents_;
    std::vector<uint32_t> id_at_;    // slot -> node identity (stable within a pass)
    std::vector<uint32_t> slot_of_;  // identity -> slot

    void refit_from(uint32_t i) {
        while (true) {
            Node& nd = bvh_.nodes[i];
            if (!nd.is_leaf()) nd.box = BBox::merge(bvh_.nodes[nd.first].box, bvh_.nodes[nd.first + 1].box);
            if (i == 0) break;
            i = parents_[i];
        }
    }

    void place(const Node& nd, uint32_t id, uint32_t slot) {
        bvh_.nodes[slot] = nd;
        if (!nd.is_leaf()) { parents_[nd.first] = slot; parents_[nd.first + 1] = slot; }
        id_at_[slot] = id;
        slot_of_[id] = slot;
    }

    /// Insertion point for `box` minimising the induced area (Bittner et al. 2013).
    uint32_t best_position(const BBox& box, double* best_cost_out) const {
        using Item = std::pair<double, uint32_t>;
        std::priority_queue<Item, std::vector<Item>, std::greater<Item>> q;
        const double area = box.half_area();
        double best_cost = std::numeric_limits<double>::infinity();
        uint32_t best = 0;
        q.push({0.0, 0});
        while (!q.empty()) {
            auto [induced, i] = q.top(); q.pop();
            if (induced + area >= best_cost) break;
            const Node& nd = bvh_.nodes[i];
            double merged = BBox::merge(nd.box, box).half_area();
            double c = induced + merged;
            if (c < best_cost) { best_cost = c; best = i; }
            if (!nd.is_leaf()) {
                double ci = c - nd.box.half_area();
                if (ci + area < best_cost) { q.push({ci, nd.first}); q.push({ci, nd.first + 1}); }
            }
        }
        *best_cost_out = best_cost;
        return best;
    }

    bool reinsert(uint32_t slot) {
        const uint32_t p = parents_[slot];
        const uint32_t pair = bvh_.nodes[p].first;
        const uint32_t s = slot == pair ? pair + 1 : pair;
        const uint32_t id_l = id_at_[slot], id_s = id_at_[s], id_p = id_at_[p];
        const Node detached = bvh_.nodes[slot];
        const Node parent_node = bvh_.nodes[p];

        // Area of the path above p before detaching.
        double before = 0.0;
        for (uint32_t i = p; ; i = parents_[i]) { before += bvh_.nodes[i].box.half_area(); if (i == 0) break; }
        // Detach: the sibling takes the parent's slot.
        place(bvh_.nodes[s], id_s, p);
        refit_from(p);
        double after = 0.0;
        for (uint32_t i = p; ; i = parents_[i]) {
            after += i == p ? 0.0 : bvh_.nodes[i].box.half_area();
            if (i == 0) break;
        }
        const double gain = before - after;   // includes the vanished parent

        double cost = 0.0;
        uint32_t target = best_position(detached.box, &cost);
        bool moved = cost < gain * (1.0 - 1e-7);
        if (!moved) target = p;   // back next to the sibling
        // Insert: the node at `target` and the detached subtree become children
        // of `target`'s slot, stored in the freed pair.
        const uint32_t id_t = id_at_[target];
        const Node target_node = bvh_.nodes[target];
        place(target_node, id_t, pair);
        place(detached, id_l, pair + 1);
        Node inner = parent_node;
        inner.first = pair;
        inner.count = 0;
        place(inner, id_p, target);
        parents_[pair] = target;
        parents_[pair + 1] = target;
        refit_from(target);
        return moved;
    }
};

/// Convenience: boxes and centres of an indexed triangle mesh.
inline void triangle_bounds(const float* vertices, const uint32_t* indices, size_t ntri,
                            std::vector<BBox>& boxes, std::vector<float>& centers) {
    boxes.resize(ntri);
    centers.resize(3 * ntri);
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)ntri; ++i) {
        BBox b = BBox::empty();
        for (int k = 0; k < 3; ++k) b.extend(vertices + 3 * (size_t)indices[3 * i + k]);
        boxes[i] = b;
        for (int a = 0; a < 3; ++a) centers[3 * i + a] = (b.lo[a] + b.hi[a]) * 0.5f;
    }
}

}  // namespace sol_b200::bvh
