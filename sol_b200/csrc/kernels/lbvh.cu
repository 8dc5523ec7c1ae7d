// GPU BVH construction (linear BVH): an alternative to the host builder for
// large meshes, producing the same device layout (64-byte nodes holding both
// child boxes, triangles in leaf order, leaves of at most 8 triangles).
//
// Method: Karras, "Maximizing Parallelism in the Construction of BVHs, Octrees,
// and k-d Trees" (HPG 2012).  Triangles are sorted by the 63-bit Morton code of
// their centroid in the scene's centroid box (21 bits per axis, so that the
// triangles of small, dense objects still get distinct codes); equal codes are
// ordered by triangle index, which the radix tree uses as the tie-break of its
// prefix lengths.  The n - 1 internal nodes of the binary radix tree over the
// sorted keys are then found independently, node i covering a contiguous range
// of sorted triangles split where the highest differing key bit changes; boxes
// are merged bottom-up, the second child to arrive at a node computing its box
// and its surface-area-heuristic cost (traversal 1, triangle 1, as the host
// builder).  A subtree of at most 8 triangles becomes a leaf when that is
// cheaper than keeping its split; internal nodes inside a leaf, or that became
// one, stay unused in the node array.
//
// The hierarchy differs from the host builder's (no SAH, no reinsertion), so
// closest hits at exactly equal distances may resolve to a different triangle;
// everything else about the render is unchanged.
#include <cuda_runtime.h>

#include <algorithm>

#include <cub/device/device_radix_sort.cuh>

#include "../core/layout.h"
#include "../core/math.h"
#include "lbvh.h"

namespace sol_b200 {

namespace {

constexpr int kLbvhLeafMax = 8;
constexpr float kSahTraversal = 1.0f;   // per node, relative to one triangle test
constexpr float kSahTriangle = 1.0f;
constexpr int kLbvhRounds = 3;          // bottom-up passes, each restructuring the treelets

/// 21 bits -> every third bit of 63.
__device__ __forceinline__ unsigned long long expand_bits21(uint32_t v) {
    unsigned long long x = v & 0x1fffffu;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

/// float -> uint order-preserving key (for min/max reductions with integer atomics).
__device__ __forceinline__ uint32_t float_key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct TriBox {
    float lo[3], hi[3];
};

__device__ __forceinline__ float half_area(const TriBox& b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

__global__ void tri_boxes(const float* __restrict__ v, const uint32_t* __restrict__ idx, uint32_t nt,
                          TriBox* __restrict__ boxes, uint32_t* __restrict__ cbounds) {
    __shared__ uint32_t s_lo[3], s_hi[3];
    if (threadIdx.x < 3) { s_lo[threadIdx.x] = 0xffffffffu; s_hi[threadIdx.x] = 0u; }
    __syncthreads();
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        TriBox b;
        for (int k = 0; k < 3; ++k) { b.lo[k] = kFloatMax; b.hi[k] = -kFloatMax; }
        for (int c = 0; c < 3; ++c) {
            const uint32_t i = idx[3 * t + c];
            for (int k = 0; k < 3; ++k) {
                const float x = v[3 * i + k];
                b.lo[k] = fminf(b.lo[k], x);
                b.hi[k] = fmaxf(b.hi[k], x);
            }
        }
        boxes[t] = b;
        for (int k = 0; k < 3; ++k) {
            const float c = (b.lo[k] + b.hi[k]) * 0.5f;
            atomicMin(&s_lo[k], float_key(c));
            atomicMax(&s_hi[k], float_key(c));
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&cbounds[threadIdx.x], s_lo[threadIdx.x]);
        atomicMax(&cbounds[3 + threadIdx.x], s_hi[threadIdx.x]);
    }
}

__global__ void morton_keys(const TriBox* __restrict__ boxes, uint32_t nt, const uint32_t* __restrict__ cbounds,
                            unsigned long long* __restrict__ keys, uint32_t* __restrict__ order) {
    float lo[3], ext[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = key_float(cbounds[k]);
        const float e = key_float(cbounds[3 + k]) - lo[k];
        ext[k] = e > 0.0f ? e : 1.0f;
    }
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        const TriBox b = boxes[t];
        unsigned long long m = 0;
        for (int k = 0; k < 3; ++k) {
            const float c = ((b.lo[k] + b.hi[k]) * 0.5f - lo[k]) / ext[k];
            const uint32_t q = (uint32_t)fminf(fmaxf(c * 2097152.0f, 0.0f), 2097151.0f);
            m |= expand_bits21(q) << (2 - k);
        }
        keys[t] = m;
        order[t] = t;
    }
}

/// Common prefix length of sorted keys i and j, extended by the positions'
/// common prefix when the keys are equal (every key made unique by its index).
__device__ __forceinline__ int delta(const unsigned long long* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long x = keys[i] ^ keys[j];
    return x ? __clzll(x) : 64 + __clz((uint32_t)(i ^ j));
}

/// Internal node i of the radix tree: its range [first, last] and children.
/// child >= 0: internal node; child < 0: leaf ~sorted_index.
__global__ void radix_tree(const unsigned long long* __restrict__ keys, int n, int* __restrict__ count, int2* __restrict__ child, int* __restrict__ parent_internal,
                           int* __restrict__ parent_leaf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1) > 0 ? 1 : -1;
        const int dmin = delta(keys, n, i, i - d);
        int lmax = 2;
        while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;   // at most ~log2(n) doublings
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta(keys, n, i, j);
        int s = 0;
        int div = 2;
        for (int t = (l + div - 1) / div; ; ) {
            if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
            div *= 2;
            t = (l + div - 1) / div;
        }
        const int gamma = i + s * d + min(d, 0);
        const int first = min(i, j), last = max(i, j);
        count[i] = last - first + 1;
        const int left = first == gamma ? ~gamma : gamma;
        const int right = last == gamma + 1 ? ~(gamma + 1) : gamma + 1;
        child[i] = make_int2(left, right);
        if (left >= 0) parent_internal[left] = i; else parent_leaf[~left] = i;
        if (right >= 0) parent_internal[right] = i; else parent_leaf[~right] = i;
    }
}

/// A value written by another block: read from L2 (not a possibly stale L1 line).
__device__ __forceinline__ TriBox load_box_cg(const TriBox* p) {
    const float* f = reinterpret_cast<const float*>(p);
    TriBox b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = __ldcg(f + k); b.hi[k] = __ldcg(f + 3 + k); }
    return b;
}

__device__ __forceinline__ TriBox box_union(const TriBox& a, const TriBox& b) {
    TriBox m;
    for (int k = 0; k < 3; ++k) { m.lo[k] = fminf(a.lo[k], b.lo[k]); m.hi[k] = fmaxf(a.hi[k], b.hi[k]); }
    return m;
}

/// The radix tree while it is optimised: child references (>= 0 internal node,
/// < 0 ~sorted triangle), parents, and per internal node its box, triangle
/// count, SAH cost (not normalised: area x expected cost) and whether it is a
/// leaf.  Costs: a triangle kSahTriangle x area; a node min(leaf: count x
/// kSahTriangle x area when count <= 8 and not the root, split: kSahTraversal
/// x area + the children's costs).
struct Tree {
    const uint32_t* order;
    const TriBox* tri_boxes;
    int2* child;
    int* parent_internal;
    int* parent_leaf;
    TriBox* box;
    int* count;
    float* cost;
    int* leaf;

    /// Box, cost and triangle count of a reference (nodes read through L2).
    __device__ __forceinline__ void info(int ref, TriBox& b, float& c, int& n) const {
        if (ref >= 0) {
            b = load_box_cg(box + ref);
            c = __ldcg(cost + ref);
            n = __ldcg(count + ref);
        } else {
            b = tri_boxes[order[~ref]];
            c = kSahTriangle * half_area(b);
            n = 1;
        }
    }
    __device__ __forceinline__ void set_parent(int ref, int parent) const {
        if (ref >= 0) parent_internal[ref] = parent;
        else parent_leaf[~ref] = parent;
    }
};

constexpr int kTreeletLeaves = 7;                    // leaves of a restructured treelet
constexpr int kTreeletSets = 1 << kTreeletLeaves;
constexpr int kTreeletMinCount = kLbvhLeafMax + 1;  // treelet roots: nodes that cannot be leaves

/// Treelet restructuring (Karras and Aila, "Fast Parallel Construction of
/// High-Quality Bounding Volume Hierarchies", HPG 2013), one thread per
/// treelet: the treelet of `root` grows from its two children by opening the
/// internal leaf of largest area until it has 7 leaves; the cost of every
/// subset of the leaves is the best of making it a leaf (at most 8 triangles)
/// and of its best split into two subsets; if the best tree over all leaves is
/// cheaper than the current one, the treelet's internal nodes are rewired into
/// it (root stays the treelet's root).  All nodes below `root` are final.
__device__ void restructure(const Tree& t, int root) {
    int leaf[kTreeletLeaves], inner[kTreeletLeaves - 1];
    TriBox lb[kTreeletLeaves];
    float lc[kTreeletLeaves];
    int ln[kTreeletLeaves];
    const int2 c0 = __ldcg(&t.child[root]);
    leaf[0] = c0.x;
    leaf[1] = c0.y;
    t.info(leaf[0], lb[0], lc[0], ln[0]);
    t.info(leaf[1], lb[1], lc[1], ln[1]);
    int nl = 2, ni = 1;
    inner[0] = root;
    while (nl < kTreeletLeaves) {
        int best = -1;
        float best_area = -1.0f;
        for (int k = 0; k < nl; ++k)
            if (leaf[k] >= 0 && half_area(lb[k]) > best_area) { best_area = half_area(lb[k]); best = k; }
        if (best < 0) break;
        const int node = leaf[best];
        const int2 cc = __ldcg(&t.child[node]);
        inner[ni++] = node;
        leaf[best] = cc.x;
        t.info(cc.x, lb[best], lc[best], ln[best]);
        leaf[nl] = cc.y;
        t.info(cc.y, lb[nl], lc[nl], ln[nl]);
        ++nl;
    }
    if (nl < 3) return;

    const int full = (1 << nl) - 1;
    float cost[kTreeletSets];
    int cnt[kTreeletSets];
    unsigned char part[kTreeletSets];   // low 7 bits: the left subset; bit 7: a leaf
    for (int s = 1; s <= full; ++s) {
        if ((s & (s - 1)) == 0) {
            const int k = __ffs(s) - 1;
            cost[s] = lc[k];
            cnt[s] = ln[k];
            part[s] = 0;
            continue;
        }
        TriBox b;
        int n = 0;
        bool first = true;
        for (int k = 0; k < nl; ++k) {
            if (!(s >> k & 1)) continue;
            b = first ? lb[k] : box_union(b, lb[k]);
            first = false;
            n += ln[k];
        }
        const float a = half_area(b);
        const int low = s & -s;
        float best = 3.0e38f;
        int bp = low;
        for (int p = (s - 1) & s; p != 0; p = (p - 1) & s) {
            if (!(p & low)) continue;
            const float c = cost[p] + cost[s ^ p];
            if (c < best) { best = c; bp = p; }
        }
        const float split = kSahTraversal * a + best;
        const float as_leaf = kSahTriangle * (float)n * a;
        const bool make_leaf = n <= kLbvhLeafMax && !(s == full && root == 0) && as_leaf <= split;
        cnt[s] = n;
        cost[s] = make_leaf ? as_leaf : split;
        part[s] = (unsigned char)(bp | (make_leaf ? 0x80 : 0));
    }
    if (!(cost[full] < __ldcg(&t.cost[root]) * 0.999999f)) return;

    // Rewire: internal nodes of the new tree taken from `inner` in creation order.
    int set_of[kTreeletLeaves - 1], node_of[kTreeletLeaves - 1];
    int made = 0, next = 1, top = 0;
    int st_set[kTreeletLeaves - 1], st_node[kTreeletLeaves - 1];
    st_set[top] = full;
    st_node[top++] = root;
    while (top > 0) {
        --top;
        const int s = st_set[top], id = st_node[top];
        set_of[made] = s;
        node_of[made++] = id;
        const int l = part[s] & 0x7f, r = s ^ l;
        int ref[2];
        const int side[2] = {l, r};
        for (int k = 0; k < 2; ++k) {
            if ((side[k] & (side[k] - 1)) == 0) {
                ref[k] = leaf[__ffs(side[k]) - 1];
            } else {
                ref[k] = inner[next++];
                st_set[top] = side[k];
                st_node[top++] = ref[k];
            }
            t.set_parent(ref[k], id);
        }
        t.child[id] = make_int2(ref[0], ref[1]);
    }
    for (int m = 0; m < made; ++m) {
        const int s = set_of[m], id = node_of[m];
        TriBox b;
        bool first = true;
        for (int k = 0; k < nl; ++k) {
            if (!(s >> k & 1)) continue;
            b = first ? lb[k] : box_union(b, lb[k]);
            first = false;
        }
        t.box[id] = b;
        t.count[id] = cnt[s];
        t.cost[id] = cost[s];
        t.leaf[id] = (part[s] & 0x80) ? 1 : 0;
    }
}

/// One bottom-up pass: each triangle walks up; the second arrival at a node
/// merges its children's boxes, counts and costs, decides whether the node is a
/// leaf, and restructures the treelet the node roots.  A walk longer than any
/// tree of n leaves sets `*fail` (the build is then rejected).
__global__ void bottom_up(Tree t, int n, unsigned int* __restrict__ arrived, unsigned int* __restrict__ fail) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        int node = t.parent_leaf[j];
        int guard = 0;
        for (; node >= 0 && guard < n; ++guard) {
            __threadfence();
            if (atomicAdd(&arrived[node], 1u) == 0u) { node = -1; break; }   // the sibling is not done yet
            const int2 c = __ldcg(&t.child[node]);
            TriBox a, b;
            float ca, cb;
            int na, nb;
            t.info(c.x, a, ca, na);
            t.info(c.y, b, cb, nb);
            const TriBox m = box_union(a, b);
            const float area = half_area(m);
            const int count = na + nb;
            const float split = kSahTraversal * area + ca + cb;
            const float as_leaf = kSahTriangle * (float)count * area;
            const bool leaf = node != 0 && count <= kLbvhLeafMax && as_leaf <= split;
            t.box[node] = m;
            t.count[node] = count;
            t.cost[node] = leaf ? as_leaf : split;
            t.leaf[node] = leaf ? 1 : 0;
            if (count >= kTreeletMinCount) restructure(t, node);
            __threadfence();
            node = node == 0 ? -1 : __ldcg(&t.parent_internal[node]);
        }
        if (node >= 0) atomicOr(fail, 1u);
    }
}

/// Whether internal node i is emitted: the root, or a node that is not a leaf
/// and has no ancestor that is (ancestors covering more than 8 triangles never
/// are, so the walk stops there).
__device__ __forceinline__ bool emitted(int i, const int* __restrict__ count, const int* __restrict__ leaf,
                                        const int* __restrict__ parent_internal) {
    if (i == 0) return true;
    if (leaf[i]) return false;
    for (int p = parent_internal[i], guard = 0; p != 0 && guard < 16; p = parent_internal[p], ++guard) {
        if (leaf[p]) return false;
        if (count[p] > kLbvhLeafMax) break;
    }
    return true;
}

/// Position of the first triangle below a reference in the depth-first leaf
/// order (left subtree first): the counts of the left siblings on the way up.
__device__ __forceinline__ int first_position(int ref, const int2* __restrict__ child, const int* __restrict__ count,
                                              const int* __restrict__ parent_internal,
                                              const int* __restrict__ parent_leaf, int n) {
    int pos = 0;
    int node = ref;
    int p = ref >= 0 ? (ref == 0 ? -1 : parent_internal[ref]) : parent_leaf[~ref];
    for (int guard = 0; p >= 0 && guard < n; ++guard) {
        const int2 c = child[p];
        if (c.y == node) pos += c.x >= 0 ? count[c.x] : 1;
        node = p;
        p = p == 0 ? -1 : parent_internal[p];
    }
    return pos;
}

__device__ __forceinline__ int32_t leaf_ref_(uint32_t first, uint32_t count) {
    return (int32_t)~((first << 3) | (count - 1u));
}

__device__ __forceinline__ void put_box(DNode& g, int c, const TriBox& b) {
    float* xy = c == 0 ? g.b0 : g.b1;
    xy[0] = b.lo[0]; xy[1] = b.hi[0]; xy[2] = b.lo[1]; xy[3] = b.hi[1];
    g.b2[2 * c + 0] = b.lo[2]; g.b2[2 * c + 1] = b.hi[2];
}

/// Device nodes: every emitted internal node; a child that is a leaf is
/// referenced by its triangles' depth-first positions (at most 8).
__global__ void emit_nodes(Tree t, int n, const int* __restrict__ tri_pos, DNode* __restrict__ nodes) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        if (!emitted(i, t.count, t.leaf, t.parent_internal)) continue;
        const int2 c = t.child[i];
        DNode g{};
        for (int side = 0; side < 2; ++side) {
            const int ch = side == 0 ? c.x : c.y;
            if (ch < 0) {
                put_box(g, side, t.tri_boxes[t.order[~ch]]);
                g.ref[side] = leaf_ref_((uint32_t)tri_pos[~ch], 1);
            } else {
                put_box(g, side, t.box[ch]);
                g.ref[side] = t.leaf[ch] ? leaf_ref_((uint32_t)first_position(ch, t.child, t.count, t.parent_internal,
                                                                             t.parent_leaf, n),
                                                     (uint32_t)t.count[ch])
                                         : ch;
            }
        }
        nodes[i] = g;
    }
}

/// Depth-first position of every sorted triangle.
__global__ void tri_positions(Tree t, int n, int* __restrict__ tri_pos) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        tri_pos[j] = first_position(~j, t.child, t.count, t.parent_internal, t.parent_leaf, n);
}

/// Depth of the emitted hierarchy (for the traversal stack bound): every
/// emitted node counts its emitted ancestors.
__global__ void node_depth(Tree t, int n, unsigned int* __restrict__ max_depth) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        if (!emitted(i, t.count, t.leaf, t.parent_internal)) continue;
        unsigned int depth = 1;
        for (int node = i; node != 0 && depth < 1024u; node = t.parent_internal[node]) ++depth;
        atomicMax(max_depth, depth + 1u);   // + the leaf level
    }
}

/// Triangles and shading records at their depth-first positions.
__global__ void gather_tris(const uint32_t* __restrict__ order, const int* __restrict__ tri_pos, uint32_t nt,
                            const float* __restrict__ v, const float* __restrict__ nrm, const float* __restrict__ uv,
                            const uint32_t* __restrict__ idx, const int32_t* __restrict__ tri_bsdf,
                            const int32_t* __restrict__ tri_light, DTri* __restrict__ tris,
                            DTriShade* __restrict__ shade) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nt; j += gridDim.x * blockDim.x) {
        const uint32_t p = order[j];
        const uint32_t dst = (uint32_t)tri_pos[j];
        const uint32_t i0 = idx[3 * p], i1 = idx[3 * p + 1], i2 = idx[3 * p + 2];
        DTri t;
        for (int k = 0; k < 3; ++k) { t.v0[k] = v[3 * i0 + k]; t.v1[k] = v[3 * i1 + k]; t.v2[k] = v[3 * i2 + k]; }
        t.prim = p;
        t.bsdf = tri_bsdf[p];
        t.light = tri_light[p];
        tris[dst] = t;
        DTriShade s;
        for (int k = 0; k < 3; ++k) { s.n0[k] = nrm[3 * i0 + k]; s.n1[k] = nrm[3 * i1 + k]; s.n2[k] = nrm[3 * i2 + k]; }
        s.uv0x = uv[2 * i0]; s.uv0y = uv[2 * i0 + 1];
        s.uv1x = uv[2 * i1]; s.uv1y = uv[2 * i1 + 1];
        s.uv2x = uv[2 * i2]; s.uv2y = uv[2 * i2 + 1];
        s.bsdf = t.bsdf;
        s.light = t.light;
        const Vec3 fn = triangle_normal(vec3(t.v0[0], t.v0[1], t.v0[2]), vec3(t.v1[0], t.v1[1], t.v1[2]),
                                        vec3(t.v2[0], t.v2[1], t.v2[2]));
        s.fn[0] = fn.x; s.fn[1] = fn.y; s.fn[2] = fn.z;
        shade[dst] = s;
    }
}

template <typename T>
cudaError_t alloc(T** p, size_t n) { return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (n ? n : 1)); }

}  // namespace

cudaError_t build_lbvh(const float* vertices, const uint32_t* indices, const float* normals, const float* uvs,
                       const int32_t* tri_bsdf, const int32_t* tri_light, uint32_t num_triangles,
                       cudaStream_t stream, LbvhResult* out) {
    const int n = (int)num_triangles;
    *out = LbvhResult{};
    if (n < 2) return cudaErrorInvalidValue;   // the caller uses the host builder for tiny meshes
    TriBox* boxes = nullptr;
    TriBox* node_boxes = nullptr;
    unsigned long long *keys = nullptr, *keys_sorted = nullptr;
    uint32_t *order = nullptr, *order_sorted = nullptr;
    float* node_cost = nullptr;
    int *count = nullptr, *leaf = nullptr, *tri_pos = nullptr;
    uint32_t* cbounds = nullptr;
    int2* child = nullptr;
    int *parent_internal = nullptr, *parent_leaf = nullptr;
    unsigned int *arrived = nullptr, *depth = nullptr, *fail = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    cudaError_t e = alloc(&boxes, n);
    if (e == cudaSuccess) e = alloc(&node_boxes, n);
    if (e == cudaSuccess) e = alloc(&keys, n);
    if (e == cudaSuccess) e = alloc(&keys_sorted, n);
    if (e == cudaSuccess) e = alloc(&order, n);
    if (e == cudaSuccess) e = alloc(&order_sorted, n);
    if (e == cudaSuccess) e = alloc(&node_cost, n);
    if (e == cudaSuccess) e = alloc(&count, n);
    if (e == cudaSuccess) e = alloc(&leaf, n);
    if (e == cudaSuccess) e = alloc(&tri_pos, n);
    if (e == cudaSuccess) e = alloc(&cbounds, 6);
    if (e == cudaSuccess) e = alloc(&child, n);
    if (e == cudaSuccess) e = alloc(&parent_internal, n);
    if (e == cudaSuccess) e = alloc(&parent_leaf, n);
    if (e == cudaSuccess) e = alloc(&arrived, n);
    if (e == cudaSuccess) e = alloc(&depth, 1);
    if (e == cudaSuccess) e = alloc(&fail, 1);
    if (e == cudaSuccess) e = alloc(&out->nodes, n - 1);
    if (e == cudaSuccess) e = alloc(&out->tris, n);
    if (e == cudaSuccess) e = alloc(&out->shade, n);
    const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    if (e == cudaSuccess) e = cudaMemcpyAsync(cbounds, init, sizeof(init), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(leaf, 0, sizeof(int) * n, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(depth, 0, sizeof(unsigned int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(fail, 0, sizeof(unsigned int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(out->nodes, 0, sizeof(DNode) * (n - 1), stream);
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 8192);
    if (e == cudaSuccess) { tri_boxes<<<grid, 256, 0, stream>>>(vertices, indices, num_triangles, boxes, cbounds); e = cudaGetLastError(); }
    if (e == cudaSuccess) { morton_keys<<<grid, 256, 0, stream>>>(boxes, num_triangles, cbounds, keys, order); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys_sorted, order, order_sorted, n, 0, 63, stream);
    if (e == cudaSuccess) e = cudaMalloc(&temp, temp_bytes ? temp_bytes : 1);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_sorted, order, order_sorted, n, 0, 63, stream);
    if (e == cudaSuccess) { radix_tree<<<grid, 256, 0, stream>>>(keys_sorted, n, count, child, parent_internal, parent_leaf); e = cudaGetLastError(); }
    Tree t{order_sorted, boxes, child, parent_internal, parent_leaf, node_boxes, count, node_cost, leaf};
    for (int round = 0; round < kLbvhRounds && e == cudaSuccess; ++round) {
        e = cudaMemsetAsync(arrived, 0, sizeof(unsigned int) * n, stream);
        if (e == cudaSuccess) { bottom_up<<<grid, 256, 0, stream>>>(t, n, arrived, fail); e = cudaGetLastError(); }
    }
    if (e == cudaSuccess) { tri_positions<<<grid, 256, 0, stream>>>(t, n, tri_pos); e = cudaGetLastError(); }
    if (e == cudaSuccess) { emit_nodes<<<grid, 256, 0, stream>>>(t, n, tri_pos, out->nodes); e = cudaGetLastError(); }
    if (e == cudaSuccess) { node_depth<<<grid, 256, 0, stream>>>(t, n, depth); e = cudaGetLastError(); }
    if (e == cudaSuccess) { gather_tris<<<grid, 256, 0, stream>>>(order_sorted, tri_pos, num_triangles, vertices, normals, uvs, indices, tri_bsdf, tri_light, out->tris, out->shade); e = cudaGetLastError(); }
    unsigned int d = 0, failed = 0;
    float root_cost = 0.0f;
    TriBox root_box{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&d, depth, sizeof(d), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&failed, fail, sizeof(failed), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&root_cost, node_cost, sizeof(float), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&root_box, node_boxes, sizeof(TriBox), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(boxes); cudaFree(node_boxes); cudaFree(keys); cudaFree(keys_sorted); cudaFree(order);
    cudaFree(order_sorted); cudaFree(node_cost); cudaFree(count); cudaFree(leaf); cudaFree(tri_pos); cudaFree(cbounds);
    cudaFree(fail); cudaFree(child); cudaFree(parent_internal); cudaFree(parent_leaf); cudaFree(arrived);
    cudaFree(depth); cudaFree(temp);
    if (e == cudaSuccess && failed) e = cudaErrorUnknown;   // a bottom-up walk did not reach the root
    if (e != cudaSuccess) {
        cudaFree(out->nodes); cudaFree(out->tris); cudaFree(out->shade);
        *out = LbvhResult{};
        return e;
    }
    out->num_nodes = (uint32_t)(n - 1);
    out->depth = d;
    const float dx = root_box.hi[0] - root_box.lo[0], dy = root_box.hi[1] - root_box.lo[1];
    const float dz = root_box.hi[2] - root_box.lo[2];
    const float root_area = dx * dy + dy * dz + dz * dx;
    out->sah_cost = root_area > 0.0f ? root_cost / root_area : 0.0f;
    return cudaSuccess;
}

}  // namespace sol_b200
