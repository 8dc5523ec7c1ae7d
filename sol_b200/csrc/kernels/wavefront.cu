// K2-K6: batched wavefront path tracer for many views (cameras, films of uneven
// size and sample count) over one or more scenes in a single launch sequence.
//
// Work items are (view, sample, pixel) triples, taken sample-major in 8x4
// pixel tiles as the megakernel's split schedule takes them; a pool of C path
// slots holds the paths in flight.  Each bounce runs five stages:
//   generate (K2): every slot whose path ended writes the path's colour to its
//                  view's per-sample scratch, claims the next work item and
//                  starts its camera ray (path regeneration, so the pool stays
//                  full until the items run out).
//   extend   (K3): closest-hit traversal of the queued rays.  Rays travel in
//                  the queue by value, so the stage reads its rays and writes
//                  its hits in queue order; hits may be binned by the BSDF kind
//                  of the hit triangle (K6).  Persistent warps fetch rays lane
//                  by lane: when fewer than `refill_below` lanes of a warp are
//                  still traversing, the warp pauses, gives its idle lanes new
//                  rays and resumes.
//   shade    (K5): SoL's per-vertex step (emission MIS, light sample, Russian
//                  roulette, BSDF bounce) per queue position, or per bin; the
//                  next ray goes to the other parity's extend queue and the
//                  light sample's shadow ray to the shadow queue.
//   shadow   (K4): any-hit traversal of the shadow rays; an unoccluded light
//                  sample adds its contribution to the path's colour.  With
//                  the packed-shadow order, shade leaves each shadow ray at
//                  its extend position and a packing kernel queues them in
//                  that order first.
//   advance      : resets the consumed queues and decides whether to loop.
// Queue appends are warp-aggregated (one atomic per distinct target per warp).
// The five stages form the body of a CUDA graph WHILE node whose condition the
// advance kernel sets, so a whole batch renders in one graph launch.
//
// Every path computes what the megakernel computes for it, in the same order
// (the shadow stage runs before the next vertex's emission is added), and the
// sum pass adds each pixel's colours in sample order starting from 0, so films
// are bit-identical to the megakernel's.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "path.cuh"
#include "wavefront.h"

namespace sol_b200 {

namespace {

constexpr uint32_t kIdle = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

/// Appends the calling lanes to one queue: one atomic per warp.
__device__ __forceinline__ uint32_t append(uint32_t* counter) {
    const unsigned mask = __activemask();
    const int leader = __ffs(mask) - 1;
    const unsigned rank = __popc(mask & ((1u << lane_id()) - 1u));
    uint32_t base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    return __shfl_sync(mask, base, leader) + rank;
}

/// Appends the calling lanes to the queue selected by `key`: one atomic per
/// distinct key per warp.
__device__ __forceinline__ uint32_t append_keyed(uint32_t* counters, int key) {
    const unsigned mask = __match_any_sync(__activemask(), key);
    const int leader = __ffs(mask) - 1;
    const unsigned rank = __popc(mask & ((1u << lane_id()) - 1u));
    uint32_t base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(&counters[key], (uint32_t)__popc(mask));
    return __shfl_sync(mask, base, leader) + rank;
}

/// Sum over the whole warp; every lane of the warp must call it.
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
    __syncwarp();
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ uint32_t find_view(const WfView* views, uint32_t n, uint32_t item) {
    uint32_t lo = 0, hi = n;   // last view with item_begin <= item
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (views[mid].item_begin <= item) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ DCamera view_camera(const WfView& v) {
    DCamera c;
    for (int k = 0; k < 3; ++k) { c.eye[k] = v.eye[k]; c.dir[k] = v.dir[k]; c.right[k] = v.right[k]; c.up[k] = v.up[k]; }
    return c;
}

__device__ __forceinline__ float tag_bits(uint32_t slot, uint32_t scene) {
    return __uint_as_float(slot | (scene << kWfSlotBits));
}

__global__ void __launch_bounds__(256) wf_init(const WfParams* __restrict__ Pp) {
    const WfParams& P = *Pp;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.capacity; i += gridDim.x * blockDim.x) {
        P.q_ended[0][i] = i;
        P.item[i] = make_uint2(kIdle, 0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        WfCounters* c = P.ctr;
        c->ended[0] = P.capacity;
        c->ended[1] = 0;
        c->extend[0] = c->extend[1] = 0;
        for (int b = 0; b < kWfBins; ++b) c->bins[b] = 0;
        c->shadow = 0;
        c->fetch_extend = c->fetch_shadow = 0;
        c->next_item = 0;
        c->iter = 0;
        c->more = 1;
        if (!P.keep_counts) c->paths = c->rays = c->shadow_rays = 0;
        c->error = 0;
    }
}

/// Ends the path of `slot` (colour `col` to the scratch of its work item) and
/// starts the slot's next path: claims work items until one is a pixel, writes
/// the new path's state and appends its camera ray to extend queue `qp`.  A
/// slot that finds no item left goes idle.  Returns the paths started (0 or
/// more: paths of length 0 end at once with a black colour).
__device__ __forceinline__ uint32_t restart_slot(const WfParams& P, const WfView* views, uint32_t slot, float4 col,
                                                 uint32_t qp) {
    WfCounters* ctr = P.ctr;
    const uint32_t total = P.total_items;
    uint2 it = P.item[slot];
    uint32_t claims = 0, paths = 0;
    while (true) {
        if (it.x != kIdle) {
            // path_tracer.cpp:19 -- the pixel's sum is formed by the sum pass
            reinterpret_cast<float4*>(views[it.x].scratch)[it.y] = make_float4(col.x, col.y, col.z, 0.0f);
            it.x = kIdle;
        }
        if (++claims > total + 2u) { atomicOr(&ctr->error, kFaultClaimLoop); break; }
        const uint32_t item = append(&ctr->next_item);
        if (item >= total) break;
        const uint32_t vi = find_view(views, P.num_views, item);
        const WfView& v = views[vi];
        const uint32_t per_sample = v.tiles_x * ((v.height + 3u) / 4u) * 32u;
        const uint32_t local = item - v.item_begin;
        const uint32_t k = local / per_sample;
        const uint32_t in_sample = local - k * per_sample;
        const uint32_t tile = in_sample >> 5, l = in_sample & 31u;
        const uint32_t x = (tile % v.tiles_x) * 8u + (l & 7u);
        const uint32_t y = (tile / v.tiles_x) * 4u + (l >> 3);
        if (x >= v.width || y >= v.height) continue;   // padding of a partial tile: no pixel
        PathState ps;
        start_path(ps, view_camera(v), v.sample_index + k, x, y, v.width, v.height);
        ++paths;
        it = make_uint2(vi, local);
        col = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (P.cfg.max_path_len == 0) continue;   // empty path: black, written above
        P.thru[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        P.color[slot] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0u));
        P.rng[slot] = ps.rng.state;
        const uint32_t q = append(&ctr->extend[qp]);
        P.ray_o[qp][q] = make_float4(ps.org.x, ps.org.y, ps.org.z, ps.tmin);
        P.ray_d[qp][q] = make_float4(ps.dir.x, ps.dir.y, ps.dir.z, tag_bits(slot, v.scene));
        break;
    }
    P.item[slot] = it;
    return paths;
}

/// K2: the slots on the ended list (all slots at the start; later, the paths
/// that ended after their last shadow ray, and with SOL_WF_SHADE_RESTART off
/// every ended path) restart: colour out, next work item in.
__global__ void __launch_bounds__(256) wf_generate(const WfParams* __restrict__ Pp) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t p = ctr->iter & 1u;
    const uint32_t n = ctr->ended[p];
    unsigned long long paths = 0;
#if SOL_WF_GEN_SMEM_VIEWS
    // The view table in shared memory when it is small: the claim loop's
    // binary search and the view fields then cost no global round trips.
    __shared__ uint4 view_smem[kGenSmemViews * sizeof(WfView) / sizeof(uint4)];
    const WfView* views = P.views;
    if (P.num_views <= kGenSmemViews) {
        const uint4* src = reinterpret_cast<const uint4*>(P.views);
        const uint32_t words = P.num_views * (uint32_t)(sizeof(WfView) / sizeof(uint4));
        for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) view_smem[w] = src[w];
        views = reinterpret_cast<const WfView*>(view_smem);
    }
    __syncthreads();
#else
    const WfView* views = P.views;
#endif
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        if (i >= n) continue;
        const uint32_t slot = P.q_ended[p][i];
        paths += restart_slot(P, views, slot, P.color[slot], p);
    }
    paths = warp_sum(paths);
    if (lane_id() == 0 && paths) atomicAdd(&ctr->paths, paths);
}

/// The wavefront's sum pass: one thread per pixel of the views laid end to end
/// from WfView::sum_begin adds the pixel's path colours (item-ordered float4
/// scratch) in sample order to its running sum -- 0 for a view's first chunk
/// of samples -- and the last chunk adds the sum into the film, so each
/// channel sees the additions of SoL's per-pixel loop (path_tracer.cpp:15-21).
__global__ void __launch_bounds__(256)
sum_items_views(const WfView* __restrict__ views, uint32_t num_views, uint64_t total) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total; g += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = num_views;
        while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (views[mid].sum_begin <= g) lo = mid; else hi = mid; }
        const WfView& V = views[lo];
        const uint32_t px = (uint32_t)(g - V.sum_begin);
        const uint32_t x = px % V.width, y = px / V.width;
        const size_t plane = (size_t)V.width * V.height;
        const uint32_t per_sample = V.tiles_x * ((V.height + 3u) / 4u) * 32u;
        const uint32_t at = ((y >> 2) * V.tiles_x + (x >> 3)) * 32u + (y & 3u) * 8u + (x & 7u);
        const float4* __restrict__ c = reinterpret_cast<const float4*>(V.scratch) + at;
        float r = 0.0f, gg = 0.0f, b = 0.0f;
        if (!V.first_chunk) { r = V.running[px]; gg = V.running[px + plane]; b = V.running[px + 2 * plane]; }
        for (uint32_t k = 0; k < V.sample_count; ++k) {
            const float4 v = c[(size_t)k * per_sample];
            r += v.x;
            gg += v.y;
            b += v.z;
        }
        if (V.last_chunk) {
            V.film[px] += r;
            V.film[px + plane] += gg;
            V.film[px + 2 * plane] += b;
        } else {
            V.running[px] = r;
            V.running[px + plane] = gg;
            V.running[px + 2 * plane] = b;
        }
    }
}

/// The traversal stack of a trace-stage lane (see kWfSharedStack).
#if SOL_WF_SHARED_STACK
using WfStack = SharedStackDyn;
__device__ __forceinline__ WfStack make_stack() {
    extern __shared__ int wf_stack_smem[];
    return WfStack{wf_stack_smem + threadIdx.x, (int)blockDim.x, {}};
}
#else
using WfStack = LocalStack;
__device__ __forceinline__ WfStack make_stack() { return WfStack{}; }
#endif

template <bool kAnyHit, class Fetch, class Finish>
__device__ __forceinline__ void trace_queue(const WfSceneTable& scenes, uint32_t n, uint32_t* fetch_counter,
                                            int refill_below, Fetch fetch, Finish finish,
                                            unsigned long long& rays) {
    Traversal<kAnyHit, false, true> tr;
    WfStack stack = make_stack();
    const SceneView* sv = &scenes.v[0];
    uint32_t at = 0;
    bool has = false;
    bool more = true;   // warp-uniform: the queue may still hold entries
    TraversalCounters tc{0u, 0u};
    while (true) {
        __syncwarp();
        if (more) {
            const unsigned want = __ballot_sync(0xffffffffu, !has);
            if (want) {
                const int leader = __ffs(want) - 1;
                uint32_t base = 0;
                if ((int)lane_id() == leader) base = atomicAdd(fetch_counter, (uint32_t)__popc(want));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + (uint32_t)__popc(want) >= n) more = false;
                if (!has) {
                    const uint32_t i = base + __popc(want & ((1u << lane_id()) - 1u));
                    if (i < n) {
                        at = i;
                        sv = &scenes.v[fetch(i, tr, stack)];
                        has = true;
                        ++rays;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, has)) break;
        // Once the queue is drained there is nothing to refill: run to the end.
        if (has && tr.run(sv->nodes, sv->tris, tc, sv->num_nodes, sv->num_tris, sv->max_steps, sv->fault, stack,
                          more ? refill_below : 0)) {
            finish(at, tr);
            has = false;
        }
    }
}

/// K3: closest hit for every queued ray, written in queue order; hits binned by
/// BSDF kind (K6) when the queue is long enough.
__global__ void __launch_bounds__(256, kWfTraceMinBlocks)
wf_extend(const WfParams* __restrict__ Pp, const __grid_constant__ WfSceneTable scenes) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t p = ctr->iter & 1u;
    const uint32_t n = ctr->extend[p];
    const bool sort = n >= P.sort_threshold;
    const float4* __restrict__ ro = P.ray_o[p];
    const float4* __restrict__ rd = P.ray_d[p];
    unsigned long long rays = 0;
    auto fetch = [&](uint32_t i, Traversal<false, false, true>& tr, WfStack& stack) -> uint32_t {
        const float4 o = ro[i], d = rd[i];
        const uint32_t scene = __float_as_uint(d.w) >> kWfSlotBits;
        tr.start(vec3(o.x, o.y, o.z), vec3(d.x, d.y, d.z), o.w, kFloatMax, scenes.v[scene].num_tris > 0, stack);
        return scene;
    };
    auto finish = [&](uint32_t i, const Traversal<false, false, true>& tr) {
        P.hit[i] = make_float4(__int_as_float(tr.hit), tr.tmax, tr.hu, tr.hv);
        if (sort) {
            int kind = kWfBins - 1;
            if (tr.hit >= 0) {
                const SceneView& sv = scenes.v[__float_as_uint(rd[i].w) >> kWfSlotBits];
                const int b = __ldg(&sv.tris[tr.hit].bsdf);
                kind = b < 0 ? kWfBins - 1 : sv.bsdfs[b].kind;
            }
            P.q_bins[(size_t)kind * P.capacity + append_keyed(ctr->bins, kind)] = i;
        }
    };
    trace_queue<false>(scenes, n, &ctr->fetch_extend, P.refill_below, fetch, finish, rays);
    rays = warp_sum(rays);
    if (lane_id() == 0 && rays) atomicAdd(&ctr->rays, rays);
}

/// K5: SoL's per-vertex step for every closest hit (kind by kind when binned).
template <bool kBasic>
__global__ void __launch_bounds__(256, kWfShadeMinBlocks)
wf_shade(const WfParams* __restrict__ Pp, const __grid_constant__ WfSceneTable scenes) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t p = ctr->iter & 1u;
    const uint32_t q = p ^ 1u;
    const uint32_t n = ctr->extend[p];
    const bool sort = n >= P.sort_threshold;
    uint32_t counts[kWfBins];
    for (int b = 0; b < kWfBins; ++b) counts[b] = sort ? ctr->bins[b] : 0u;
    unsigned long long paths = 0;
    const bool packed = P.shadow_packed != 0;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        uint32_t i = idx;
        if (sort) {
            uint32_t j = idx;
            int b = 0;
            while (b < kWfBins - 1 && j >= counts[b]) { j -= counts[b]; ++b; }
            i = P.q_bins[(size_t)b * P.capacity + j];
        }
        const float4 o = P.ray_o[p][i], d = P.ray_d[p][i];
        const float4 h = P.hit[i];
        const uint32_t tag = __float_as_uint(d.w);
        const uint32_t slot = tag & kWfSlotMask;
        const int tri = __float_as_int(h.x);
        if (tri < 0) {   // path_tracer.cpp:43-44: no hit, the path ends
            if (packed) P.alt[1][i].w = -1.0f;   // no shadow ray at this extend position
#if SOL_WF_SHADE_RESTART
            paths += restart_slot(P, P.views, slot, P.color[slot], q);
#else
            P.q_ended[q][append(&ctr->ended[q])] = slot;
#endif
            continue;
        }
        const SceneView& sv = scenes.v[tag >> kWfSlotBits];
        PathState ps;
        const float4 t4 = P.thru[slot], c4 = P.color[slot];
        ps.org = vec3(o.x, o.y, o.z);
        ps.tmin = o.w;
        ps.dir = vec3(d.x, d.y, d.z);
        ps.T = rgb(t4.x, t4.y, t4.z);
        ps.pdf_prev = t4.w;
        ps.color = rgb(c4.x, c4.y, c4.z);
        ps.path_len = __float_as_uint(c4.w);
        ps.rng.state = P.rng[slot];
        VertexOut vo;
        shade_vertex<kBasic>(sv, P.cfg, 1.0f / (float)sv.num_lights, tri, h.y, ps, vo, true, h.z, h.w);
        bool end = vo.end;
        if (!end) {
            ++ps.path_len;
            end = ps.path_len >= P.cfg.max_path_len;
        }
        P.color[slot] = make_float4(ps.color.r, ps.color.g, ps.color.b, __uint_as_float(ps.path_len));
        if (!end) {
            P.thru[slot] = make_float4(ps.T.r, ps.T.g, ps.T.b, ps.pdf_prev);
            P.rng[slot] = ps.rng.state;
            const uint32_t j = append(&ctr->extend[q]);
            P.ray_o[q][j] = make_float4(ps.org.x, ps.org.y, ps.org.z, ps.tmin);
            P.ray_d[q][j] = make_float4(ps.dir.x, ps.dir.y, ps.dir.z, d.w);
        }
        if (packed) {
            // Shadow rays are staged at the extend position and packed in
            // extend order afterwards (wf_shadow_compact); -1 marks no ray.
            P.alt[1][i] = make_float4(vo.sh_dir.x, vo.sh_dir.y, vo.sh_dir.z,
                                      vo.has_shadow ? (end ? 1.0f : 0.0f) : -1.0f);
            if (vo.has_shadow) {
                P.alt[0][i] = make_float4(vo.sh_org.x, vo.sh_org.y, vo.sh_org.z, d.w);
                P.alt[2][i] = make_float4(vo.pending.r, vo.pending.g, vo.pending.b, 0.0f);
            }
        } else if (vo.has_shadow) {
            const uint32_t j = append(&ctr->shadow);
            P.sh_o[j] = make_float4(vo.sh_org.x, vo.sh_org.y, vo.sh_org.z, d.w);
            P.sh_d[j] = make_float4(vo.sh_dir.x, vo.sh_dir.y, vo.sh_dir.z, end ? 1.0f : 0.0f);
            P.sh_c[j] = make_float4(vo.pending.r, vo.pending.g, vo.pending.b, 0.0f);
        }
        if (!vo.has_shadow && end) {
#if SOL_WF_SHADE_RESTART
            paths += restart_slot(P, P.views, slot, make_float4(ps.color.r, ps.color.g, ps.color.b, 0.0f), q);
#else
            P.q_ended[q][append(&ctr->ended[q])] = slot;
#endif
        }
    }
    paths = warp_sum(paths);
    if (lane_id() == 0 && paths) atomicAdd(&ctr->paths, paths);
}

/// K4: shadow rays; the light sample's contribution is added when unoccluded.
__global__ void __launch_bounds__(256, kWfTraceMinBlocks)
wf_shadow(const WfParams* __restrict__ Pp, const __grid_constant__ WfSceneTable scenes) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t q = (ctr->iter & 1u) ^ 1u;
    const uint32_t n = ctr->shadow;
    const float offset = P.cfg.ray_offset;
    unsigned long long rays = 0;
    auto fetch = [&](uint32_t i, Traversal<true, false, true>& tr, WfStack& stack) -> uint32_t {
        const float4 o = P.sh_o[i], d = P.sh_d[i];
        const uint32_t scene = __float_as_uint(o.w) >> kWfSlotBits;
        tr.start(vec3(o.x, o.y, o.z), vec3(d.x, d.y, d.z), offset, 1.0f - offset, scenes.v[scene].num_tris > 0, stack);
        return scene;
    };
    auto finish = [&](uint32_t i, const Traversal<true, false, true>& tr) {
        const uint32_t slot = __float_as_uint(P.sh_o[i].w) & kWfSlotMask;
        if (tr.hit < 0) {
            const float4 c = P.color[slot], a = P.sh_c[i];
            P.color[slot] = make_float4(c.x + a.x, c.y + a.y, c.z + a.z, c.w);
        }
        if (P.sh_d[i].w != 0.0f) P.q_ended[q][append(&ctr->ended[q])] = slot;
    };
    trace_queue<true>(scenes, n, &ctr->fetch_shadow, P.refill_below, fetch, finish, rays);
    rays = warp_sum(rays);
    if (lane_id() == 0 && rays) { atomicAdd(&ctr->rays, rays); atomicAdd(&ctr->shadow_rays, rays); }
}

/// Spreads the low 10 bits of x to every third bit.
__device__ __forceinline__ uint32_t spread3(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

/// Sort key of a ray (see kWfSortBits): scene index, direction octant, Morton
/// cell of the origin in the scene's bounds, from the high bits down.
__device__ __forceinline__ uint32_t ray_key(const WfParams& P, float4 o, float4 d, uint32_t scene) {
    const int per = (kWfSortBits - 3 - (int)P.scene_bits) / 3;   // Morton bits per axis
    const float cells = (float)(1u << per);
    const float4 lo = P.scene_box[2 * scene], hi = P.scene_box[2 * scene + 1];
    const float fx = fminf(fmaxf((o.x - lo.x) / fmaxf(hi.x - lo.x, 1e-20f), 0.0f), 0.999999f);
    const float fy = fminf(fmaxf((o.y - lo.y) / fmaxf(hi.y - lo.y, 1e-20f), 0.0f), 0.999999f);
    const float fz = fminf(fmaxf((o.z - lo.z) / fmaxf(hi.z - lo.z, 1e-20f), 0.0f), 0.999999f);
    // NaN origins (none arise; they would compare false above) land in cell 0.
    const uint32_t ix = fx == fx ? (uint32_t)(fx * cells) : 0u;
    const uint32_t iy = fy == fy ? (uint32_t)(fy * cells) : 0u;
    const uint32_t iz = fz == fz ? (uint32_t)(fz * cells) : 0u;
    const uint32_t morton = spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2);
    const uint32_t octant = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
    const uint32_t key = (scene << (kWfSortBits - P.scene_bits)) | (octant << (3 * per)) | morton;
    return key & (kWfSortBins - 1u);
}

/// Packed shadow queue (SOL_GPU_RAY_ORDER_PACKED_SHADOWS): the shade stage leaves each
/// shadow ray at its extend position in the spare arrays; this kernel packs
/// them into the shadow queue keeping their order inside each block's 1024
/// positions (a block scan, then one atomic per block for its place), so that
/// neighbouring lanes trace shadow rays of neighbouring pixels even when the
/// shading ran material by material.
__global__ void __launch_bounds__(1024) wf_shadow_compact(const WfParams* __restrict__ Pp) {
    __shared__ uint32_t warp_counts[32];
    __shared__ uint32_t block_base;
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t n = ctr->extend[ctr->iter & 1u];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        float4 d = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        if (i < n) d = P.alt[1][i];
        const bool valid = d.w >= 0.0f;
        const unsigned ballot = __ballot_sync(0xffffffffu, valid);
        if (lane == 0) warp_counts[warp] = __popc(ballot);
        __syncthreads();
        if (warp == 0) {
            const uint32_t c = lane < (blockDim.x >> 5) ? warp_counts[lane] : 0u;
            uint32_t incl = c;
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
                if ((int)lane >= off) incl += v;
            }
            warp_counts[lane] = incl - c;                     // exclusive prefix per warp
            const uint32_t block_total = __shfl_sync(0xffffffffu, incl, 31);
            if (lane == 0) block_base = block_total ? atomicAdd(&ctr->shadow, block_total) : 0u;
        }
        __syncthreads();
        if (valid) {
            const uint32_t at = block_base + warp_counts[warp] + __popc(ballot & ((1u << lane) - 1u));
            P.sh_o[at] = P.alt[0][i];
            P.sh_d[at] = d;
            P.sh_c[at] = P.alt[2][i];
        }
        __syncthreads();
    }
}

/// Reordering, step 1: the key of every queued ray and the key histogram
/// (per block in shared memory, then added to P.sort_bins).  `shadow`: the
/// shadow queue (tag in the origin's w), else the extend queue of this
/// iteration's parity (tag in the direction's w).
__global__ void __launch_bounds__(1024) wf_sort_hist(const WfParams* __restrict__ Pp, int shadow) {
    extern __shared__ uint32_t hist[];
    const WfParams& P = *Pp;
    const uint32_t p = P.ctr->iter & 1u;
    const uint32_t n = shadow ? P.ctr->shadow : P.ctr->extend[p];
    const float4* __restrict__ so = shadow ? P.sh_o : P.ray_o[p];
    const float4* __restrict__ sd = shadow ? P.sh_d : P.ray_d[p];
    for (uint32_t b = threadIdx.x; b < kWfSortBins; b += blockDim.x) hist[b] = 0u;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 o = so[i], d = sd[i];
        const uint32_t tag = __float_as_uint(shadow ? o.w : d.w);
        const uint32_t key = ray_key(P, o, d, tag >> kWfSlotBits);
        P.sort_key[i] = key;
        atomicAdd(&hist[key], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < kWfSortBins; b += blockDim.x)
        if (hist[b]) atomicAdd(&P.sort_bins[b], hist[b]);
}

/// Reordering, step 2 (one block of 1024 threads): exclusive prefix sums of
/// the histogram into the bins' offsets; the counts are cleared for the next use.
__global__ void __launch_bounds__(1024) wf_sort_scan(const WfParams* __restrict__ Pp) {
    __shared__ uint32_t part[1024];
    const WfParams& P = *Pp;
    constexpr uint32_t per = kWfSortBins / 1024;
    const uint32_t t = threadIdx.x;
    uint32_t local[per];
    uint32_t sum = 0;
    for (uint32_t k = 0; k < per; ++k) {
        local[k] = P.sort_bins[t * per + k];
        sum += local[k];
    }
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {   // inclusive scan of the per-thread sums
        const uint32_t v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t at = part[t] - sum;
    for (uint32_t k = 0; k < per; ++k) {
        P.sort_bins[kWfSortBins + t * per + k] = at;
        P.sort_bins[t * per + k] = 0u;
        at += local[k];
    }
}

/// Reordering, step 3: every ray moves to its bin's next place in the spare
/// arrays (the order inside a bin is that of the atomics; results do not
/// depend on it, only on each ray).
__global__ void __launch_bounds__(256) wf_sort_scatter(const WfParams* __restrict__ Pp, int shadow) {
    const WfParams& P = *Pp;
    const uint32_t p = P.ctr->iter & 1u;
    const uint32_t n = shadow ? P.ctr->shadow : P.ctr->extend[p];
    const float4* __restrict__ so = shadow ? P.sh_o : P.ray_o[p];
    const float4* __restrict__ sd = shadow ? P.sh_d : P.ray_d[p];
    uint32_t* offsets = P.sort_bins + kWfSortBins;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t key = P.sort_key[i];
        const uint32_t at = append_keyed(offsets, (int)key);
        P.alt[0][at] = so[i];
        P.alt[1][at] = sd[i];
        if (shadow) P.alt[2][at] = P.sh_c[i];
    }
}

/// Reordering, step 4 (one thread): the reordered arrays become the queue's,
/// the queue's become the spares.
__global__ void wf_sort_swap(WfParams* __restrict__ P, int shadow) {
    const uint32_t p = P->ctr->iter & 1u;
    float4*& o = shadow ? P->sh_o : P->ray_o[p];
    float4*& d = shadow ? P->sh_d : P->ray_d[p];
    float4* t = o; o = P->alt[0]; P->alt[0] = t;
    t = d; d = P->alt[1]; P->alt[1] = t;
    if (shadow) { t = P->sh_c; P->sh_c = P->alt[2]; P->alt[2] = t; }
}

/// Resets the consumed queues, flips the parity and sets the loop condition.
__global__ void wf_advance(const WfParams* __restrict__ Pp, cudaGraphConditionalHandle handle, int use_handle) {
    const WfParams& P = *Pp;
    WfCounters* c = P.ctr;
    const uint32_t p = c->iter & 1u;
    c->extend[p] = 0;
    c->ended[p] = 0;
    for (int b = 0; b < kWfBins; ++b) c->bins[b] = 0;
    c->shadow = 0;
    c->fetch_extend = c->fetch_shadow = 0;
    c->iter += 1;
    bool more = c->extend[p ^ 1u] + c->ended[p ^ 1u] > 0;
    if (more && c->iter >= P.max_iterations) { c->error |= kFaultPathLoop; more = false; }
    c->more = more ? 1u : 0u;
    if (use_handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

/// Dynamic shared memory of a traversal-stage block of `block` threads.
size_t trace_smem(int block) { return kWfSharedStack ? sizeof(int) * kSharedStackDepth * (size_t)block : 0; }

/// Lets the traversal stages use more than 48 KiB of dynamic shared memory
/// (their stacks at 256 threads per block and kSharedStackDepth above 48), on
/// the current device.
cudaError_t allow_trace_smem() {
    const int bytes = (int)trace_smem(256);
    if (bytes <= 48 * 1024) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(wf_extend, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(wf_shadow, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

}  // namespace

int wavefront_blocks_per_sm(int stage, int block) {
    int n = 0;
    if (allow_trace_smem() != cudaSuccess) return -1;
    cudaError_t e = cudaSuccess;
    switch (stage) {
        case 0: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_generate, block, 0); break;
        case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_extend, block, trace_smem(block)); break;
        case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shade<false>, block, 0); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shadow, block, trace_smem(block)); break;
    }
    return e == cudaSuccess ? n : -1;
}

cudaError_t launch_sum_items_views(const WfView* views, uint32_t num_views, uint64_t total_pixels, cudaStream_t stream) {
    if (total_pixels == 0) return cudaSuccess;
    const int blocks = (int)std::min<uint64_t>((total_pixels + 255) / 256, 8192);
    sum_items_views<<<blocks, 256, 0, stream>>>(views, num_views, total_pixels);
    return cudaGetLastError();
}

cudaError_t launch_wf_init(const WfParams* params, uint32_t capacity, cudaStream_t stream) {
    uint32_t grid = (capacity + 255) / 256;
    grid = grid > 4096 ? 4096 : (grid == 0 ? 1 : grid);
    wf_init<<<grid, 256, 0, stream>>>(params);
    return cudaGetLastError();
}

namespace {

/// The four reordering launches of one queue (see wf_sort_hist).
void launch_sort(WfParams* params, int shadow, int sms, cudaStream_t stream) {
    wf_sort_hist<<<2 * sms, 1024, kWfSortBins * sizeof(uint32_t), stream>>>(params, shadow);
    wf_sort_scan<<<1, 1024, 0, stream>>>(params);
    wf_sort_scatter<<<8 * sms, 256, 0, stream>>>(params, shadow);
    wf_sort_swap<<<1, 1, 0, stream>>>(params, shadow);
}

}  // namespace

cudaError_t allow_sort_smem() {
    return cudaFuncSetAttribute(wf_sort_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kWfSortBins * sizeof(uint32_t)));
}

cudaError_t launch_wf_iteration(WfParams* params, const WfSceneTable& scenes, bool basic, bool ray_sort,
                                bool packed_shadows, const WfLaunch& L, cudaGraphConditionalHandle handle,
                                int use_handle, cudaStream_t stream) {
    const int sms = L.sms > 0 ? L.sms : 1;
    wf_generate<<<L.grid[0], L.block[0], 0, stream>>>(params);
    if (ray_sort) launch_sort(params, 0, sms, stream);
    wf_extend<<<L.grid[1], L.block[1], trace_smem(L.block[1]), stream>>>(params, scenes);
    if (basic) wf_shade<true><<<L.grid[2], L.block[2], 0, stream>>>(params, scenes);
    else wf_shade<false><<<L.grid[2], L.block[2], 0, stream>>>(params, scenes);
    if (packed_shadows) wf_shadow_compact<<<4 * sms, 1024, 0, stream>>>(params);
    if (ray_sort) launch_sort(params, 1, sms, stream);
    wf_shadow<<<L.grid[3], L.block[3], trace_smem(L.block[3]), stream>>>(params, scenes);
    wf_advance<<<1, 1, 0, stream>>>(params, handle, use_handle);
    return cudaGetLastError();
}

}  // namespace sol_b200
