// K2-K6: batched wavefront path tracer for many views (cameras, films of uneven
// size and sample count) over one or more scenes in a single launch sequence.
//
// A pool of C path slots lives in device memory (structure of arrays).  Each
// bounce runs five stages over index queues:
//   generate (K2): slots whose path ended add it to their pixel's sum; a pixel
//                  that has run all its samples is written to its view's film
//                  and the slot claims the next pixel of any view; the slot then
//                  starts its pixel's next sample (camera ray).
//   extend   (K3): closest-hit traversal of the queued rays; hits are binned by
//                  the BSDF kind of the hit triangle (K6), misses end the path.
//                  Persistent warps fetch rays lane by lane: when fewer than
//                  `refill_below` lanes of a warp are still traversing, the warp
//                  pauses, gives its idle lanes new rays and resumes.
//   shade    (K5): SoL's per-vertex step (emission MIS, light sample, Russian
//                  roulette, BSDF bounce) over the bins, kind by kind.
//   shadow   (K4): any-hit traversal of the light samples' shadow rays.
//   advance      : resets the consumed queues and decides whether to loop.
// Queue appends are warp-aggregated (one atomic per distinct target per warp).
// The five stages form the body of a CUDA graph WHILE node whose condition the
// advance kernel sets, so a whole batch renders in one graph launch.
//
// A slot runs all samples of its pixel in order, so every pixel's sum is formed
// in SoL's sample order and the films are bit-identical to the megakernel's.
#include <cuda_runtime.h>

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

__device__ __forceinline__ uint32_t claim(uint32_t* counter) { return append(counter); }

/// Sum over the whole warp; every lane of the block must call it (the stage
/// kernels have no early exits, so all lanes reach their final reduction).
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

__device__ __forceinline__ void load_path(const WfParams& P, uint32_t slot, PathState& ps) {
    const float4 o = P.ray_o[slot], d = P.ray_d[slot], t = P.thru[slot], c = P.color[slot];
    ps.org = vec3(o.x, o.y, o.z);
    ps.tmin = o.w;
    ps.dir = vec3(d.x, d.y, d.z);
    ps.pdf_prev = d.w;
    ps.T = rgb(t.x, t.y, t.z);
    ps.path_len = __float_as_uint(t.w);
    ps.color = rgb(c.x, c.y, c.z);
    ps.rng.state = P.rng[slot];
}

__device__ __forceinline__ void store_path(const WfParams& P, uint32_t slot, const PathState& ps) {
    P.ray_o[slot] = make_float4(ps.org.x, ps.org.y, ps.org.z, ps.tmin);
    P.ray_d[slot] = make_float4(ps.dir.x, ps.dir.y, ps.dir.z, ps.pdf_prev);
    P.thru[slot] = make_float4(ps.T.r, ps.T.g, ps.T.b, __uint_as_float(ps.path_len));
    P.color[slot] = make_float4(ps.color.r, ps.color.g, ps.color.b, 0.0f);
    P.rng[slot] = ps.rng.state;
}

__global__ void __launch_bounds__(256) wf_init(const WfParams* __restrict__ Pp) {
    const WfParams& P = *Pp;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.capacity; i += gridDim.x * blockDim.x) {
        P.q_regen[0][i] = i;
        P.pix[i] = make_uint4(kIdle, 0, 0, 0);
        P.color[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        P.sum[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        WfCounters* c = P.ctr;
        c->regen[0] = P.capacity;
        c->regen[1] = 0;
        c->extend[0] = c->extend[1] = 0;
        for (int b = 0; b < kWfBins; ++b) c->bins[b] = 0;
        c->shadow = 0;
        c->fetch_extend = c->fetch_shadow = 0;
        c->next_item = 0;
        c->iter = 0;
        c->paths = c->rays = c->shadow_rays = 0;
        c->error = 0;
    }
}

/// K2: finish ended paths, write finished pixels, claim work, start samples.
__global__ void __launch_bounds__(256) wf_generate(const WfParams* __restrict__ Pp) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t p = ctr->iter & 1u;
    const uint32_t n = ctr->regen[p];
    const uint32_t total = P.total_items;
    unsigned long long paths = 0;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        if (i >= n) continue;
        const uint32_t slot = P.q_regen[p][i];
        uint4 px = P.pix[slot];
        float4 s = P.sum[slot];
        if (px.x != kIdle) {
            const float4 c = P.color[slot];
            s = make_float4(s.x + c.x, s.y + c.y, s.z + c.z, 0.0f);   // path_tracer.cpp:19
            px.w += 1;
        }
        bool started = false;
        uint32_t claims = 0;
        while (!started) {
            if (++claims > total + 2u) { atomicOr(&ctr->error, kFaultClaimLoop); break; }
            if (px.x != kIdle) {
                const WfView& v = P.views[px.x];
                if (px.w < v.sample_count) {
                    PathState ps;
                    start_path(ps, view_camera(v), v.sample_index + px.w, px.y, px.z, v.width, v.height);
                    ++paths;
                    if (P.cfg.max_path_len == 0) { px.w += 1; continue; }   // empty path: black
                    store_path(P, slot, ps);
                    started = true;
                    break;
                }
                // image.h:54-60 accumulate into the view's film
                const size_t plane = (size_t)v.width * v.height;
                const size_t at = (size_t)px.z * v.width + px.y;
                v.film[at] += s.x;
                v.film[at + plane] += s.y;
                v.film[at + 2 * plane] += s.z;
                px.x = kIdle;
            }
            const uint32_t item = claim(&ctr->next_item);
            if (item >= total) break;
            const uint32_t vi = find_view(P.views, P.num_views, item);
            const WfView& v = P.views[vi];
            const uint32_t local = item - v.item_begin;
            const uint32_t tile = local >> 5, l = local & 31u;
            const uint32_t x = (tile % v.tiles_x) * 8u + (l & 7u);
            const uint32_t y = (tile / v.tiles_x) * 4u + (l >> 3);
            if (x < v.width && y < v.height) {
                px = make_uint4(vi, x, y, 0);
                s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
        P.pix[slot] = px;
        P.sum[slot] = s;
        if (started) {
            P.color[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            P.q_extend[p][append(&ctr->extend[p])] = slot;
        }
    }
    paths = warp_sum(paths);
    if (lane_id() == 0 && paths) atomicAdd(&ctr->paths, paths);
}

/// Persistent traversal of a ray queue with dynamic ray fetch: every lane keeps
/// one ray; at the top of each round the warp claims queue entries for its idle
/// lanes with one atomic, then traverses until the ray is done or the warp has
/// fewer than `refill_below` busy lanes.  `fetch(i, tr, stack, slot, sv)` starts
/// queue entry i; `finish(slot, tr)` consumes a finished ray.
template <bool kAnyHit, class Fetch, class Finish>
__device__ __forceinline__ void trace_queue(uint32_t n, uint32_t* fetch_counter, int refill_below, Fetch fetch,
                                            Finish finish, unsigned long long& rays) {
    Traversal<kAnyHit, false, true> tr;
    LocalStack stack;
    const SceneView* sv = nullptr;
    uint32_t slot = 0;
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
                        fetch(i, tr, stack, slot, sv);
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
            finish(slot, tr);
            has = false;
        }
    }
}

/// K3: closest hit for every queued ray; hits binned by BSDF kind (K6), misses end.
__global__ void __launch_bounds__(256, kWfTraceMinBlocks) wf_extend(const WfParams* __restrict__ Pp) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t p = ctr->iter & 1u;
    const uint32_t n = ctr->extend[p];
    const bool sort = n >= P.sort_threshold;
    unsigned long long rays = 0;
    auto fetch = [&](uint32_t i, Traversal<false, false, true>& tr, LocalStack& stack, uint32_t& slot,
                     const SceneView*& sv) {
        slot = P.q_extend[p][i];
        const float4 o = P.ray_o[slot], d = P.ray_d[slot];
        sv = &P.scenes[P.views[P.pix[slot].x].scene];
        tr.start(vec3(o.x, o.y, o.z), vec3(d.x, d.y, d.z), o.w, kFloatMax, sv->num_tris > 0, stack);
    };
    auto finish = [&](uint32_t slot, const Traversal<false, false, true>& tr) {
        if (tr.hit < 0) {
            P.q_regen[p ^ 1u][append(&ctr->regen[p ^ 1u])] = slot;
        } else {
            P.hit[slot] = make_float2(__int_as_float(tr.hit), tr.tmax);
            int kind = kWfBins - 1;
            if (sort) {
                const SceneView& sv = P.scenes[P.views[P.pix[slot].x].scene];
                const int b = __ldg(&sv.tris[tr.hit].bsdf);
                kind = b < 0 ? kWfBins - 1 : sv.bsdfs[b].kind;
            }
            P.q_bins[(size_t)kind * P.capacity + append_keyed(ctr->bins, kind)] = slot;
        }
    };
    trace_queue<false>(n, &ctr->fetch_extend, P.refill_below, fetch, finish, rays);
    rays = warp_sum(rays);
    if (lane_id() == 0 && rays) atomicAdd(&ctr->rays, rays);
}

/// K5: SoL's per-vertex step over the BSDF bins, kind by kind.
__global__ void __launch_bounds__(256) wf_shade(const WfParams* __restrict__ Pp) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t p = ctr->iter & 1u;
    uint32_t counts[kWfBins];
    uint32_t total = 0;
    for (int b = 0; b < kWfBins; ++b) { counts[b] = ctr->bins[b]; total += counts[b]; }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        uint32_t j = i;
        int b = 0;
        while (j >= counts[b]) { j -= counts[b]; ++b; }
        const uint32_t slot = P.q_bins[(size_t)b * P.capacity + j];
        PathState ps;
        load_path(P, slot, ps);
        const float2 h = P.hit[slot];
        const SceneView& sv = P.scenes[P.views[P.pix[slot].x].scene];
        VertexOut vo;
        shade_vertex(sv, P.cfg, 1.0f / (float)sv.num_lights, __float_as_int(h.x), h.y, ps, vo);
        bool end = vo.end;
        if (!end) {
            ++ps.path_len;
            end = ps.path_len >= P.cfg.max_path_len;
        }
        store_path(P, slot, ps);
        if (vo.has_shadow) {
            P.sh_o[slot] = make_float4(vo.sh_org.x, vo.sh_org.y, vo.sh_org.z, 0.0f);
            P.sh_d[slot] = make_float4(vo.sh_dir.x, vo.sh_dir.y, vo.sh_dir.z, 0.0f);
            P.pending[slot] = make_float4(vo.pending.r, vo.pending.g, vo.pending.b, end ? 1.0f : 0.0f);
            P.q_shadow[append(&ctr->shadow)] = slot;
        } else if (end) {
            P.q_regen[p ^ 1u][append(&ctr->regen[p ^ 1u])] = slot;
        } else {
            P.q_extend[p ^ 1u][append(&ctr->extend[p ^ 1u])] = slot;
        }
    }
}

/// K4: shadow rays; the light sample's contribution is added when unoccluded.
__global__ void __launch_bounds__(256, kWfTraceMinBlocks) wf_shadow(const WfParams* __restrict__ Pp) {
    const WfParams& P = *Pp;
    WfCounters* ctr = P.ctr;
    const uint32_t p = ctr->iter & 1u;
    const uint32_t n = ctr->shadow;
    const float offset = P.cfg.ray_offset;
    unsigned long long rays = 0;
    auto fetch = [&](uint32_t i, Traversal<true, false, true>& tr, LocalStack& stack, uint32_t& slot,
                     const SceneView*& sv) {
        slot = P.q_shadow[i];
        const float4 o = P.sh_o[slot], d = P.sh_d[slot];
        sv = &P.scenes[P.views[P.pix[slot].x].scene];
        tr.start(vec3(o.x, o.y, o.z), vec3(d.x, d.y, d.z), offset, 1.0f - offset, sv->num_tris > 0, stack);
    };
    auto finish = [&](uint32_t slot, const Traversal<true, false, true>& tr) {
        const float4 pend = P.pending[slot];
        if (tr.hit < 0) {
            const float4 c = P.color[slot];
            P.color[slot] = make_float4(c.x + pend.x, c.y + pend.y, c.z + pend.z, 0.0f);
        }
        if (pend.w != 0.0f) P.q_regen[p ^ 1u][append(&ctr->regen[p ^ 1u])] = slot;
        else P.q_extend[p ^ 1u][append(&ctr->extend[p ^ 1u])] = slot;
    };
    trace_queue<true>(n, &ctr->fetch_shadow, P.refill_below, fetch, finish, rays);
    rays = warp_sum(rays);
    if (lane_id() == 0 && rays) { atomicAdd(&ctr->rays, rays); atomicAdd(&ctr->shadow_rays, rays); }
}

/// Resets the consumed queues, flips the parity and sets the loop condition.
__global__ void wf_advance(const WfParams* __restrict__ Pp, cudaGraphConditionalHandle handle, int use_handle) {
    const WfParams& P = *Pp;
    WfCounters* c = P.ctr;
    const uint32_t p = c->iter & 1u;
    c->extend[p] = 0;
    c->regen[p] = 0;
    for (int b = 0; b < kWfBins; ++b) c->bins[b] = 0;
    c->shadow = 0;
    c->fetch_extend = c->fetch_shadow = 0;
    c->iter += 1;
    bool more = c->extend[p ^ 1u] + c->regen[p ^ 1u] > 0;
    if (more && c->iter >= P.max_iterations) { c->error |= kFaultPathLoop; more = false; }
    c->more = more ? 1u : 0u;
    if (use_handle) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

}  // namespace

int wavefront_blocks_per_sm(int stage, int block) {
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch (stage) {
        case 0: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_generate, block, 0); break;
        case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_extend, block, 0); break;
        case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shade, block, 0); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wf_shadow, block, 0); break;
    }
    return e == cudaSuccess ? n : -1;
}

cudaError_t launch_wf_init(const WfParams* params, uint32_t capacity, cudaStream_t stream) {
    uint32_t grid = (capacity + 255) / 256;
    grid = grid > 4096 ? 4096 : (grid == 0 ? 1 : grid);
    wf_init<<<grid, 256, 0, stream>>>(params);
    return cudaGetLastError();
}

cudaError_t launch_wf_iteration(const WfParams* params, const WfLaunch& L, cudaGraphConditionalHandle handle,
                                int use_handle, cudaStream_t stream) {
    wf_generate<<<L.grid[0], L.block[0], 0, stream>>>(params);
    wf_extend<<<L.grid[1], L.block[1], 0, stream>>>(params);
    wf_shade<<<L.grid[2], L.block[2], 0, stream>>>(params);
    wf_shadow<<<L.grid[3], L.block[3], 0, stream>>>(params);
    wf_advance<<<1, 1, 0, stream>>>(params, handle, use_handle);
    return cudaGetLastError();
}

}  // namespace sol_b200
