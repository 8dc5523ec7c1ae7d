// K1: per-pixel path-tracing megakernel — the device statement of
// PathTracer::render + PathTracer::trace_path (src/algorithms/path_tracer.cpp:9-120).
//
// Schedule.  The grid is persistent (one wave of resident blocks).  Work items are
// pixels taken in 8x4 tiles so that a warp starts on a compact block of the image;
// a lane claims a new pixel through a warp-aggregated atomic when its current
// pixel has run all of its samples, and starts the next sample of its pixel as
// soon as a path ends (path regeneration), so lanes stay busy until the image is
// exhausted.  One lane owns a pixel for all of its samples, which keeps the
// per-pixel sum in SoL's sample order and the result bit-identical to the host.
//
// Renders of more than one sample use the split schedule instead (the host's
// AUTO choice): a work item is one (pixel, sample), so the samples of a pixel
// run on different lanes; each writes its path's colour (0 + colour, as the
// per-pixel sum starts) to a scratch plane of its sample, and sum_samples adds
// each pixel's colours in sample order, which is the same sequence of
// additions as the per-pixel loop and gives the same bits.
//
// One iteration of the loop traces one closest-hit ray, shades the hit (direct
// emission with MIS, light sample + MIS, Russian roulette, BSDF sample), then
// traces the shadow ray of that vertex.  The light contribution is added after
// the shadow ray returns and before the next vertex's emission, which is the
// order SoL adds them in; the random draws happen in SoL's order regardless of
// the shadow ray's outcome.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "path.cuh"
#include "wavefront.h"

namespace sol_b200 {

namespace {

__device__ __forceinline__ uint32_t claim_items(uint32_t* counter) {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    const unsigned rank = __popc(mask & ((1u << lane) - 1u));
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + rank;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

template <bool kCount, bool kSplit, int kMinBlocks, bool kBasic>
__global__ void __launch_bounds__(kMegakernelBlock, kMinBlocks)
pt_megakernel(SceneView s, DCamera cam, DConfig cfg, uint64_t sample_index, uint32_t sample_count,
              uint32_t width, uint32_t height, float* __restrict__ film, DeviceCounters* __restrict__ ctr) {
    const uint32_t tiles_x = (width + 7u) / 8u;
    const uint32_t total = tiles_x * ((height + 3u) / 4u) * 32u;
    // Split: `film` is the scratch of sample_count x 3 planes; items are (sample, pixel).
    const uint32_t items = kSplit ? total * sample_count : total;
    const uint32_t item_samples = kSplit ? 1u : sample_count;
    const size_t plane = (size_t)width * height;
    const float light_pick_prob = 1.0f / (float)s.num_lights;

    TraversalCounters tc{0u, 0u};
    uint32_t n_paths = 0, n_rays = 0, n_shadow = 0;
#if SOL_MEGAKERNEL_SHARED_STACK
    __shared__ int stack_smem[kSharedStackDepth * kMegakernelBlock];
    SharedStack<kMegakernelBlock> stack{stack_smem + threadIdx.x};
#else
    LocalStack stack;
#endif

    bool have_pixel = false;
    uint32_t px = 0, py = 0, sample = 0, sample_end = 0;
    Rgb pix_sum = rgb(0.0f);
    PathState ps;
    bool done = false;
    // Self-check bounds: a lane never needs more iterations than the pixels it
    // can claim times their samples times the path length (plus one per claim).
    const unsigned long long loop_bound = (unsigned long long)items * ((unsigned long long)item_samples + 1ull) *
                                          ((unsigned long long)cfg.max_path_len + 1ull) + 64ull;
    unsigned long long iterations = 0, claims = 0;
    bool alive = false;   // the lane has a path in flight

    while (true) {
        if (++iterations > loop_bound) { atomicOr(s.fault, kFaultPathLoop); break; }
        // --- make sure this lane has a live path (or stop) ------------------
        while (!alive) {
            if (++claims > loop_bound) { atomicOr(s.fault, kFaultClaimLoop); done = true; break; }
            if (have_pixel && sample < sample_end) {
                start_path(ps, cam, sample_index + sample, px, py, width, height);
                ++n_paths;
                if (cfg.max_path_len == 0) { pix_sum = pix_sum + ps.color; ++sample; continue; }
                alive = true;
            } else {
                if (have_pixel) {
                    size_t i = (size_t)py * width + px;
                    if (kSplit) {
                        float* f = film + (size_t)(sample_end - 1u) * 3u * plane;
                        f[i] = pix_sum.r;
                        f[i + plane] = pix_sum.g;
                        f[i + 2 * plane] = pix_sum.b;
                    } else {
                        // image.h:54-60 accumulate
                        film[i] += pix_sum.r;
                        film[i + plane] += pix_sum.g;
                        film[i + 2 * plane] += pix_sum.b;
                    }
                    have_pixel = false;
                }
                const uint32_t item = claim_items(&ctr->next_item);
                if (item >= items) { done = true; break; }
                const uint32_t k = kSplit ? item / total : 0u;
                const uint32_t it = item - k * total;
                uint32_t tile = it >> 5, l = it & 31u;
                px = (tile % tiles_x) * 8u + (l & 7u);
                py = (tile / tiles_x) * 4u + (l >> 3);
                if (px < width && py < height) {
                    have_pixel = true;
                    sample = k;
                    sample_end = k + item_samples;
                    pix_sum = rgb(0.0f);
                }
            }
        }
        if (done) break;

        // --- closest hit (path_tracer.cpp:42) ------------------------------
        float t = kFloatMax, hu, hv;
        const int slot = traverse_closest_uv<kCount>(s, ps.org, ps.dir, ps.tmin, t, hu, hv, tc, stack);
        ++n_rays;

        VertexOut vo;
        vo.has_shadow = false;
        vo.end = slot < 0;
        if (!vo.end) shade_vertex<kBasic>(s, cfg, light_pick_prob, slot, t, ps, vo, true, hu, hv);

        // --- shadow ray of this vertex (path_tracer.cpp:72-74) -------------
        if (vo.has_shadow) {
            float smax = 1.0f - cfg.ray_offset;
            const int occ = traverse<true, kCount>(s, vo.sh_org, vo.sh_dir, cfg.ray_offset, smax, tc, stack);
            ++n_rays;
            ++n_shadow;
            if (occ < 0) ps.color = ps.color + vo.pending;
        }

        bool end = vo.end;
        if (!end) {
            ++ps.path_len;
            end = ps.path_len >= cfg.max_path_len;
        }
        if (end) {
            pix_sum = pix_sum + ps.color;   // path_tracer.cpp:19
            ++sample;
            alive = false;
        }
    }

    // Counters: all lanes of the warp meet here before reducing.
    __syncwarp();
    unsigned long long v0 = warp_sum_u64(n_paths), v1 = warp_sum_u64(n_rays), v2 = warp_sum_u64(n_shadow);
    unsigned long long v3 = warp_sum_u64(tc.nodes), v4 = warp_sum_u64(tc.tris);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&ctr->paths, v0);
        atomicAdd(&ctr->rays, v1);
        atomicAdd(&ctr->shadow_rays, v2);
        if (kCount) { atomicAdd(&ctr->nodes, v3); atomicAdd(&ctr->tris, v4); }
    }
}

/// K1 in the split schedule, lean form: every work item is one path, so a lane
/// claims an item, traces its path to the end and writes the colour (0 +
/// colour, as the per-pixel sum starts) to the scratch plane of its sample,
/// then claims the next.  The same path computation and the same scratch as
/// pt_megakernel<kCount = false, kSplit = true>, with less state live across
/// the traversal (no per-pixel sum, sample range or loop bounds: the claim
/// loop ends with the items and the bounce loop with the path length, and
/// the traversal keeps its own step bound), so the register-capped builds
/// spill less.  When the warp claims work is set by SOL_LEAN_REGEN_MIN: by
/// default its idle lanes claim consecutive items together once 20 of its 32
/// lanes are idle; with 0 the warp claims 32 items at once (one sample of one
/// 8x4 tile) and waits for its longest path before the next claim.  Both beat
/// regenerating each lane's path at once, which lets the lanes drift apart.
template <int kMinBlocks, bool kBasic>
__global__ void __launch_bounds__(kMegakernelBlock, kMinBlocks)
pt_megakernel_lean(SceneView s, DCamera cam, DConfig cfg, uint64_t sample_index, uint32_t sample_count,
                   uint32_t width, uint32_t height, float* __restrict__ scratch, DeviceCounters* __restrict__ ctr) {
    const uint32_t tiles_x = (width + 7u) / 8u;
    const uint32_t total = tiles_x * ((height + 3u) / 4u) * 32u;   // items of one sample
    const uint32_t items = total * sample_count;
    const size_t plane = (size_t)width * height;
    const float light_pick_prob = 1.0f / (float)s.num_lights;
    TraversalCounters tc{0u, 0u};
    uint32_t n_paths = 0, n_rays = 0, n_shadow = 0;
    LocalStack stack;
#if SOL_LEAN_REGEN_MIN
    // One bounce per iteration; the warp's idle lanes claim new items together
    // once at least SOL_LEAN_REGEN_MIN of them are idle (or no lane has a
    // path), so lanes neither wait for the warp's longest path nor drift apart
    // one by one.  Every lane stays in the loop until the whole warp is done
    // (the exit test is a warp-uniform vote), so the full-warp votes and the
    // barrier see all 32 lanes; every iteration either advances a live path by
    // one bounce or claims items, so the loop ends with the items.
    PathState ps;
    uint32_t k = 0, px = 0, py = 0;
    bool alive = false, done = false;
    while (true) {
        __syncwarp();
        const unsigned idle = __ballot_sync(0xffffffffu, !alive && !done);
        const unsigned busy = __ballot_sync(0xffffffffu, alive);
        if (busy == 0u && idle == 0u) break;
        if (!alive && !done && (__popc(idle) >= SOL_LEAN_REGEN_MIN || busy == 0u)) {
            const uint32_t item = claim_items(&ctr->next_item);
            if (item >= items) {
                done = true;
            } else {
                k = item / total;
                const uint32_t it = item - k * total;
                const uint32_t tile = it >> 5, l = it & 31u;
                px = (tile % tiles_x) * 8u + (l & 7u);
                py = (tile / tiles_x) * 4u + (l >> 3);
                if (px < width && py < height) {
                    start_path(ps, cam, sample_index + k, px, py, width, height);
                    ++n_paths;
                    alive = true;
                }
            }
        }
        if (alive) {
            bool end = ps.path_len >= cfg.max_path_len;
            if (!end) {
                // closest hit (path_tracer.cpp:42)
                float t = kFloatMax;
                float hu, hv;
                const int slot = traverse_closest_uv<false>(s, ps.org, ps.dir, ps.tmin, t, hu, hv, tc, stack);
                ++n_rays;
                if (slot < 0) {
                    end = true;
                } else {
                    VertexOut vo;
                    shade_vertex<kBasic>(s, cfg, light_pick_prob, slot, t, ps, vo, true, hu, hv);
                    // shadow ray of this vertex (path_tracer.cpp:72-74)
                    if (vo.has_shadow) {
                        float smax = 1.0f - cfg.ray_offset;
                        const int occ =
                            traverse<true, false>(s, vo.sh_org, vo.sh_dir, cfg.ray_offset, smax, tc, stack);
                        ++n_rays;
                        ++n_shadow;
                        if (occ < 0) ps.color = ps.color + vo.pending;
                    }
                    if (vo.end) end = true;
                    else end = ++ps.path_len >= cfg.max_path_len;
                }
            }
            if (end) {
                const Rgb c = rgb(0.0f) + ps.color;   // path_tracer.cpp:19; the sum pass adds in sample order
                float* f = scratch + (size_t)k * 3u * plane + (size_t)py * width + px;
                f[0] = c.r;
                f[plane] = c.g;
                f[2 * plane] = c.b;
                alive = false;
            }
        }
    }
#else
    while (true) {
        const uint32_t item = claim_items(&ctr->next_item);
        if (item >= items) break;
        const uint32_t k = item / total;
        const uint32_t it = item - k * total;
        const uint32_t tile = it >> 5, l = it & 31u;
        const uint32_t px = (tile % tiles_x) * 8u + (l & 7u);
        const uint32_t py = (tile / tiles_x) * 4u + (l >> 3);
        if (px >= width || py >= height) continue;   // padding of a partial tile
        PathState ps;
        start_path(ps, cam, sample_index + k, px, py, width, height);
        ++n_paths;
        while (ps.path_len < cfg.max_path_len) {
            // closest hit (path_tracer.cpp:42)
            float t = kFloatMax;
            float hu, hv;
            const int slot = traverse_closest_uv<false>(s, ps.org, ps.dir, ps.tmin, t, hu, hv, tc, stack);
            ++n_rays;
            if (slot < 0) break;
            VertexOut vo;
            shade_vertex<kBasic>(s, cfg, light_pick_prob, slot, t, ps, vo, true, hu, hv);
            // shadow ray of this vertex (path_tracer.cpp:72-74)
            if (vo.has_shadow) {
                float smax = 1.0f - cfg.ray_offset;
                const int occ = traverse<true, false>(s, vo.sh_org, vo.sh_dir, cfg.ray_offset, smax, tc, stack);
                ++n_rays;
                ++n_shadow;
                if (occ < 0) ps.color = ps.color + vo.pending;
            }
            if (vo.end) break;
            ++ps.path_len;
        }
        const Rgb c = rgb(0.0f) + ps.color;   // path_tracer.cpp:19, the sum pass adds the rest in sample order
        float* f = scratch + (size_t)k * 3u * plane + (size_t)py * width + px;
        f[0] = c.r;
        f[plane] = c.g;
        f[2 * plane] = c.b;
    }
#endif
    __syncwarp();
    unsigned long long v0 = warp_sum_u64(n_paths), v1 = warp_sum_u64(n_rays), v2 = warp_sum_u64(n_shadow);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&ctr->paths, v0);
        atomicAdd(&ctr->rays, v1);
        atomicAdd(&ctr->shadow_rays, v2);
    }
}

/// K1b: the megakernel over many views (cameras, films of uneven size and spp)
/// of one or more scenes in one persistent launch.  Work items are the views'
/// 8x4 pixel tiles laid end to end (WfView::item_begin); a lane claims a pixel
/// of any view, renders all its samples in order with path regeneration, adds
/// the sum into that view's film and claims the next — the schedule of K1 with
/// the view (scene, camera, film) looked up per pixel.  Split views (small
/// images) have one item per (sample, pixel) as K1's split schedule does, and
/// sum_samples_views adds their scratch planes afterwards, so every film has
/// the bits a separate K1 launch gives it.
///
/// With kTable the scenes come in `table`, a kernel parameter in constant
/// space as K1's scene is, so the traversal reads array pointers and sizes as
/// constant operands; otherwise from the device array `scenes`.
template <bool kCount, bool kTable, bool kBasic>
__global__ void __launch_bounds__(kMegakernelBlock, kMegakernelViewsMinBlocks)
pt_megakernel_views(const WfView* __restrict__ views, uint32_t num_views, uint32_t total, uint32_t max_spp,
                    const SceneView* __restrict__ scenes, const __grid_constant__ SceneTable table, DConfig cfg,
                    DeviceCounters* __restrict__ ctr, unsigned int* __restrict__ fault) {
    TraversalCounters tc{0u, 0u};
    uint32_t n_paths = 0, n_rays = 0, n_shadow = 0;
    LocalStack stack;
    bool have_pixel = false;
    uint32_t px = 0, py = 0, sample = 0, sample_end = 0, vi = 0;
    Rgb pix_sum = rgb(0.0f);
    PathState ps;
    const SceneView* s = kTable ? &table.v[0] : scenes;
    float light_pick_prob = 1.0f;
    bool done = false;
    // Self-check bound: a lane claims at most every item, each with at most
    // max_spp samples of at most max_path_len vertices.
    const unsigned long long loop_bound = (unsigned long long)total * ((unsigned long long)max_spp + 1ull) *
                                          ((unsigned long long)cfg.max_path_len + 1ull) + 64ull;
    unsigned long long iterations = 0, claims = 0;
    bool alive = false;

    while (true) {
        if (++iterations > loop_bound) { atomicOr(fault, kFaultPathLoop); break; }
        while (!alive) {
            if (++claims > loop_bound) { atomicOr(fault, kFaultClaimLoop); done = true; break; }
            const WfView& V = views[vi];
            if (have_pixel && sample < sample_end) {
                DCamera cam;
                for (int k = 0; k < 3; ++k) {
                    cam.eye[k] = V.eye[k]; cam.dir[k] = V.dir[k]; cam.right[k] = V.right[k]; cam.up[k] = V.up[k];
                }
                start_path(ps, cam, V.sample_index + sample, px, py, V.width, V.height);
                ++n_paths;
                if (cfg.max_path_len == 0) { pix_sum = pix_sum + ps.color; ++sample; continue; }
                alive = true;
            } else {
                if (have_pixel) {
                    const size_t plane = (size_t)V.width * V.height;
                    const size_t i = (size_t)py * V.width + px;
                    if (V.split) {
                        float* f = V.scratch + (size_t)(sample_end - 1u) * 3u * plane;
                        f[i] = pix_sum.r;
                        f[i + plane] = pix_sum.g;
                        f[i + 2 * plane] = pix_sum.b;
                    } else {
                        // image.h:54-60 accumulate
                        V.film[i] += pix_sum.r;
                        V.film[i + plane] += pix_sum.g;
                        V.film[i + 2 * plane] += pix_sum.b;
                    }
                    have_pixel = false;
                }
                const uint32_t item = claim_items(&ctr->next_item);
                if (item >= total) { done = true; break; }
                // Consecutive claims almost always stay in the lane's current view:
                // check it before searching the table.
                uint32_t lo = vi;
                if (!(views[vi].item_begin <= item && (vi + 1u == num_views || item < views[vi + 1u].item_begin))) {
                    lo = 0;
                    uint32_t hi = num_views;
                    while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (views[mid].item_begin <= item) lo = mid; else hi = mid; }
                }
                const WfView& W = views[lo];
                uint32_t local = item - W.item_begin, k = 0;
                if (W.split) {
                    const uint32_t per_sample = W.tiles_x * ((W.height + 3u) / 4u) * 32u;
                    k = local / per_sample;
                    local -= k * per_sample;
                }
                const uint32_t tile = local >> 5, l = local & 31u;
                px = (tile % W.tiles_x) * 8u + (l & 7u);
                py = (tile / W.tiles_x) * 4u + (l >> 3);
                if (px < W.width && py < W.height) {
                    have_pixel = true;
                    vi = lo;
                    sample = k;
                    sample_end = W.split ? k + 1u : W.sample_count;
                    pix_sum = rgb(0.0f);
                    s = kTable ? &table.v[W.scene] : scenes + W.scene;
                    light_pick_prob = 1.0f / (float)s->num_lights;
                }
            }
        }
        if (done) break;

        float t = kFloatMax, hu, hv;
        const int slot = traverse_closest_uv<kCount>(*s, ps.org, ps.dir, ps.tmin, t, hu, hv, tc, stack);
        ++n_rays;
        VertexOut vo;
        vo.has_shadow = false;
        vo.end = slot < 0;
        if (!vo.end) shade_vertex<kBasic>(*s, cfg, light_pick_prob, slot, t, ps, vo, true, hu, hv);
        if (vo.has_shadow) {
            float smax = 1.0f - cfg.ray_offset;
            const int occ = traverse<true, kCount>(*s, vo.sh_org, vo.sh_dir, cfg.ray_offset, smax, tc, stack);
            ++n_rays;
            ++n_shadow;
            if (occ < 0) ps.color = ps.color + vo.pending;
        }
        bool end = vo.end;
        if (!end) {
            ++ps.path_len;
            end = ps.path_len >= cfg.max_path_len;
        }
        if (end) {
            pix_sum = pix_sum + ps.color;   // path_tracer.cpp:19
            ++sample;
            alive = false;
        }
    }
    __syncwarp();
    unsigned long long v0 = warp_sum_u64(n_paths), v1 = warp_sum_u64(n_rays), v2 = warp_sum_u64(n_shadow);
    unsigned long long v3 = warp_sum_u64(tc.nodes), v4 = warp_sum_u64(tc.tris);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&ctr->paths, v0);
        atomicAdd(&ctr->rays, v1);
        atomicAdd(&ctr->shadow_rays, v2);
        if (kCount) { atomicAdd(&ctr->nodes, v3); atomicAdd(&ctr->tris, v4); }
    }
}

/// Adds each pixel's per-sample colours of one chunk of samples (scratch:
/// sample_count x 3 planes) in sample order to the pixel's running sum, which
/// starts from 0 with the first chunk as the per-pixel loop's sum does; after
/// the last chunk the sum is added into the film.  One chunk is both.
__global__ void __launch_bounds__(256)
sum_samples(const float* __restrict__ scratch, uint32_t sample_count, size_t plane, float* __restrict__ running,
            bool first, bool last, float* __restrict__ film) {
    const size_t n = 3 * plane;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float sum = first ? 0.0f : running[i];
        for (uint32_t k = 0; k < sample_count; ++k) sum += scratch[(size_t)k * n + i];
        if (last) film[i] += sum;
        else running[i] = sum;
    }
}

/// The sum pass of split views (K1b's, the wavefront's): every float of those
/// views' films (laid end to end from WfView::sum_begin) gets its pixel's
/// per-sample colours added in sample order, starting from 0 -- or, for a
/// chunk of a view's samples after the first, from the sum the earlier chunks
/// left in `running`; the last chunk adds the sum into the film.
__global__ void __launch_bounds__(256)
sum_samples_views(const WfView* __restrict__ views, uint32_t num_views, uint64_t total) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total; g += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = num_views;
        while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (views[mid].sum_begin <= g) lo = mid; else hi = mid; }
        // Non-split views occupy no range: the last split view starting at or before g owns g.
        while (lo > 0 && !views[lo].split) --lo;
        if (!views[lo].split) continue;
        const WfView& V = views[lo];
        const size_t n = 3 * (size_t)V.width * V.height;
        const size_t i = (size_t)(g - V.sum_begin);
        float sum = V.first_chunk ? 0.0f : V.running[i];
        for (uint32_t k = 0; k < V.sample_count; ++k) sum += V.scratch[(size_t)k * n + i];
        if (V.last_chunk) V.film[i] += sum;
        else V.running[i] = sum;
    }
}

}  // namespace

namespace {

/// The K1 instantiation for a counting flag, schedule, occupancy target and
/// shading (basic: the scene has no image textures and no Interp BSDFs; the
/// counting build always has full shading).
template <bool kSplit>
auto megakernel_fn(bool instrumented, bool full, bool basic) {
    if (instrumented) return full ? pt_megakernel<true, kSplit, kMegakernelMinBlocks, false>
                                  : pt_megakernel<true, kSplit, kMegakernelSmallMinBlocks, false>;
#if SOL_MEGAKERNEL_SPLIT_LEAN
    if (kSplit) {
        if (basic) return full ? pt_megakernel_lean<kMegakernelMinBlocks, true>
                               : pt_megakernel_lean<kMegakernelSmallMinBlocks, true>;
        return full ? pt_megakernel_lean<kMegakernelMinBlocks, false>
                    : pt_megakernel_lean<kMegakernelSmallMinBlocks, false>;
    }
#endif
    if (basic) return full ? pt_megakernel<false, kSplit, kMegakernelMinBlocks, true>
                           : pt_megakernel<false, kSplit, kMegakernelSmallMinBlocks, true>;
    return full ? pt_megakernel<false, kSplit, kMegakernelMinBlocks, false>
                : pt_megakernel<false, kSplit, kMegakernelSmallMinBlocks, false>;
}

}  // namespace

int megakernel_blocks_per_sm(bool instrumented, bool full, bool basic) {
    int n = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, megakernel_fn<true>(instrumented, full, basic),
                                                                  kMegakernelBlock, 0);
    return e == cudaSuccess ? n : -1;
}

cudaError_t launch_megakernel(const SceneView& s, const DCamera& cam, const DConfig& cfg,
                              uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                              float* film, DeviceCounters* counters, bool instrumented, bool full, bool basic,
                              int grid, cudaStream_t stream, const L2Window& l2) {
    return launch_l2(megakernel_fn<false>(instrumented, full, basic), grid, kMegakernelBlock, 0, stream, l2, s, cam, cfg,
                     sample_index, sample_count, width, height, film, counters);
}

int megakernel_views_blocks_per_sm() {
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pt_megakernel_views<false, true, false>, kMegakernelBlock, 0) ==
                   cudaSuccess
               ? n : -1;
}

cudaError_t launch_megakernel_views(const WfView* views, uint32_t num_views, uint32_t total_items, uint32_t max_spp,
                                    const SceneView* scenes, const SceneView* host_scenes, uint32_t num_scenes,
                                    bool basic, const DConfig& cfg, DeviceCounters* counters, unsigned int* fault,
                                    int grid, cudaStream_t stream, const L2Window& l2) {
    SceneTable table{};
    if (num_scenes <= kViewsTableScenes) {
        for (uint32_t i = 0; i < num_scenes; ++i) table.v[i] = host_scenes[i];
        return launch_l2(basic ? pt_megakernel_views<false, true, true> : pt_megakernel_views<false, true, false>,
                         grid, kMegakernelBlock, 0, stream, l2, views, num_views, total_items, max_spp, scenes, table,
                         cfg, counters, fault);
    }
    return launch_l2(pt_megakernel_views<false, false, false>, grid, kMegakernelBlock, 0, stream, l2, views, num_views,
                     total_items, max_spp, scenes, table, cfg, counters, fault);
}

cudaError_t launch_sum_samples_views(const WfView* views, uint32_t num_views, uint64_t total_floats,
                                     cudaStream_t stream) {
    if (total_floats == 0) return cudaSuccess;
    const int blocks = (int)std::min<uint64_t>((total_floats + 255) / 256, 8192);
    sum_samples_views<<<blocks, 256, 0, stream>>>(views, num_views, total_floats);
    return cudaGetLastError();
}

cudaError_t launch_megakernel_split(const SceneView& s, const DCamera& cam, const DConfig& cfg,
                                    uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                                    float* film, float* scratch, float* running, uint32_t chunk,
                                    DeviceCounters* counters, bool instrumented, bool full, bool basic, int grid,
                                    cudaStream_t stream, const L2Window& l2) {
    if (chunk == 0 || (chunk < sample_count && running == nullptr)) return cudaErrorInvalidValue;
    const size_t plane = (size_t)width * height;
    const int blocks = (int)std::min<size_t>((3 * plane + 255) / 256, 4096);
    for (uint32_t c0 = 0; c0 < sample_count; c0 += chunk) {
        const uint32_t k = std::min(chunk, sample_count - c0);
        cudaError_t e = cudaSuccess;
        if (c0 > 0) e = cudaMemsetAsync(&counters->next_item, 0, sizeof(counters->next_item), stream);
        if (e != cudaSuccess) return e;
        e = launch_l2(megakernel_fn<true>(instrumented, full, basic), grid, kMegakernelBlock, 0, stream, l2, s, cam, cfg,
                      sample_index + c0, k, width, height, scratch, counters);
        if (e != cudaSuccess) return e;
        sum_samples<<<blocks, 256, 0, stream>>>(scratch, k, plane, running, c0 == 0, c0 + k == sample_count, film);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace sol_b200
