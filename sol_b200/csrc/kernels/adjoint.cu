// K7: path-replay adjoint of the forward render, and K8: the L2 image loss.
//
// The gradient is that of an image loss L with respect to the scene's texture
// values (constant albedos, specular colours and emissions, and image texels;
// the parameter layout is described in include/sol_gpu.h), for the same
// Monte Carlo estimate the forward render computes: every path is replayed
// from its seed (Path Replay Backpropagation; Vicini, Speierer, Jakob, SIGGRAPH
// 2021), so no path is stored between kernels.  Geometry is fixed, so texture
// values change no sampled direction and no visibility; the derivative of each
// replayed path is exact, including the dependence of the Russian roulette
// probability clamp(lum(T)) on the throughput (path_tracer.cpp:100-107).
//
// One lane owns a pixel and replays its samples one after another.  A replay
// records per vertex the quantities the reverse sweep needs (at most
// kAdjointMaxDepth vertices, in registers/local memory), then sweeps from the
// last vertex to the first carrying dL/dT, and adds the texture gradients with
// warp-reduced atomics (lanes writing the same address are summed first).
#include <cuda_runtime.h>

#include "adjoint.h"
#include "kernels.h"
#include "path.cuh"

namespace sol_b200 {

namespace {

constexpr uint32_t kEmit = 1u, kNee = 2u, kBounce = 4u, kRrLive = 8u;

/// A texture value's factor in a colour: colour = value * scale (per channel).
struct TexTerm {
    int tex;
    float scale;
};

struct VertexRec {
    Rgb T;                      // throughput before the vertex
    Rgb E; float m;             // emission and its MIS weight
    int etex; Vec2 euv;
    Rgb Ls; Rgb f; float s;     // light sample: intensity, BSDF value, scalar factor
    int ltex; Vec2 luv;
    TexTerm fterm[2];
    Rgb c; float r;             // bounce: T' = T * c * r
    TexTerm cterm[2];
    float q;                    // Russian roulette survival probability
    Vec2 uv;                    // shading texture coordinates
    uint32_t flags;
};

__device__ __forceinline__ uint32_t lane() { return threadIdx.x & 31u; }

/// atomicAdd that first sums the values of the lanes that target the same address.
__device__ __forceinline__ void atomic_add_reduced(float* addr, float v) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, (unsigned long long)addr);
    const int n = __popc(peers);
    const int rank = __popc(peers & ((1u << lane()) - 1u));
    float sum = v;
    for (int s = 1; s < n; s <<= 1) {
        const int src = rank + s < n ? (int)__fns(peers, 0, rank + s + 1) : (int)lane();
        const float other = __shfl_sync(peers, sum, src);
        if (rank + s < n && (rank & (2 * s - 1)) == 0) sum += other;
    }
    if (rank == 0 && sum != 0.0f) atomicAdd(addr, sum);
}

/// Adds `a` (d loss / d colour value) into the parameters of colour texture `tex` at `uv`.
__device__ void scatter_color(const SceneView& s, float* grad, int tex, Vec2 uv, Rgb a) {
    if (tex < 0) return;
    const DTexture t = s.textures[tex];
    float* base = grad + s.param_offsets[tex];
    if (t.kind == SOL_GPU_TEX_CONSTANT_COLOR) {
        atomic_add_reduced(base + 0, a.r);
        atomic_add_reduced(base + 1, a.g);
        atomic_add_reduced(base + 2, a.b);
        return;
    }
    if (t.kind != SOL_GPU_TEX_IMAGE) return;
    // The texels and weights of image_color (src/textures.cpp:5-52).
    if (t.border == SOL_GPU_BORDER_CLAMP) {
        uv = vec2(clampf(uv.x, 0.0f, 1.0f), clampf(uv.y, 0.0f, 1.0f));
    } else if (t.border == SOL_GPU_BORDER_REPEAT) {
        uv = vec2(uv.x - floor_(uv.x), uv.y - floor_(uv.y));
    } else {
        float u = fmodf(uv.x, 2.0f), v = fmodf(uv.x, 2.0f);
        uv = vec2(u > 1.0f ? 2.0f - u : u, v > 1.0f ? 2.0f - v : v);
    }
    const DImage img = s.images[t.image];
    const int w = (int)img.width, h = (int)img.height;
    const size_t plane = (size_t)img.width * img.height;
    int xs[4], ys[4];
    float ws[4];
    int n;
    if (t.filter == SOL_GPU_FILTER_NEAREST) {
        xs[0] = clampi((int)(uv.x * (float)img.width), 0, w - 1);
        ys[0] = clampi((int)(uv.y * (float)img.height), 0, h - 1);
        ws[0] = 1.0f;
        n = 1;
    } else {
        float i = uv.x * (float)(img.width - 1), j = uv.y * (float)(img.height - 1);
        float fu = i - floor_(i), fv = j - floor_(j);
        int x0 = clampi((int)i, 0, w - 1), y0 = clampi((int)j, 0, h - 1);
        int x1 = clampi(x0 + 1, 0, w - 1), y1 = clampi(y0 + 1, 0, h - 1);
        xs[0] = x0; ys[0] = y0; ws[0] = (1.0f - fu) * (1.0f - fv);
        xs[1] = x1; ys[1] = y0; ws[1] = fu * (1.0f - fv);
        xs[2] = x0; ys[2] = y1; ws[2] = (1.0f - fu) * fv;
        xs[3] = x1; ys[3] = y1; ws[3] = fu * fv;
        n = 4;
    }
    for (int k = 0; k < n; ++k) {
        float* p = base + (size_t)ys[k] * img.width + xs[k];
        atomic_add_reduced(p, ws[k] * a.r);
        atomic_add_reduced(p + plane, ws[k] * a.g);
        atomic_add_reduced(p + 2 * plane, ws[k] * a.b);
    }
}

__device__ __forceinline__ void scatter_terms(const SceneView& s, float* grad, const TexTerm* terms, Vec2 uv, Rgb a) {
    for (int k = 0; k < 2; ++k)
        if (terms[k].tex >= 0 && terms[k].scale != 0.0f) scatter_color(s, grad, terms[k].tex, uv, a * terms[k].scale);
}

/// d(eval)/d(colour value) of a non-interpolating BSDF for `in_dir`: the factor
/// its colour texture is multiplied by (bsdfs.cpp:35-37, 102-104).
__device__ __forceinline__ TexTerm eval_term(const SceneView& s, const DBsdf& b, Vec3 in_dir, const Surface& sf,
                                             Vec3 out_dir) {
    TexTerm t{-1, 0.0f};
    if (b.kind == SOL_GPU_BSDF_DIFFUSE) {
        t.tex = b.tex[0];
        t.scale = kInvPi;
    } else if (b.kind == SOL_GPU_BSDF_PHONG) {
        const float ns = tex_scalar(s, b.tex[1], sf.uv);
        t.tex = b.tex[0];
        t.scale = pow_(reflect_cosine(in_dir, sf.normal(), out_dir), ns) * (ns + 2.0f) * (0.5f * kInvPi);
    }
    return t;
}

/// Terms of Bsdf::eval for any kind (InterpBsdf: both operands, bsdfs.cpp:185-190).
__device__ __forceinline__ void eval_terms(const SceneView& s, int id, Vec3 in_dir, const Surface& sf, Vec3 out_dir,
                                           TexTerm* out) {
    const DBsdf b = s.bsdfs[id];
    out[1] = TexTerm{-1, 0.0f};
    if (b.kind != SOL_GPU_BSDF_INTERP) { out[0] = eval_term(s, b, in_dir, sf, out_dir); return; }
    const float k = tex_scalar(s, b.tex[0], sf.uv);
    out[0] = eval_term(s, s.bsdfs[b.a], in_dir, sf, out_dir);
    out[1] = eval_term(s, s.bsdfs[b.b], in_dir, sf, out_dir);
    out[0].scale *= 1.0f - k;
    out[1].scale *= k;
}

/// Terms of a basic BSDF's sampled colour (bsdfs.cpp:39-48, 72-85, 112-119, 138-165).
__device__ __forceinline__ TexTerm sample_term(const SceneView& s, const DBsdf& b, const BsdfSample& bs,
                                               const Surface& sf, Vec3 out_dir) {
    if (b.kind == SOL_GPU_BSDF_MIRROR) return TexTerm{b.tex[0], 1.0f};
    if (b.kind == SOL_GPU_BSDF_GLASS) {
        const bool refracted = dot(bs.in_dir, sf.face_normal) < 0.0f;
        return TexTerm{refracted ? b.tex[1] : b.tex[0], 1.0f};
    }
    return eval_term(s, b, bs.in_dir, sf, out_dir);
}

/// Whether Light::emission returns the intensity texture (lights.cpp:94-106):
/// area lights seen from the side their normal points to.
__device__ __forceinline__ bool emits(const DLight& l, Vec3 dir, Vec2 uv) {
    if (l.kind == SOL_GPU_LIGHT_POINT) return false;
    Vec3 n;
    if (l.kind == SOL_GPU_LIGHT_TRIANGLE) {
        n = vec3(l.n[0], l.n[1], l.n[2]);
    } else {
        float pdf;
        n = sample_uniform_sphere(uv.x, uv.y, &pdf);
    }
    return dot(dir, n) > 0.0f;
}

/// Adjoint of one path (one pixel sample): replay, then reverse sweep.
__device__ void adjoint_path(const SceneView& s, const DConfig& cfg, const DCamera& cam, uint64_t frame,
                             uint32_t px, uint32_t py, uint32_t width, uint32_t height, Rgb G, float* grad,
                             VertexRec* rec, uint32_t& n_rays) {
    PathState ps;
    start_path(ps, cam, frame, px, py, width, height);
    const float light_pick_prob = 1.0f / (float)s.num_lights;
    const uint32_t nl = s.num_lights;
    int K = 0;
    for (uint32_t path_len = 0; path_len < cfg.max_path_len && K < kAdjointMaxDepth; ++path_len) {
        float t = kFloatMax;
        TraversalCounters tc{0u, 0u};
        const int slot = traverse<false, false>(s, ps.org, ps.dir, ps.tmin, t, tc);
        ++n_rays;
        if (slot < 0) break;
        VertexRec& R = rec[K++];
        R.flags = 0;
        R.T = ps.T;
        R.fterm[0] = R.fterm[1] = R.cterm[0] = R.cterm[1] = TexTerm{-1, 0.0f};
        int bsdf_id, light_id;
        const Surface sf = make_surface(s, slot, ps.org, ps.dir, t, ps.tmin, &bsdf_id, &light_id);
        R.uv = sf.uv;
        const Vec3 out_dir = -ps.dir;
        if (light_id >= 0 && sf.front) {
            const float pdf_prev_area = ps.pdf_prev * dot(out_dir, sf.normal()) / (t * t);
            Rgb le; float pdf_from;
            const DLight light = s.lights[light_id];
            light_emission(s, light, out_dir, sf.surf, &le, &pdf_from);
            const float mis = ps.pdf_prev != 0.0f ? balance_heuristic(pdf_prev_area, pdf_from * light_pick_prob) : 1.0f;
            R.flags |= kEmit;
            R.E = le;
            R.m = mis;
            R.etex = emits(light, out_dir, sf.surf) ? light.tex : -1;
            R.euv = sf.surf;
        }
        if (bsdf_id < 0) break;
        const bool skip_nee = s.bsdfs[bsdf_id].type == kTypeSpecular;
        if (!skip_nee && nl > 0) {
            uint32_t li = (uint32_t)(ps.rng.next_float() * (float)nl);
            li = li < nl - 1 ? li : nl - 1;
            const DLight light = s.lights[li];
            // The light sample's surface coordinates, as light_sample_area folds them.
            Pcg peek = ps.rng;
            float lv = peek.next_float(), lu = peek.next_float();
            if (light.kind == SOL_GPU_LIGHT_TRIANGLE && lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
            LightSample ls;
            if (light_sample_area(s, light, ps.rng, sf.point, &ls)) {
                Vec3 in_dir = ls.pos - sf.point;
                float cos_surf = dot(in_dir, sf.normal());
                float smax = 1.0f - cfg.ray_offset;
                const int occ = traverse<true, false>(s, sf.point, ls.pos - sf.point, cfg.ray_offset, smax, tc);
                ++n_rays;
                if (occ < 0) {
                    const float inv_light_dist = 1.0f / length(in_dir);
                    cos_surf = cos_surf * inv_light_dist;
                    in_dir = in_dir * inv_light_dist;
                    const bool has_area = light.kind != SOL_GPU_LIGHT_POINT;
                    const float pdf_bounce = has_area ? bsdf_pdf(s, bsdf_id, in_dir, sf, out_dir) : 0.0f;
                    const float pdf_light = ls.pdf_from * light_pick_prob;
                    const float geom_term = ls.cos * inv_light_dist * inv_light_dist;
                    const float mis = has_area ? balance_heuristic(pdf_light, pdf_bounce * geom_term) : 1.0f;
                    R.flags |= kNee;
                    R.Ls = ls.intensity;
                    R.f = bsdf_eval(s, bsdf_id, in_dir, sf, out_dir);
                    R.s = geom_term * cos_surf * mis / pdf_light;
                    R.ltex = light.kind == SOL_GPU_LIGHT_POINT ? -1 : light.tex;
                    R.luv = vec2(lu, lv);
                    eval_terms(s, bsdf_id, in_dir, sf, out_dir, R.fterm);
                }
            }
        }
        float survival = 1.0f;
        if (path_len >= cfg.min_rr_path_len) {
            const float lum = luminance(ps.T);
            survival = clampf(lum, cfg.min_survival_prob, cfg.max_survival_prob);
            if (lum > cfg.min_survival_prob && lum < cfg.max_survival_prob) R.flags |= kRrLive;
            if (ps.rng.next_float() >= survival) break;
        }
        R.q = survival;
        // Which operand an InterpBsdf samples is its first draw (bsdfs.cpp:192-198).
        const DBsdf b = s.bsdfs[bsdf_id];
        int target = bsdf_id, other = -1;
        float k = 1.0f;
        if (b.kind == SOL_GPU_BSDF_INTERP) {
            Pcg peek = ps.rng;
            k = tex_scalar(s, b.tex[0], sf.uv);
            target = b.b; other = b.a;
            if (peek.next_float() > k) { target = b.a; other = b.b; k = 1.0f - k; }
        }
        BsdfSample bs;
        if (!bsdf_sample(s, bsdf_id, ps.rng, sf, out_dir, &bs)) break;
        R.flags |= kBounce;
        R.c = bs.color;
        R.r = bs.cos / (bs.pdf * survival);
        R.cterm[0] = sample_term(s, s.bsdfs[target], bs, sf, out_dir);
        if (other >= 0) {
            R.cterm[0].scale *= k;
            R.cterm[1] = eval_term(s, s.bsdfs[other], bs.in_dir, sf, out_dir);
            R.cterm[1].scale *= 1.0f - k;
        }
        ps.T = ps.T * (bs.color * (bs.cos / (bs.pdf * survival)));
        ps.org = sf.point;
        ps.dir = bs.in_dir;
        ps.tmin = cfg.ray_offset;
        ps.pdf_prev = skip_nee ? 0.0f : bs.pdf;
    }
    // Reverse sweep: a = dL/dT of the vertex after the current one.
    Rgb a = rgb(0.0f);
    for (int v = K - 1; v >= 0; --v) {
        const VertexRec& R = rec[v];
        Rgb aT = rgb(0.0f);
        if (R.flags & kBounce) {
            scatter_terms(s, grad, R.cterm, R.uv, a * R.T * R.r);
            aT = a * R.c * R.r;
            if (R.flags & kRrLive) {
                const Rgb aTc = a * R.T * R.c;
                const float a_q = -(aTc.r + aTc.g + aTc.b) * R.r / R.q;
                aT = aT + rgb(0.2126f * a_q, 0.7152f * a_q, 0.0722f * a_q);
            }
        }
        if (R.flags & kNee) {
            aT = aT + G * R.Ls * R.f * R.s;
            scatter_terms(s, grad, R.fterm, R.uv, G * R.Ls * R.T * R.s);
            scatter_color(s, grad, R.ltex, R.luv, G * R.T * R.f * R.s);
        }
        if (R.flags & kEmit) {
            aT = aT + G * R.E * R.m;
            scatter_color(s, grad, R.etex, R.euv, G * R.T * R.m);
        }
        a = aT;
    }
}

__global__ void __launch_bounds__(kAdjointBlock)
prb_adjoint(SceneView s, DCamera cam, DConfig cfg, uint64_t sample_index, uint32_t sample_count, uint32_t width,
            uint32_t height, const float* __restrict__ dl_dfilm, float* __restrict__ grad, DeviceCounters* ctr) {
    VertexRec rec[kAdjointMaxDepth];
    const uint32_t tiles_x = (width + 7u) / 8u;
    const uint32_t total = tiles_x * ((height + 3u) / 4u) * 32u;
    const size_t plane = (size_t)width * height;
    uint32_t n_rays = 0, n_paths = 0;
    while (true) {
        const unsigned mask = __activemask();
        const int leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if ((int)lane() == leader) base = atomicAdd(&ctr->next_item, (uint32_t)__popc(mask));
        const uint32_t item = __shfl_sync(mask, base, leader) + __popc(mask & ((1u << lane()) - 1u));
        if (item >= total) break;
        const uint32_t tile = item >> 5, l = item & 31u;
        const uint32_t px = (tile % tiles_x) * 8u + (l & 7u);
        const uint32_t py = (tile / tiles_x) * 4u + (l >> 3);
        if (px >= width || py >= height) continue;
        const size_t i = (size_t)py * width + px;
        const Rgb G = rgb(dl_dfilm[i], dl_dfilm[i + plane], dl_dfilm[i + 2 * plane]);
        if (G.r == 0.0f && G.g == 0.0f && G.b == 0.0f) continue;
        for (uint32_t k = 0; k < sample_count; ++k) {
            adjoint_path(s, cfg, cam, sample_index + k, px, py, width, height, G, grad, rec, n_rays);
            ++n_paths;
        }
    }
    atomicAdd(&ctr->rays, (unsigned long long)n_rays);
    atomicAdd(&ctr->paths, (unsigned long long)n_paths);
}

/// Forward render and adjoint of an L2 loss for many views of many scenes in
/// one persistent launch.  Per pixel: the samples are rendered exactly as the
/// megakernel renders them (their sum is added to the film), the pixel's loss
/// (estimate - target)^2 and its gradient 2 (estimate - target) / spp are formed
/// locally (the L2 loss of a pixel depends on that pixel alone), and the same
/// samples are replayed backwards into the view's scene gradient.
__global__ void __launch_bounds__(kAdjointBlock)
fused_forward_adjoint(const AdjView* __restrict__ views, uint32_t num_views, uint32_t total,
                      const SceneView* __restrict__ scenes, DConfig cfg, DeviceCounters* ctr) {
    VertexRec rec[kAdjointMaxDepth];
    uint32_t n_rays = 0, n_paths = 0;
    while (true) {
        const unsigned mask = __activemask();
        const int leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if ((int)lane() == leader) base = atomicAdd(&ctr->next_item, (uint32_t)__popc(mask));
        const uint32_t item = __shfl_sync(mask, base, leader) + __popc(mask & ((1u << lane()) - 1u));
        if (item >= total) break;
        uint32_t lo = 0, hi = num_views;
        while (hi - lo > 1) { uint32_t mid = (lo + hi) >> 1; if (views[mid].item_begin <= item) lo = mid; else hi = mid; }
        const AdjView& V = views[lo];
        const uint32_t local = item - V.item_begin;
        const uint32_t tx = (V.width + 7u) / 8u;
        const uint32_t tile = local >> 5, l = local & 31u;
        const uint32_t px = (tile % tx) * 8u + (l & 7u);
        const uint32_t py = (tile / tx) * 4u + (l >> 3);
        if (px >= V.width || py >= V.height) continue;
        const SceneView& s = scenes[V.scene];
        const DCamera cam = V.cam;
        const float light_pick_prob = 1.0f / (float)s.num_lights;
        // Forward: SoL's per-pixel loop (path_tracer.cpp:14-21).
        Rgb sum = rgb(0.0f);
        for (uint32_t k = 0; k < V.sample_count; ++k) {
            PathState ps;
            start_path(ps, cam, V.sample_index + k, px, py, V.width, V.height);
            ++n_paths;
            for (uint32_t len = 0; len < cfg.max_path_len; ++len) {
                float t = kFloatMax;
                TraversalCounters tc{0u, 0u};
                const int slot = traverse<false, false>(s, ps.org, ps.dir, ps.tmin, t, tc);
                ++n_rays;
                if (slot < 0) break;
                VertexOut vo;
                shade_vertex(s, cfg, light_pick_prob, slot, t, ps, vo);
                if (vo.has_shadow) {
                    float smax = 1.0f - cfg.ray_offset;
                    const int occ = traverse<true, false>(s, vo.sh_org, vo.sh_dir, cfg.ray_offset, smax, tc);
                    ++n_rays;
                    if (occ < 0) ps.color = ps.color + vo.pending;
                }
                if (vo.end) break;
                ps.path_len = len + 1;
            }
            sum = sum + ps.color;
        }
        const size_t plane = (size_t)V.width * V.height;
        const size_t i = (size_t)py * V.width + px;
        V.film[i] += sum.r;
        V.film[i + plane] += sum.g;
        V.film[i + 2 * plane] += sum.b;
        // Loss of this pixel and its gradient with respect to each sample's colour.
        const float inv = 1.0f / (float)V.sample_count;
        const Rgb d = rgb(sum.r * inv - V.target[i], sum.g * inv - V.target[i + plane], sum.b * inv - V.target[i + 2 * plane]);
        atomicAdd(V.loss, (double)d.r * d.r + (double)d.g * d.g + (double)d.b * d.b);
        const Rgb G = d * (2.0f * inv);
        for (uint32_t k = 0; k < V.sample_count; ++k) {
            adjoint_path(s, cfg, cam, V.sample_index + k, px, py, V.width, V.height, G, V.grad, rec, n_rays);
        }
    }
    atomicAdd(&ctr->rays, (unsigned long long)n_rays);
    atomicAdd(&ctr->paths, (unsigned long long)n_paths);
}

/// K8: L = sum (scale * film - target)^2 and dL/dfilm = 2 scale (scale * film - target).
__global__ void __launch_bounds__(256)
l2_loss(const float* __restrict__ film, const float* __restrict__ target, uint64_t n, float scale,
        float* __restrict__ dl_dfilm, double* __restrict__ loss) {
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float d = scale * film[i] - target[i];
        acc += (double)d * (double)d;
        if (dl_dfilm) dl_dfilm[i] = 2.0f * scale * d;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += part[w];
        atomicAdd(loss, sum);
    }
}

}  // namespace

int fused_blocks_per_sm() {
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fused_forward_adjoint, kAdjointBlock, 0) == cudaSuccess ? n : -1;
}

cudaError_t launch_fused_forward_adjoint(const AdjView* views, uint32_t num_views, uint32_t total_items,
                                         const SceneView* scenes, const DConfig& cfg, DeviceCounters* counters, int grid,
                                         cudaStream_t stream) {
    fused_forward_adjoint<<<grid, kAdjointBlock, 0, stream>>>(views, num_views, total_items, scenes, cfg, counters);
    return cudaGetLastError();
}

int adjoint_blocks_per_sm() {
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, prb_adjoint, kAdjointBlock, 0) == cudaSuccess ? n : -1;
}

cudaError_t launch_adjoint(const SceneView& s, const DCamera& cam, const DConfig& cfg, uint64_t sample_index,
                           uint32_t sample_count, uint32_t width, uint32_t height, const float* dl_dfilm, float* grad,
                           DeviceCounters* counters, int grid, cudaStream_t stream) {
    prb_adjoint<<<grid, kAdjointBlock, 0, stream>>>(s, cam, cfg, sample_index, sample_count, width, height, dl_dfilm,
                                                     grad, counters);
    return cudaGetLastError();
}

cudaError_t launch_l2_loss(const float* film, const float* target, uint64_t n, float scale, float* dl_dfilm,
                           double* loss, int grid, cudaStream_t stream) {
    l2_loss<<<grid, 256, 0, stream>>>(film, target, n, scale, dl_dfilm, loss);
    return cudaGetLastError();
}

}  // namespace sol_b200
