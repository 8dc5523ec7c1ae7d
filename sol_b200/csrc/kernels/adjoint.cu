// K7: path-replay adjoint of the forward render, and K8: the L2 image loss.
//
// The gradient is that of an image loss L with respect to the scene's texture
// values (constant albedos, specular colours and emissions, image texels, and
// Phong exponents; the parameter layout is described in include/sol_gpu.h),
// for the same Monte Carlo estimate the forward render computes: every path is
// replayed from its seed (Path Replay Backpropagation; Vicini, Speierer, Jakob,
// SIGGRAPH 2021), so no path is stored between kernels.  Geometry is fixed, so
// colour values change no sampled direction and no visibility; their derivative
// along each replayed path is exact, including the dependence of the Russian
// roulette probability clamp(lum(T)) on the throughput (path_tracer.cpp:100-107):
// it is the derivative of the estimate the forward computes, which central
// differences with common random numbers converge to.  (Holding the
// probability constant instead, as for an estimator of the expected image's
// derivative, was measured off by up to 4x from those differences on the
// Cornell box at path length 16, where throughputs pass many roulette tests.)
// A Phong exponent also shapes the lobe the bounce is sampled from; its
// derivative is taken with sampling detached (the sampled directions, their
// pdfs and the MIS weights held fixed, as in PRB): per vertex the BSDF value's
// derivative d f / d ns replaces f.  That estimator is unbiased for the
// derivative of the expected image, while a finite difference with common
// random numbers also follows the moving directions; the two agree in
// expectation, not per sample.
//
// One lane owns a pixel and replays its samples one after another.  A replay
// records per vertex the quantities the reverse sweep needs (at most
// kAdjointMaxDepth vertices, in registers/local memory), then sweeps from the
// last vertex to the first carrying dL/dT, and adds the texture gradients with
// warp-reduced atomics (lanes writing the same address are summed first).
#include <cuda_runtime.h>

#include <algorithm>

// The adjoint kernels are large: keeping the image-texture lookup out of line
// here (one copy instead of one per call site) measured 7 % faster for them,
// while the forward kernels keep it inline.
#ifndef SOL_TEX_OUTLINE
#define SOL_TEX_OUTLINE 1
#endif

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

/// A scalar texture value's effect on a colour: d colour / d value = d (per channel).
struct ScalarTerm {
    int tex;
    Rgb d;
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
    ScalarTerm nterm[2];        // d f / d (Phong exponent) of the light sample's BSDF value
    ScalarTerm bterm[2];        // d c / d (Phong exponent) of the bounce
    float q;                    // Russian roulette survival probability
    Vec2 uv;                    // shading texture coordinates
    uint32_t flags;
};

__device__ __forceinline__ uint32_t lane() { return threadIdx.x & 31u; }

/// Where gradients go: the caller's vector `global`, and for its first
/// `n_shared` entries (the constant textures' values, which every path of a
/// material adds into) a block-local copy in shared memory that the block adds
/// into `global` once, when it finishes.
struct GradSink {
    float* global;
    float* shared;
    uint32_t n_shared;
    float4* texels4;   // when set: image-texel gradients as (r, g, b, 0) per texel, gathered afterwards
};

/// Sums `v` over the lanes of the warp that pass the same `addr` and returns
/// the sum on the lowest such lane (rank 0), 0 elsewhere.
template <typename T>
__device__ __forceinline__ T reduce_by_address(const void* addr, T v, bool& leader) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, (unsigned long long)addr);
    const int n = __popc(peers);
    const int rank = __popc(peers & ((1u << lane()) - 1u));
    T sum = v;
    for (int s = 1; s < n; s <<= 1) {
        const int src = rank + s < n ? (int)__fns(peers, 0, rank + s + 1) : (int)lane();
        const T other = __shfl_sync(peers, sum, src);
        if (rank + s < n && (rank & (2 * s - 1)) == 0) sum += other;
    }
    leader = rank == 0;
    return sum;
}

#ifndef SOL_ADJOINT_NOINLINE
#define SOL_ADJOINT_NOINLINE 0
#endif
// SOL_ADJOINT_NOINLINE = 1 keeps the path tracer, the sweep and the texture
// scatter as single out-of-line copies (less code for the instruction cache,
// at the price of calls and of registers saved across them).  Since the
// shading code shrank, inlining them is faster: Cornell adjoint 1.53 against
// 1.91 ms.
#if SOL_ADJOINT_NOINLINE
#define SOL_ADJ_OUTLINE __noinline__
#else
#define SOL_ADJ_OUTLINE
#endif

#ifndef SOL_ADJOINT_SAMPLE_MINOR
#define SOL_ADJOINT_SAMPLE_MINOR 1
#endif

#ifndef SOL_ADJOINT_REDUCE_TEXELS
#define SOL_ADJOINT_REDUCE_TEXELS 0
#endif

/// Adds `v` into texel parameter `idx`.  Texels are spread over the image, so
/// lanes rarely meet on one; with SOL_ADJOINT_REDUCE_TEXELS the lanes that do
/// are summed first, otherwise every lane issues its own reduction.
__device__ __forceinline__ void atomic_add_texel(const GradSink& g, uint64_t idx, float v);

/// Adds `v` into parameter `idx`, after summing over the lanes that add into the same one.
__device__ __forceinline__ void atomic_add_reduced(const GradSink& g, uint64_t idx, float v) {
    bool leader;
    const float sum = reduce_by_address(g.global + idx, v, leader);
    if (!leader || sum == 0.0f) return;
    if (idx < g.n_shared) atomicAdd(g.shared + idx, sum);
    else atomicAdd(g.global + idx, sum);
}

__device__ __forceinline__ void atomic_add_texel(const GradSink& g, uint64_t idx, float v) {
#if SOL_ADJOINT_REDUCE_TEXELS
    atomic_add_reduced(g, idx, v);
#else
    if (v != 0.0f) atomicAdd(g.global + idx, v);
#endif
}

/// Adds `a` (d loss / d colour value) into the parameters of colour texture `tex` at `uv`.
__device__ SOL_ADJ_OUTLINE void scatter_color(const SceneView& s, const GradSink& grad, int tex, Vec2 uv, Rgb a) {
    if (tex < 0) return;
    const DTexture t = s.textures[tex];
    const uint64_t base = s.param_offsets[tex];
    if (t.kind == SOL_GPU_TEX_CONSTANT_COLOR) {
        atomic_add_reduced(grad, base + 0, a.r);
        atomic_add_reduced(grad, base + 1, a.g);
        atomic_add_reduced(grad, base + 2, a.b);
        return;
    }
    if (t.kind != SOL_GPU_TEX_IMAGE) return;
    // The texels and weights of image_color (src/textures.cpp:5-52), including
    // SoL's mirror mode, which folds both coordinates from u (textures.cpp:16-17).
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
    const uint64_t plane = (uint64_t)img.width * img.height;
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
    if (grad.texels4) {
        // One vector reduction per texel into the interleaved scratch
        // (img.offset is a multiple of 3: every image holds three planes).
        float4* t4 = grad.texels4 + img.offset / 3;
        for (int k = 0; k < n; ++k)
            atomicAdd(t4 + (uint64_t)ys[k] * img.width + xs[k], make_float4(ws[k] * a.r, ws[k] * a.g, ws[k] * a.b, 0.0f));
        return;
    }
    for (int k = 0; k < n; ++k) {
        const uint64_t p = base + (uint64_t)ys[k] * img.width + xs[k];
        atomic_add_texel(grad, p, ws[k] * a.r);
        atomic_add_texel(grad, p + plane, ws[k] * a.g);
        atomic_add_texel(grad, p + 2 * plane, ws[k] * a.b);
    }
}

__device__ __forceinline__ void scatter_terms(const SceneView& s, const GradSink& grad, const TexTerm* terms, Vec2 uv, Rgb a) {
    for (int k = 0; k < 2; ++k)
        if (terms[k].tex >= 0 && terms[k].scale != 0.0f) scatter_color(s, grad, terms[k].tex, uv, a * terms[k].scale);
}

/// Adds `a` (d loss / d scalar value) into scalar texture `tex` at `uv`.  A
/// colour texture read as a scalar is read through its luminance
/// (include/sol/textures.h:97-99), so its channels receive the luminance weights.
__device__ void scatter_scalar(const SceneView& s, const GradSink& grad, int tex, Vec2 uv, float a) {
    if (tex < 0 || a == 0.0f) return;
    const DTexture t = s.textures[tex];
    if (t.kind == SOL_GPU_TEX_CONSTANT) {
        atomic_add_reduced(grad, s.param_offsets[tex], a);
        return;
    }
    scatter_color(s, grad, tex, uv, rgb(0.2126f * a, 0.7152f * a, 0.0722f * a));
}

__device__ __forceinline__ void scatter_scalar_terms(const SceneView& s, const GradSink& grad, const ScalarTerm* terms, Vec2 uv,
                                                     Rgb w) {
    for (int k = 0; k < 2; ++k)
        if (terms[k].tex >= 0) {
            const Rgb p = w * terms[k].d;
            scatter_scalar(s, grad, terms[k].tex, uv, p.r + p.g + p.b);
        }
}

/// d(eval)/d(colour value) and d(eval)/d(ns) of a non-interpolating BSDF for
/// `in_dir`, weighted by `weight` (an InterpBsdf operand's share; 1 otherwise).
/// The colour texture's factor: kd / pi's 1 / pi (bsdfs.cpp:35-37), or with c
/// the reflection cosine ks's c^ns (ns + 2) / (2 pi) (bsdfs.cpp:68-70,
/// 102-104).  The Phong exponent's term: d eval / d ns = ks c^ns ((ns + 2) ln c
/// + 1) / (2 pi), zero where c = 0.  c^ns is evaluated once for both.
__device__ __forceinline__ void basic_terms(const SceneView& s, const DBsdf& b, Vec3 in_dir, const Surface& sf,
                                            Vec3 out_dir, float weight, TexTerm* et, ScalarTerm* nt) {
    *nt = ScalarTerm{-1, rgb(0.0f)};
    if (b.kind == SOL_GPU_BSDF_DIFFUSE) {
        *et = TexTerm{b.tex[0], kInvPi * weight};
        return;
    }
    if (b.kind != SOL_GPU_BSDF_PHONG) {
        *et = TexTerm{-1, 0.0f};
        return;
    }
    const float ns = tex_scalar(s, b.tex[1], sf.uv);
    const float c = reflect_cosine(in_dir, sf.normal(), out_dir);
    const float p = pow_(c, ns);
    *et = TexTerm{b.tex[0], p * (ns + 2.0f) * (0.5f * kInvPi) * weight};
    if (weight != 0.0f && c > 0.0f) {
        const float g = p * (0.5f * kInvPi) * ((ns + 2.0f) * (float)log_float_(c) + 1.0f);
        *nt = ScalarTerm{b.tex[1], tex_color(s, b.tex[0], sf.uv) * (g * weight)};
    }
}

/// basic_terms of Bsdf::eval for any kind (InterpBsdf: both operands,
/// bsdfs.cpp:185-190): colour factors into `et`, exponent terms into `nt`.
__device__ __forceinline__ void eval_terms(const SceneView& s, int id, Vec3 in_dir, const Surface& sf, Vec3 out_dir,
                                           TexTerm* et, ScalarTerm* nt) {
    const DBsdf b = s.bsdfs[id];
    et[1] = TexTerm{-1, 0.0f};
    nt[1] = ScalarTerm{-1, rgb(0.0f)};
    if (b.kind != SOL_GPU_BSDF_INTERP) {
        basic_terms(s, b, in_dir, sf, out_dir, 1.0f, &et[0], &nt[0]);
        return;
    }
    const float k = tex_scalar(s, b.tex[0], sf.uv);
    basic_terms(s, s.bsdfs[b.a], in_dir, sf, out_dir, 1.0f - k, &et[0], &nt[0]);
    basic_terms(s, s.bsdfs[b.b], in_dir, sf, out_dir, k, &et[1], &nt[1]);
}

/// Terms of a basic BSDF's sampled colour (bsdfs.cpp:39-48, 72-85, 112-119,
/// 138-165), weighted by `weight`: the specular kinds' colour texture, or
/// basic_terms for the sampled direction.
__device__ __forceinline__ void sample_terms(const SceneView& s, const DBsdf& b, const BsdfSample& bs,
                                             const Surface& sf, Vec3 out_dir, float weight, TexTerm* ct,
                                             ScalarTerm* bt) {
    if (b.kind == SOL_GPU_BSDF_MIRROR || b.kind == SOL_GPU_BSDF_GLASS) {
        const bool refracted = b.kind == SOL_GPU_BSDF_GLASS && dot(bs.in_dir, sf.face_normal) < 0.0f;
        *ct = TexTerm{refracted ? b.tex[1] : b.tex[0], 1.0f * weight};
        *bt = ScalarTerm{-1, rgb(0.0f)};
        return;
    }
    basic_terms(s, b, bs.in_dir, sf, out_dir, weight, ct, bt);
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

/// shade_vertex observer of the adjoint: fills the record of the current vertex
/// (`R`) with what the reverse sweep needs.  The light sample's surface
/// coordinates and an InterpBsdf's pick are the next draws of the sampler, read
/// from a copy of it before the forward draws them.
struct Recorder {
    VertexRec* R;
    Vec2 luv;
    int target, other;
    float k;

    __device__ __forceinline__ void begin(const PathState& ps, const Surface& sf) {
        R->flags = 0;
        R->T = ps.T;
        R->uv = sf.uv;
        R->q = 1.0f;
        R->fterm[0] = R->fterm[1] = R->cterm[0] = R->cterm[1] = TexTerm{-1, 0.0f};
        R->nterm[0] = R->nterm[1] = R->bterm[0] = R->bterm[1] = ScalarTerm{-1, rgb(0.0f)};
    }
    __device__ __forceinline__ void emission(const SceneView&, const DLight& light, Vec3 out_dir, const Surface& sf,
                                             Rgb le, float mis) {
        R->flags |= kEmit;
        R->E = le;
        R->m = mis;
        R->etex = emits(light, out_dir, sf.surf) ? light.tex : -1;
        R->euv = sf.surf;
    }
    __device__ __forceinline__ void before_light_sample(const DLight& light, const Pcg& rng) {
        Pcg peek = rng;
        float lv = peek.next_float(), lu = peek.next_float();
        if (light.kind == SOL_GPU_LIGHT_TRIANGLE && lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
        luv = vec2(lu, lv);
    }
    __device__ __forceinline__ void light_sample(const SceneView& s, int bsdf_id, const DLight& light,
                                                 const Surface& sf, Vec3 in_dir, Vec3 out_dir, Rgb intensity, Rgb f,
                                                 float scale) {
        // Counted only if the shadow ray is unoccluded: the caller sets kNee.
        R->Ls = intensity;
        R->f = f;
        R->s = scale;
        R->ltex = light.kind == SOL_GPU_LIGHT_POINT ? -1 : light.tex;
        R->luv = luv;
        eval_terms(s, bsdf_id, in_dir, sf, out_dir, R->fterm, R->nterm);
    }
    __device__ __forceinline__ void survival(float q, bool live) {
        R->q = q;
        if (live) R->flags |= kRrLive;
    }
    __device__ __forceinline__ void before_bounce(const SceneView& s, int bsdf_id, const Surface& sf, const Pcg& rng) {
        // Which operand an InterpBsdf samples is its first draw (bsdfs.cpp:192-198).
        const DBsdf b = s.bsdfs[bsdf_id];
        target = bsdf_id;
        other = -1;
        k = 1.0f;
        if (b.kind == SOL_GPU_BSDF_INTERP) {
            Pcg peek = rng;
            k = tex_scalar(s, b.tex[0], sf.uv);
            target = b.b;
            other = b.a;
            if (peek.next_float() > k) { target = b.a; other = b.b; k = 1.0f - k; }
        }
    }
    __device__ __forceinline__ void bounce(const SceneView& s, int, const Surface& sf, Vec3 out_dir,
                                           const BsdfSample& bs, float r) {
        R->flags |= kBounce;
        R->c = bs.color;
        R->r = r;
        sample_terms(s, s.bsdfs[target], bs, sf, out_dir, other >= 0 ? k : 1.0f, &R->cterm[0], &R->bterm[0]);
        if (other >= 0) basic_terms(s, s.bsdfs[other], bs.in_dir, sf, out_dir, 1.0f - k, &R->cterm[1], &R->bterm[1]);
    }
};

/// Traces one path (one pixel sample) exactly as the forward render does,
/// recording every vertex into `rec`.  Returns the number of records; `color`
/// receives the path's colour (the same bits as the forward's).
__device__ SOL_ADJ_OUTLINE int trace_recorded(const SceneView& s, const DConfig& cfg, const DCamera& cam, uint64_t frame,
                              uint32_t px, uint32_t py, uint32_t width, uint32_t height, VertexRec* rec, Rgb& color,
                              uint32_t& n_rays) {
    PathState ps;
    start_path(ps, cam, frame, px, py, width, height);
    const float light_pick_prob = 1.0f / (float)s.num_lights;
    Recorder recd;
    int K = 0;
    for (uint32_t len = 0; len < cfg.max_path_len; ++len) {
        float t = kFloatMax, hu, hv;
        TraversalCounters tc{0u, 0u};
        LocalStack stack;
        const int slot = traverse_closest_uv<false>(s, ps.org, ps.dir, ps.tmin, t, hu, hv, tc, stack);
        ++n_rays;
        if (slot < 0) break;
        // The host limits max_path_len to kAdjointMaxDepth; this guards the record array regardless.
        if (K >= kAdjointMaxDepth) { atomicOr(s.fault, kFaultPathLoop); break; }
        recd.R = rec + K++;
        VertexOut vo;
        shade_vertex(s, cfg, light_pick_prob, slot, t, ps, vo, recd, true, hu, hv);
        if (vo.has_shadow) {
            float smax = 1.0f - cfg.ray_offset;
            const int occ = traverse<true, false>(s, vo.sh_org, vo.sh_dir, cfg.ray_offset, smax, tc);
            ++n_rays;
            if (occ < 0) {
                ps.color = ps.color + vo.pending;
                recd.R->flags |= kNee;
            }
        }
        if (vo.end) break;
        ps.path_len = len + 1;
    }
    color = ps.color;
    return K;
}

/// The colour-texture and scalar-texture contributions of one vertex that are
/// looked up at the vertex's own texture coordinates (bounce and light-sample
/// BSDF terms), merged by texture so that each texture is scattered once.
struct VertexTerms {
    int ctex[4];
    Rgb ca[4];
    int stex[4];
    float sa[4];
    int nc, ns;

    __device__ __forceinline__ void color(int tex, Rgb a) {
        if (tex < 0) return;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i < nc && ctex[i] == tex) { ca[i] = ca[i] + a; return; }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i == nc) { ctex[i] = tex; ca[i] = a; }
        ++nc;
    }
    __device__ __forceinline__ void scalar(int tex, float a) {
        if (tex < 0) return;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i < ns && stex[i] == tex) { sa[i] += a; return; }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i == ns) { stex[i] = tex; sa[i] = a; }
        ++ns;
    }
    __device__ __forceinline__ void colors(const TexTerm* t, Rgb w) {
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (t[k].tex >= 0 && t[k].scale != 0.0f) color(t[k].tex, w * t[k].scale);
    }
    __device__ __forceinline__ void scalars(const ScalarTerm* t, Rgb w) {
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (t[k].tex >= 0) {
                const Rgb p = w * t[k].d;
                scalar(t[k].tex, p.r + p.g + p.b);
            }
    }
};

/// Reverse sweep over the K records of one path with G = dL/d(path colour):
/// carries a = dL/dT of the vertex after the current one from the last vertex
/// to the first and adds every texture's share into `grad`.
__device__ SOL_ADJ_OUTLINE void sweep(const SceneView& s, const VertexRec* rec, int K, Rgb G, const GradSink& grad) {
    Rgb a = rgb(0.0f);
    for (int v = K - 1; v >= 0; --v) {
        const VertexRec& R = rec[v];
        Rgb aT = rgb(0.0f);
        VertexTerms terms;
        terms.nc = terms.ns = 0;
        if (R.flags & kBounce) {
            const Rgb w = a * R.T * R.r;
            terms.colors(R.cterm, w);
            terms.scalars(R.bterm, w);
            aT = a * R.c * R.r;
            if (R.flags & kRrLive) {
                // r = cos / (pdf q) with q = clamp(lum(T)): d r / d T = -r / q * d lum / d T.
                const Rgb aTc = a * R.T * R.c;
                const float a_q = -(aTc.r + aTc.g + aTc.b) * R.r / R.q;
                aT = aT + rgb(0.2126f * a_q, 0.7152f * a_q, 0.0722f * a_q);
            }
        }
        if (R.flags & kNee) {
            aT = aT + G * R.Ls * R.f * R.s;
            const Rgb w = G * R.Ls * R.T * R.s;
            terms.colors(R.fterm, w);
            terms.scalars(R.nterm, w);
            scatter_color(s, grad, R.ltex, R.luv, G * R.T * R.f * R.s);
        }
        for (int i = 0; i < terms.nc; ++i) scatter_color(s, grad, terms.ctex[i], R.uv, terms.ca[i]);
        for (int i = 0; i < terms.ns; ++i) scatter_scalar(s, grad, terms.stex[i], R.uv, terms.sa[i]);
        if (R.flags & kEmit) {
            aT = aT + G * R.E * R.m;
            scatter_color(s, grad, R.etex, R.euv, G * R.T * R.m);
        }
        a = aT;
    }
}

/// The adjoint of one view.  Work items are (pixel, chunk of samples): for
/// small images the samples of a pixel are spread over several lanes (gradients
/// are sums, so the order in which samples are replayed does not matter).
/// Gradients of the first `n_shared` parameters (the constant textures) are
/// gathered per block in shared memory and added into `grad` at the end.
__global__ void __launch_bounds__(kAdjointBlock, kAdjointMinBlocks)
prb_adjoint(SceneView s, DCamera cam, DConfig cfg, uint64_t sample_index, uint32_t sample_count, uint32_t chunk,
            uint32_t width, uint32_t height, const float* __restrict__ dl_dfilm, float* __restrict__ grad,
            uint32_t n_shared, float4* texels4, DeviceCounters* ctr) {
    extern __shared__ float sgrad[];
    for (uint32_t i = threadIdx.x; i < n_shared; i += blockDim.x) sgrad[i] = 0.0f;
    __syncthreads();
    const GradSink sink{grad, sgrad, n_shared, texels4};
    VertexRec rec[kAdjointMaxDepth];
    const uint32_t tiles_x = (width + 7u) / 8u;
    const uint32_t total = tiles_x * ((height + 3u) / 4u) * 32u;
    const uint32_t chunks = (sample_count + chunk - 1u) / chunk;
    const uint32_t items = total * chunks;
    const size_t plane = (size_t)width * height;
    uint32_t n_rays = 0, n_paths = 0;
    while (true) {
        const unsigned mask = __activemask();
        const int leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if ((int)lane() == leader) base = atomicAdd(&ctr->next_item, (uint32_t)__popc(mask));
        const uint32_t item = __shfl_sync(mask, base, leader) + __popc(mask & ((1u << lane()) - 1u));
        if (item >= items) break;
#if SOL_ADJOINT_SAMPLE_MINOR
        // Consecutive items are consecutive sample chunks of one pixel, so a warp
        // replays few pixels with coherent primary rays.
        const uint32_t it = item / chunks, c = item - it * chunks;
#else
        const uint32_t c = item / total, it = item - c * total;
#endif
        const uint32_t tile = it >> 5, l = it & 31u;
        const uint32_t px = (tile % tiles_x) * 8u + (l & 7u);
        const uint32_t py = (tile / tiles_x) * 4u + (l >> 3);
        if (px >= width || py >= height) continue;
        const size_t i = (size_t)py * width + px;
        const Rgb G = rgb(dl_dfilm[i], dl_dfilm[i + plane], dl_dfilm[i + 2 * plane]);
        if (G.r == 0.0f && G.g == 0.0f && G.b == 0.0f) continue;
        const uint32_t k1 = min(sample_count, (c + 1u) * chunk);
        for (uint32_t k = c * chunk; k < k1; ++k) {
            Rgb color;
            const int K = trace_recorded(s, cfg, cam, sample_index + k, px, py, width, height, rec, color, n_rays);
            sweep(s, rec, K, G, sink);
            ++n_paths;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n_shared; i += blockDim.x) {
        const float v = sgrad[i];
        if (v != 0.0f) atomicAdd(grad + i, v);
    }
    atomicAdd(&ctr->rays, (unsigned long long)n_rays);
    atomicAdd(&ctr->paths, (unsigned long long)n_paths);
}

/// Forward render and adjoint of an L2 loss for many views of many scenes in
/// one persistent launch.  A work item is one warp's worth of pixels of one
/// view: the view's samples are spread over g lanes per pixel (g the smallest
/// power of two >= spp, at most 32), so a warp holds 32 / g pixels.  Each lane
/// traces its sample and records its vertices; the g colours of a pixel are
/// summed in sample order on every lane of the group (the same additions, in
/// the same order, as SoL's per-pixel loop, path_tracer.cpp:14-21), the pixel's
/// loss (sum / spp - target)^2 and gradient 2 (sum / spp - target) / spp are
/// formed (an L2 loss of a pixel depends on that pixel alone), and every lane
/// sweeps its own records backwards.  With spp <= 32 no path is traced twice;
/// with more, the samples run in rounds of 32 and are replayed after the sum.
__global__ void __launch_bounds__(kAdjointBlock, kAdjointMinBlocks)
fused_forward_adjoint(const AdjView* __restrict__ views, uint32_t num_views, uint32_t total,
                      const SceneView* __restrict__ scenes, DConfig cfg, DeviceCounters* ctr) {
    VertexRec rec[kAdjointMaxDepth];
    uint32_t n_rays = 0, n_paths = 0;
    const uint32_t ln = lane();
    while (true) {
        uint32_t w = 0;
        if (ln == 0) w = atomicAdd(&ctr->next_item, 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= total) break;
        uint32_t lo = 0, hi = num_views;
        while (hi - lo > 1) { uint32_t mid = (lo + hi) >> 1; if (views[mid].item_begin <= w) lo = mid; else hi = mid; }
        const AdjView& V = views[lo];
        const uint32_t g = V.group;                       // the same on every lane: one view per warp item
        const uint32_t q = (w - V.item_begin) * (32u / g) + ln / g;
        const uint32_t j = ln & (g - 1u);
        const uint32_t first = ln & ~(g - 1u);
        const uint32_t tx = (V.width + 7u) / 8u;
        const uint32_t tile = q >> 5, l = q & 31u;
        const uint32_t px = (tile % tx) * 8u + (l & 7u);
        const uint32_t py = (tile / tx) * 4u + (l >> 3);
        const bool valid = px < V.width && py < V.height;
        const SceneView& s = scenes[V.scene];
        const uint32_t spp = V.sample_count;
        const uint32_t rounds = (spp + g - 1u) / g;
        Rgb sum = rgb(0.0f);
        int K = 0;
        for (uint32_t r = 0; r < rounds; ++r) {
            const uint32_t k = r * g + j;
            Rgb c = rgb(0.0f);
            if (valid && k < spp) {
                K = trace_recorded(s, cfg, V.cam, V.sample_index + k, px, py, V.width, V.height, rec, c, n_rays);
                ++n_paths;
            }
            __syncwarp();
            for (uint32_t jj = 0; jj < g; ++jj) {
                const float cr = __shfl_sync(0xffffffffu, c.r, first + jj);
                const float cg = __shfl_sync(0xffffffffu, c.g, first + jj);
                const float cb = __shfl_sync(0xffffffffu, c.b, first + jj);
                if (r * g + jj < spp) sum = sum + rgb(cr, cg, cb);
            }
        }
        Rgb G = rgb(0.0f);
        if (valid) {
            const size_t plane = (size_t)V.width * V.height;
            const size_t i = (size_t)py * V.width + px;
            const float inv = 1.0f / (float)spp;
            const Rgb d = rgb(sum.r * inv - V.target[i], sum.g * inv - V.target[i + plane],
                              sum.b * inv - V.target[i + 2 * plane]);
            G = d * (2.0f * inv);
            if (j == 0) {
                V.film[i] += sum.r;
                V.film[i + plane] += sum.g;
                V.film[i + 2 * plane] += sum.b;
                bool first_lane;
                const double l2 = reduce_by_address(V.loss, (double)d.r * d.r + (double)d.g * d.g + (double)d.b * d.b,
                                                    first_lane);
                if (first_lane) atomicAdd(V.loss, l2);
            }
        }
        const GradSink sink{V.grad, nullptr, 0u, nullptr};
        if (rounds == 1) {
            if (valid && j < spp) sweep(s, rec, K, G, sink);
        } else {
            for (uint32_t r = 0; r < rounds; ++r) {
                const uint32_t k = r * g + j;
                if (!valid || k >= spp) continue;
                Rgb c;
                K = trace_recorded(s, cfg, V.cam, V.sample_index + k, px, py, V.width, V.height, rec, c, n_rays);
                sweep(s, rec, K, G, sink);
            }
        }
        __syncwarp();
    }
    atomicAdd(&ctr->rays, (unsigned long long)n_rays);
    atomicAdd(&ctr->paths, (unsigned long long)n_paths);
}

/// Adds the interleaved texel gradients (one float4 per texel of every image,
/// images in arena order) into the planar parameter vector: image k's texel i
/// channel c is parameter `first_texel_param + images[k].offset + c * w * h + i`.
__global__ void __launch_bounds__(256)
gather_texels(const float4* __restrict__ texels4, uint64_t num_texels, const DImage* __restrict__ images,
              uint32_t num_images, uint64_t first_texel_param, float* __restrict__ grad) {
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < num_texels;
         q += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = num_images;
        while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (images[mid].offset / 3 <= q) lo = mid; else hi = mid; }
        const DImage img = images[lo];
        const uint64_t i = q - img.offset / 3, plane = (uint64_t)img.width * img.height;
        if (i >= plane) continue;
        const float4 v = texels4[q];
        float* p = grad + first_texel_param + img.offset + i;
        if (v.x != 0.0f) p[0] += v.x;
        if (v.y != 0.0f) p[plane] += v.y;
        if (v.z != 0.0f) p[2 * plane] += v.z;
    }
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

int adjoint_blocks_per_sm(uint32_t n_shared) {
    int n = 0;
    const size_t smem = sizeof(float) * (size_t)n_shared;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, prb_adjoint, kAdjointBlock, smem) == cudaSuccess ? n : -1;
}

cudaError_t launch_adjoint(const SceneView& s, const DCamera& cam, const DConfig& cfg, uint64_t sample_index,
                           uint32_t sample_count, uint32_t chunk, uint32_t width, uint32_t height,
                           const float* dl_dfilm, float* grad, uint32_t n_shared, float4* texels4, uint64_t num_texels,
                           uint32_t num_images, uint64_t first_texel_param, DeviceCounters* counters, int grid,
                           cudaStream_t stream) {
    const size_t smem = sizeof(float) * (size_t)n_shared;
    if (texels4 && num_texels) {
        cudaError_t e = cudaMemsetAsync(texels4, 0, sizeof(float4) * num_texels, stream);
        if (e != cudaSuccess) return e;
    }
    prb_adjoint<<<grid, kAdjointBlock, smem, stream>>>(s, cam, cfg, sample_index, sample_count, chunk, width, height,
                                                        dl_dfilm, grad, n_shared, num_texels ? texels4 : nullptr,
                                                        counters);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !texels4 || !num_texels) return e;
    const int blocks = (int)std::min<uint64_t>((num_texels + 255) / 256, 4096);
    gather_texels<<<blocks, 256, 0, stream>>>(texels4, num_texels, s.images, num_images, first_texel_param, grad);
    return cudaGetLastError();
}

cudaError_t launch_l2_loss(const float* film, const float* target, uint64_t n, float scale, float* dl_dfilm,
                           double* loss, int grid, cudaStream_t stream) {
    l2_loss<<<grid, 256, 0, stream>>>(film, target, n, scale, dl_dfilm, loss);
    return cudaGetLastError();
}

}  // namespace sol_b200
