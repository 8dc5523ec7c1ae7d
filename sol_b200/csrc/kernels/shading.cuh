// Device statement of SoL's shading model: textures, BSDFs, lights, camera and
// hit-surface construction.  Operation order follows the cited SoL sources so
// that results agree bit for bit with the host checker; random draws happen in
// the order g++ gives SoL's argument lists (right to left: in `f(s(), s())` the
// second argument is drawn first).
#pragma once

#include "../core/layout.h"
#include "../core/math.h"
#include "../../../include/sol_gpu.h"

// SOL_SHADE_OUTLINE = 1 keeps the texture lookup, the BSDF kinds and the light
// sampling as single out-of-line copies (less code for the instruction cache,
// at the price of calls); 0 lets the compiler inline them everywhere.
#ifndef SOL_SHADE_OUTLINE
#define SOL_SHADE_OUTLINE 0
#endif
#if SOL_SHADE_OUTLINE
#define SOL_SHADE_FN inline __noinline__
#else
#define SOL_SHADE_FN inline
#endif
// SOL_TEX_OUTLINE = 1 keeps only the image-texture lookup out of line.
#ifndef SOL_TEX_OUTLINE
#define SOL_TEX_OUTLINE 0
#endif
#if SOL_TEX_OUTLINE || SOL_SHADE_OUTLINE
#define SOL_TEX_FN inline __noinline__
#else
#define SOL_TEX_FN inline
#endif

namespace sol_b200 {

// ---------------------------------------------------------------------------
// Textures (include/sol/textures.h:97-144, src/textures.cpp:5-52)
// ---------------------------------------------------------------------------

__device__ __forceinline__ Rgb texel(const SceneView& s, const DImage& img, int x, int y) {
    size_t plane = (size_t)img.width * img.height;
    size_t i = img.offset + (size_t)y * img.width + (size_t)x;
    return rgb(__ldg(s.texels + i), __ldg(s.texels + i + plane), __ldg(s.texels + i + 2 * plane));
}

__device__ __forceinline__ float fmod2_(float x) {
    // std::fmod(x, 2.0f): exact remainder with the sign of x.
    return fmodf(x, 2.0f);
}

/// ImageTexture<Filter, Border>::sample_color (src/textures.cpp:47-52).
__device__ SOL_TEX_FN Rgb image_color(const SceneView& s, const DTexture& t, Vec2 uv) {
    // Border handling (textures.cpp:5-21); Mirror uses uv[0] for both axes as SoL does.
    if (t.border == SOL_GPU_BORDER_CLAMP) {
        uv = vec2(clampf(uv.x, 0.0f, 1.0f), clampf(uv.y, 0.0f, 1.0f));
    } else if (t.border == SOL_GPU_BORDER_REPEAT) {
        uv = vec2(uv.x - floor_(uv.x), uv.y - floor_(uv.y));
    } else {
        float u = fmod2_(uv.x), v = fmod2_(uv.x);
        u = u > 1.0f ? 2.0f - u : u;
        v = v > 1.0f ? 2.0f - v : v;
        uv = vec2(u, v);
    }
    const DImage img = s.images[t.image];
    const int w = (int)img.width, h = (int)img.height;
    if (t.filter == SOL_GPU_FILTER_NEAREST) {
        // textures.cpp:23-28
        int x = clampi((int)(uv.x * (float)img.width), 0, w - 1);
        int y = clampi((int)(uv.y * (float)img.height), 0, h - 1);
        return texel(s, img, x, y);
    }
    // Bilinear, textures.cpp:30-45
    float i = uv.x * (float)(img.width - 1);
    float j = uv.y * (float)(img.height - 1);
    float fu = i - floor_(i);
    float fv = j - floor_(j);
    int x0 = clampi((int)i, 0, w - 1);
    int y0 = clampi((int)j, 0, h - 1);
    int x1 = clampi(x0 + 1, 0, w - 1);
    int y1 = clampi(y0 + 1, 0, h - 1);
    Rgb p00 = texel(s, img, x0, y0);
    Rgb p10 = texel(s, img, x1, y0);
    Rgb p01 = texel(s, img, x0, y1);
    Rgb p11 = texel(s, img, x1, y1);
    return lerp(lerp(p00, p10, fu), lerp(p01, p11, fu), fv);
}

/// ColorTexture::sample_color.
// kBasic: the scene has no image textures and no Interp BSDFs (checked on the
// host when it is uploaded), so those branches are compiled out of the kernels
// built for such scenes — a smaller instruction footprint and fewer spills.
template <bool kBasic = false>
__device__ __forceinline__ Rgb tex_color(const SceneView& s, int id, Vec2 uv) {
    const DTexture& t = s.textures[id];
    if (!kBasic && t.kind == SOL_GPU_TEX_IMAGE) return image_color(s, t, uv);
    return rgb(t.v[0], t.v[1], t.v[2]);
}

/// Texture::sample: constants return their value, colour textures their luminance.
template <bool kBasic = false>
__device__ __forceinline__ float tex_scalar(const SceneView& s, int id, Vec2 uv) {
    const DTexture& t = s.textures[id];
    if (t.kind == SOL_GPU_TEX_CONSTANT) return t.v[0];
    return luminance(tex_color<kBasic>(s, id, uv));
}

// ---------------------------------------------------------------------------
// Surface at a hit (src/triangle_mesh.cpp:78-104, include/sol/geometry.h:15-24)
// ---------------------------------------------------------------------------

struct Surface {
    Vec3 point;
    Vec2 uv;          // texture coordinates
    Vec2 surf;        // barycentric surface coordinates (u, v)
    Vec3 face_normal;
    Mat3 local;       // column 2 = shading normal
    bool front;
    __device__ __forceinline__ Vec3 normal() const { return local.c2; }
};

// ---------------------------------------------------------------------------
// BSDFs (src/bsdfs.cpp)
// ---------------------------------------------------------------------------

/// bsdfs.cpp:11-19
__device__ __forceinline__ float reflect_cosine(Vec3 in_dir, Vec3 n, Vec3 out_dir) {
    return -negative_dot(in_dir, reflect(out_dir, n));
}

/// bsdfs.cpp:21-27
__device__ __forceinline__ float fresnel_factor(float eta, float cos_i, float cos_t) {
    float rs = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    float rp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return (rs * rs + rp * rp) * 0.5f;
}

/// bsdfs.cpp:102-104
__device__ __forceinline__ Rgb phong_eval(Vec3 in_dir, const Surface& sf, Vec3 out_dir, Rgb ks, float ns) {
    return ks * pow_(reflect_cosine(in_dir, sf.normal(), out_dir), ns) * (ns + 2.0f) * (0.5f * kInvPi);
}

/// Bsdf::eval for the non-interpolating kinds (Mirror and Glass return black).
template <bool kBasic = false>
__device__ SOL_SHADE_FN Rgb bsdf_eval_basic(const SceneView& s, const DBsdf& b, Vec3 in_dir, const Surface& sf, Vec3 out_dir) {
    if (b.kind == SOL_GPU_BSDF_DIFFUSE)                       // bsdfs.cpp:35-37
        return tex_color<kBasic>(s, b.tex[0], sf.uv) * kInvPi;
    if (b.kind == SOL_GPU_BSDF_PHONG)                         // bsdfs.cpp:68-70
        return phong_eval(in_dir, sf, out_dir, tex_color<kBasic>(s, b.tex[0], sf.uv), tex_scalar<kBasic>(s, b.tex[1], sf.uv));
    return rgb(0.0f);
}

/// Bsdf::pdf for the non-interpolating kinds (Mirror and Glass return 0).
template <bool kBasic = false>
__device__ SOL_SHADE_FN float bsdf_pdf_basic(const SceneView& s, const DBsdf& b, Vec3 in_dir, const Surface& sf, Vec3 out_dir) {
    if (b.kind == SOL_GPU_BSDF_DIFFUSE)                       // bsdfs.cpp:50-52
        return cosine_hemisphere_pdf(positive_dot(in_dir, sf.normal()));
    if (b.kind == SOL_GPU_BSDF_PHONG)                         // bsdfs.cpp:87-89
        return cosine_power_hemisphere_pdf(tex_scalar<kBasic>(s, b.tex[1], sf.uv), reflect_cosine(in_dir, sf.normal(), out_dir));
    return 0.0f;
}

template <bool kBasic = false>
__device__ __forceinline__ Rgb bsdf_eval(const SceneView& s, int id, Vec3 in_dir, const Surface& sf, Vec3 out_dir) {
    const DBsdf b = s.bsdfs[id];
    if (kBasic || b.kind != SOL_GPU_BSDF_INTERP) return bsdf_eval_basic<kBasic>(s, b, in_dir, sf, out_dir);
    // bsdfs.cpp:185-190
    Rgb ea = bsdf_eval_basic<kBasic>(s, s.bsdfs[b.a], in_dir, sf, out_dir);
    Rgb eb = bsdf_eval_basic<kBasic>(s, s.bsdfs[b.b], in_dir, sf, out_dir);
    return lerp(ea, eb, tex_scalar<kBasic>(s, b.tex[0], sf.uv));
}

template <bool kBasic = false>
__device__ __forceinline__ float bsdf_pdf(const SceneView& s, int id, Vec3 in_dir, const Surface& sf, Vec3 out_dir) {
    const DBsdf b = s.bsdfs[id];
    if (kBasic || b.kind != SOL_GPU_BSDF_INTERP) return bsdf_pdf_basic<kBasic>(s, b, in_dir, sf, out_dir);
    // bsdfs.cpp:207-212
    float pa = bsdf_pdf_basic<kBasic>(s, s.bsdfs[b.a], in_dir, sf, out_dir);
    float pb = bsdf_pdf_basic<kBasic>(s, s.bsdfs[b.b], in_dir, sf, out_dir);
    return lerp(pa, pb, tex_scalar<kBasic>(s, b.tex[0], sf.uv));
}

/// bsdf_eval and (when `want_pdf`) bsdf_pdf for the same pair of directions,
/// as next-event estimation needs them: a Phong lobe's pow_(cos, exponent)
/// is evaluated once for both (the same operands give the same bits, so the
/// results are those of the two separate calls).
template <bool kBasic = false>
__device__ __forceinline__ void bsdf_eval_pdf(const SceneView& s, int id, Vec3 in_dir, const Surface& sf, Vec3 out_dir,
                                              bool want_pdf, Rgb* f, float* pdf) {
    const DBsdf b = s.bsdfs[id];
    if (!kBasic && b.kind == SOL_GPU_BSDF_INTERP) {
        *pdf = want_pdf ? bsdf_pdf<kBasic>(s, id, in_dir, sf, out_dir) : 0.0f;
        *f = bsdf_eval<kBasic>(s, id, in_dir, sf, out_dir);
        return;
    }
    if (b.kind == SOL_GPU_BSDF_PHONG) {
        // bsdfs.cpp:68-70 and 87-89
        const float ns = tex_scalar<kBasic>(s, b.tex[1], sf.uv);
        const float p = pow_(reflect_cosine(in_dir, sf.normal(), out_dir), ns);
        *pdf = want_pdf ? (ns + 1.0f) * p * (0.5f * kInvPi) : 0.0f;
        *f = tex_color<kBasic>(s, b.tex[0], sf.uv) * p * (ns + 2.0f) * (0.5f * kInvPi);
        return;
    }
    *pdf = want_pdf ? bsdf_pdf_basic<kBasic>(s, b, in_dir, sf, out_dir) : 0.0f;
    *f = bsdf_eval_basic<kBasic>(s, b, in_dir, sf, out_dir);
}

struct BsdfSample {
    Vec3 in_dir;
    float pdf;
    float cos;
    Rgb color;
};

/// Bsdf::validate_sample (include/sol/bsdfs.h:89-94).
__device__ __forceinline__ bool validate(const Surface& sf, const BsdfSample& bs, bool expect_below) {
    bool below = dot(bs.in_dir, sf.face_normal) < 0.0f;
    return bs.pdf > 0.0f && below == expect_below;
}

/// Bsdf::sample for the non-interpolating kinds.
template <bool kBasic = false>
__device__ SOL_SHADE_FN bool bsdf_sample_basic(const SceneView& s, const DBsdf& b, Pcg& rng, const Surface& sf,
                                  Vec3 out_dir, BsdfSample* out) {
    if (b.kind == SOL_GPU_BSDF_DIFFUSE) {
        // bsdfs.cpp:39-48; sample_cosine_hemisphere(sampler(), sampler()): v drawn first
        float v = rng.next_float();
        float u = rng.next_float();
        float pdf;
        Vec3 d = sample_cosine_hemisphere(u, v, &pdf);
        Vec3 ld = mul(sf.local, d);
        out->in_dir = ld;
        out->pdf = pdf;
        out->cos = d.z;
        out->color = tex_color<kBasic>(s, b.tex[0], sf.uv) * kInvPi;
        return validate(sf, *out, false);
    }
    if (b.kind == SOL_GPU_BSDF_PHONG) {
        // bsdfs.cpp:72-85
        Rgb ks = tex_color<kBasic>(s, b.tex[0], sf.uv);
        float ns = tex_scalar<kBasic>(s, b.tex[1], sf.uv);
        Mat3 basis = ortho_basis(reflect(-out_dir, sf.normal()));
        float v = rng.next_float();
        float u = rng.next_float();
        float pdf;
        Vec3 d = sample_cosine_power_hemisphere(ns, u, v, &pdf);
        Vec3 ld = mul(basis, d);
        out->in_dir = ld;
        out->pdf = pdf;
        out->cos = positive_dot(ld, sf.normal());
        out->color = phong_eval(ld, sf, out_dir, ks, ns);
        return validate(sf, *out, false);
    }
    if (b.kind == SOL_GPU_BSDF_MIRROR) {
        // bsdfs.cpp:112-119
        out->in_dir = reflect(-out_dir, sf.normal());
        out->pdf = 1.0f;
        out->cos = 1.0f;
        out->color = tex_color<kBasic>(s, b.tex[0], sf.uv);
        return validate(sf, *out, false);
    }
    if (b.kind == SOL_GPU_BSDF_GLASS) {
        // bsdfs.cpp:138-165
        float eta = tex_scalar<kBasic>(s, b.tex[2], sf.uv);
        eta = sf.front ? eta : 1.0f / eta;
        float cos_i = dot(out_dir, sf.normal());
        float cos2_t = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
        if (cos2_t > 0.0f) {
            float cos_t = sqrt_(cos2_t);
            if (rng.next_float() > fresnel_factor(eta, cos_i, cos_t)) {
                out->in_dir = (eta * cos_i - cos_t) * sf.normal() - eta * out_dir;
                out->pdf = 1.0f;
                out->cos = 1.0f;
                out->color = tex_color<kBasic>(s, b.tex[1], sf.uv) * 1.0f;
                return validate(sf, *out, true);
            }
        }
        out->in_dir = reflect(-out_dir, sf.normal());
        out->pdf = 1.0f;
        out->cos = 1.0f;
        out->color = tex_color<kBasic>(s, b.tex[0], sf.uv);
        return validate(sf, *out, false);
    }
    return false;
}

/// Bsdf::sample, including InterpBsdf (bsdfs.cpp:192-205).
template <bool kBasic = false>
__device__ inline bool bsdf_sample(const SceneView& s, int id, Pcg& rng, const Surface& sf, Vec3 out_dir, BsdfSample* out) {
    const DBsdf b = s.bsdfs[id];
    if (kBasic || b.kind != SOL_GPU_BSDF_INTERP) return bsdf_sample_basic<kBasic>(s, b, rng, sf, out_dir, out);
    float k = tex_scalar<kBasic>(s, b.tex[0], sf.uv);
    int target = b.b, other = b.a;
    if (rng.next_float() > k) { int t = target; target = other; other = t; k = 1.0f - k; }
    const DBsdf bt = s.bsdfs[target];
    if (!bsdf_sample_basic<kBasic>(s, bt, rng, sf, out_dir, out)) return false;
    const DBsdf bo = s.bsdfs[other];
    out->pdf = lerp(bsdf_pdf_basic<kBasic>(s, bo, out->in_dir, sf, out_dir), out->pdf, k);
    out->color = lerp(bsdf_eval_basic<kBasic>(s, bo, out->in_dir, sf, out_dir), out->color, k);
    return true;
}

// ---------------------------------------------------------------------------
// Lights (src/lights.cpp, src/shapes.cpp)
// ---------------------------------------------------------------------------

struct LightSample {
    Vec3 pos;
    Rgb intensity;
    float pdf_from;
    float cos;
    float inv_dist;   // 1 / |pos - from|
};

__device__ __forceinline__ Vec3 ld3(const float* p) { return vec3(p[0], p[1], p[2]); }

/// Light::sample_area for the three light kinds (lights.cpp:15-24, 64-77;
/// shapes.cpp:13-16, 20-25, 33-37).
template <bool kBasic = false>
__device__ SOL_SHADE_FN bool light_sample_area(const SceneView& s, const DLight& l, Pcg& rng, Vec3 from, LightSample* out) {
    if (l.kind == SOL_GPU_LIGHT_POINT) {
        out->pos = ld3(l.v0);
        out->intensity = rgb(l.intensity[0], l.intensity[1], l.intensity[2]);
        out->pdf_from = 1.0f;
        out->cos = 1.0f;
        out->inv_dist = 1.0f / length(out->pos - from);
        return true;
    }
    // Vec2f(sampler(), sampler()): the second coordinate is drawn first.
    float v = rng.next_float();
    float u = rng.next_float();
    Vec3 pos, n;
    if (l.kind == SOL_GPU_LIGHT_TRIANGLE) {
        if (u + v > 1.0f) { u = 1.0f - u; v = 1.0f - v; }
        pos = lerp3(ld3(l.v0), ld3(l.v1), ld3(l.v2), u, v);
        n = ld3(l.n);
    } else {
        float pdf;
        Vec3 d = sample_uniform_sphere(u, v, &pdf);
        pos = ld3(l.v0) + d * l.radius;
        n = d;
    }
    // normalize(from - pos), keeping 1/length: |pos - from| has the same bits.
    const Vec3 to_from = from - pos;
    const float inv_dist = 1.0f / length(to_from);
    Vec3 dir = to_from * inv_dist;
    float c = positive_dot(dir, n);
    if (!(c > 0.0f)) return false;
    out->pos = pos;
    out->inv_dist = inv_dist;
    out->intensity = tex_color<kBasic>(s, l.tex, vec2(u, v));
    out->pdf_from = l.inv_area;
    out->cos = c;
    return true;
}

/// Light::emission at a hit point seen along `dir` (pointing away from the
/// light), lights.cpp:38-40, 94-106.  Returns the intensity and pdf_from.
template <bool kBasic = false>
__device__ SOL_SHADE_FN void light_emission(const SceneView& s, const DLight& l, Vec3 dir, Vec2 uv, Rgb* intensity, float* pdf_from) {
    if (l.kind == SOL_GPU_LIGHT_POINT) { *intensity = rgb(0.0f); *pdf_from = 1.0f; return; }
    Vec3 n;
    if (l.kind == SOL_GPU_LIGHT_TRIANGLE) {
        n = ld3(l.n);
    } else {
        float pdf;
        n = sample_uniform_sphere(uv.x, uv.y, &pdf);
    }
    float c = dot(dir, n);
    if (c <= 0.0f) { *intensity = rgb(0.0f); *pdf_from = 1.0f; return; }
    *intensity = tex_color<kBasic>(s, l.tex, uv);
    *pdf_from = l.inv_area;
}

// ---------------------------------------------------------------------------
// Camera (src/cameras.cpp:23-25) and pixel sampling (include/sol/renderer.h:50-54)
// ---------------------------------------------------------------------------

__device__ __forceinline__ Vec3 camera_dir(const DCamera& c, float u, float v) {
    Vec3 d = vec3(c.dir[0] + u * c.right[0], c.dir[1] + u * c.right[1], c.dir[2] + u * c.right[2]);
    d = vec3(d.x + v * c.up[0], d.y + v * c.up[1], d.z + v * c.up[2]);
    return normalize(d);
}

/// Renderer::sample_pixel: the y jitter is drawn before the x jitter.
__device__ __forceinline__ Vec2 sample_pixel(Pcg& rng, uint32_t x, uint32_t y, uint32_t w, uint32_t h) {
    float ry = rng.next_float();
    float rx = rng.next_float();
    return vec2(((float)x + rx) * (2.0f / (float)w) - 1.0f,
                1.0f - ((float)y + ry) * (2.0f / (float)h));
}

/// Renderer::balance_heuristic (renderer.h:57-60).
__device__ __forceinline__ float balance_heuristic(float x, float y) { return 1.0f / (1.0f + y / x); }

}  // namespace sol_b200
