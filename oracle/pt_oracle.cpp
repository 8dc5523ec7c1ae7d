// Test infrastructure (oracle) — not part of the product.
//
// A CPU restatement of SoL's unidirectional path tracer over the flat scene of
// include/sol_gpu.h.  Each function follows the SoL source cited beside it.  The
// primitives SoL takes from the external `proto` library (vectors, sampling
// warps, ray/triangle test, PCG seeding hash) come from sol_b200/csrc/core/math.h,
// the shared restatement of proto, because proto is not vendored with SoL; all
// SoL-level logic (path loop, BSDFs, lights, textures, camera, film) is written
// out again here.  Ray casting uses this file's own median-split BVH, so hit
// identities do not depend on the product's BVH builder.
//
// Pinned by: the PCG known-answer vectors generated from SoL's samplers.h, and
// per-pixel agreement with SoL's own sources built in oracle/_ref (see tests/).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numbers>
#include <numeric>
#include <vector>

#include <omp.h>

#include "core/math.h"
#include "oracle_camera.h"
#include "sol_gpu.h"

using namespace sol_b200;

namespace {

Vec3 ld3(const float* p) { return vec3(p[0], p[1], p[2]); }

// ---------------------------------------------------------------------------
// Sampler: PcgGenerator + uniform_real_distribution<float> (include/sol/samplers.h:20-65)
// ---------------------------------------------------------------------------
struct Sampler {
    uint64_t state;
    explicit Sampler(uint64_t init) {            // samplers.h:30-35
        state = 0;
        gen();
        state += init;
        gen();
    }
    uint32_t gen() {                             // samplers.h:37-43
        uint64_t old = state;
        state = old * UINT64_C(6364136223846793005) + 1;
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((-rot) & 31u));
    }
    float operator()() {                         // samplers.h:57: one 32-bit draw scaled by 2^-32, kept below 1
        float f = (float)gen() * 0x1p-32f;
        return f >= 1.0f ? std::nextafter(1.0f, 0.0f) : f;
    }
};

// ---------------------------------------------------------------------------
// Scene tables
// ---------------------------------------------------------------------------
struct Scene {
    const SolGpuSceneDesc* d;
    std::vector<Vec3> light_normal;
    std::vector<float> light_inv_area;
    // own BVH over the mesh
    struct Node { float lo[3], hi[3]; uint32_t left, first, count; };
    std::vector<Node> nodes;
    std::vector<uint32_t> order;
};

struct Hit {
    uint32_t tri;
    float t, u, v;
};

// Median-split BVH (largest centroid extent), leaves of up to 4 triangles.
void build_bvh(Scene& s) {
    const SolGpuSceneDesc& d = *s.d;
    const uint32_t n = d.num_triangles;
    s.order.resize(n);
    std::iota(s.order.begin(), s.order.end(), 0u);
    std::vector<float> cen(3 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k)
            cen[3 * i + k] = (d.vertices[3 * d.indices[3 * i] + k] + d.vertices[3 * d.indices[3 * i + 1] + k] +
                              d.vertices[3 * d.indices[3 * i + 2] + k]) / 3.0f;
    if (n == 0) return;
    struct Task { uint32_t node, begin, end; };
    s.nodes.push_back({});
    std::vector<Task> stack{{0, 0, n}};
    while (!stack.empty()) {
        Task t = stack.back(); stack.pop_back();
        Scene::Node nd{};
        float clo[3], chi[3];
        for (int k = 0; k < 3; ++k) { nd.lo[k] = clo[k] = INFINITY; nd.hi[k] = chi[k] = -INFINITY; }
        for (uint32_t i = t.begin; i < t.end; ++i) {
            uint32_t p = s.order[i];
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    float x = d.vertices[3 * d.indices[3 * p + j] + k];
                    nd.lo[k] = std::min(nd.lo[k], x); nd.hi[k] = std::max(nd.hi[k], x);
                }
            for (int k = 0; k < 3; ++k) { clo[k] = std::min(clo[k], cen[3 * p + k]); chi[k] = std::max(chi[k], cen[3 * p + k]); }
        }
        if (t.end - t.begin <= 4) {
            nd.first = t.begin; nd.count = t.end - t.begin;
            s.nodes[t.node] = nd;
            continue;
        }
        int axis = 0;
        for (int k = 1; k < 3; ++k) if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
        uint32_t mid = (t.begin + t.end) / 2;
        std::nth_element(s.order.begin() + t.begin, s.order.begin() + mid, s.order.begin() + t.end,
                         [&](uint32_t a, uint32_t b) { return cen[3 * a + axis] < cen[3 * b + axis] || (cen[3 * a + axis] == cen[3 * b + axis] && a < b); });
        nd.left = (uint32_t)s.nodes.size();
        nd.count = 0;
        s.nodes[t.node] = nd;
        s.nodes.push_back({});
        s.nodes.push_back({});
        stack.push_back({nd.left + 1, mid, t.end});
        stack.push_back({nd.left, t.begin, mid});
    }
}

bool box_hit(const Scene::Node& n, Vec3 org, Vec3 idir, float tmin, float tmax) {
    float tn = tmin, tf = tmax;
    for (int k = 0; k < 3; ++k) {
        float o = comp(org, k), id = comp(idir, k);
        float a = (n.lo[k] - o) * id, b = (n.hi[k] - o) * id;
        tn = std::max(tn, std::min(a, b));
        tf = std::min(tf, std::max(a, b));
    }
    return tn <= tf * kSlabWiden;
}

Vec3 vert(const SolGpuSceneDesc& d, uint32_t tri, int j) { return ld3(d.vertices + 3 * d.indices[3 * tri + j]); }

/// Closest hit: the smallest t strictly inside (tmin, tmax); among equal t the
/// lowest triangle index.  `any` stops at the first hit.
bool cast(const Scene& s, Vec3 org, Vec3 dir, float tmin, float tmax, bool any, Hit* out) {
    if (s.nodes.empty()) return false;
    const SolGpuSceneDesc& d = *s.d;
    RayShear rs = make_shear(org, dir);
    Vec3 idir = safe_inverse(dir);
    bool found = false;
    Hit best{0, tmax, 0, 0};
    uint32_t stack[256];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const Scene::Node& n = s.nodes[stack[--sp]];
        if (!box_hit(n, org, idir, tmin, best.t)) continue;
        if (n.count == 0) { stack[sp++] = n.left; stack[sp++] = n.left + 1; continue; }
        for (uint32_t i = n.first; i < n.first + n.count; ++i) {
            uint32_t p = s.order[i];
            float t, u, v;
            // Accept t == best.t only for a lower index, so ties resolve independently of traversal order.
            if (!intersect_triangle(rs, vert(d, p, 0), vert(d, p, 1), vert(d, p, 2), tmin, found ? std::nextafter(best.t, INFINITY) : best.t, &t, &u, &v))
                continue;
            if (found && (t > best.t || (t == best.t && p > best.tri))) continue;
            best = Hit{p, t, u, v};
            found = true;
            if (any) { *out = best; return true; }
        }
    }
    if (found) *out = best;
    return found;
}

// ---------------------------------------------------------------------------
// Textures (include/sol/textures.h:97-144, src/textures.cpp)
// ---------------------------------------------------------------------------
Rgb rgb_at(const SolGpuImage& im, size_t x, size_t y) {     // image.h:48-52
    size_t i = y * im.width + x;
    return rgb(im.channels[0][i], im.channels[1][i], im.channels[2][i]);
}

Rgb sample_color(const Scene& s, int32_t id, Vec2 uv) {
    const SolGpuTexture& t = s.d->textures[id];
    if (t.type == SOL_GPU_TEX_CONSTANT_COLOR) return rgb(t.value[0], t.value[1], t.value[2]);
    const SolGpuImage& im = s.d->images[t.image];
    float u, v;
    if (t.border == SOL_GPU_BORDER_CLAMP) {                 // textures.cpp:5-7
        u = std::clamp(uv.x, 0.0f, 1.0f); v = std::clamp(uv.y, 0.0f, 1.0f);
    } else if (t.border == SOL_GPU_BORDER_REPEAT) {         // textures.cpp:9-13
        u = uv.x - std::floor(uv.x); v = uv.y - std::floor(uv.y);
    } else {                                                // textures.cpp:15-21 (v from uv[0], as in SoL)
        u = std::fmod(uv.x, 2.0f); v = std::fmod(uv.x, 2.0f);
        u = u > 1.0f ? 2.0f - u : u;
        v = v > 1.0f ? 2.0f - v : v;
    }
    const int w = (int)im.width, h = (int)im.height;
    auto clampi_ = [](int x, int a, int b) { return x < a ? a : (x > b ? b : x); };
    if (t.filter == SOL_GPU_FILTER_NEAREST) {               // textures.cpp:23-28
        int x = clampi_((int)(u * (float)im.width), 0, w - 1);
        int y = clampi_((int)(v * (float)im.height), 0, h - 1);
        return rgb_at(im, x, y);
    }
    float i = u * (float)(im.width - 1);                    // textures.cpp:30-45
    float j = v * (float)(im.height - 1);
    float fu = i - std::floor(i), fv = j - std::floor(j);
    int x0 = clampi_((int)i, 0, w - 1), y0 = clampi_((int)j, 0, h - 1);
    int x1 = clampi_(x0 + 1, 0, w - 1), y1 = clampi_(y0 + 1, 0, h - 1);
    Rgb p00 = rgb_at(im, x0, y0), p10 = rgb_at(im, x1, y0), p01 = rgb_at(im, x0, y1), p11 = rgb_at(im, x1, y1);
    return lerp(lerp(p00, p10, fu), lerp(p01, p11, fu), fv);
}

float sample_scalar(const Scene& s, int32_t id, Vec2 uv) {
    const SolGpuTexture& t = s.d->textures[id];
    if (t.type == SOL_GPU_TEX_CONSTANT) return t.value[0];  // textures.h:111
    return luminance(sample_color(s, id, uv));              // textures.h:97-99
}

// ---------------------------------------------------------------------------
// Surface info (src/triangle_mesh.cpp:78-104)
// ---------------------------------------------------------------------------
struct SurfaceInfo {
    bool is_front_side;
    Vec3 point;
    Vec2 tex_coords, surf_coords;
    Vec3 face_normal;
    Mat3 local;
    Vec3 normal() const { return local.c2; }
};

SurfaceInfo surface(const Scene& s, const Hit& h, Vec3 org, Vec3 dir) {
    const SolGpuSceneDesc& d = *s.d;
    uint32_t i0 = d.indices[3 * h.tri], i1 = d.indices[3 * h.tri + 1], i2 = d.indices[3 * h.tri + 2];
    Vec3 face_normal = triangle_normal(ld3(d.vertices + 3 * i0), ld3(d.vertices + 3 * i1), ld3(d.vertices + 3 * i2));
    Vec3 normal = lerp3(ld3(d.normals + 3 * i0), ld3(d.normals + 3 * i1), ld3(d.normals + 3 * i2), h.u, h.v);
    Vec2 tc = lerp3(vec2(d.tex_coords[2 * i0], d.tex_coords[2 * i0 + 1]), vec2(d.tex_coords[2 * i1], d.tex_coords[2 * i1 + 1]),
                    vec2(d.tex_coords[2 * i2], d.tex_coords[2 * i2 + 1]), h.u, h.v);
    SurfaceInfo si;
    si.is_front_side = dot(face_normal, dir) < 0.0f;
    if (!si.is_front_side) { face_normal = -face_normal; normal = -normal; }
    si.point = org + dir * h.t;
    si.tex_coords = tc;
    si.surf_coords = vec2(h.u, h.v);
    si.face_normal = face_normal;
    si.local = ortho_basis(normalize(normal));
    return si;
}

// ---------------------------------------------------------------------------
// BSDFs (src/bsdfs.cpp, include/sol/bsdfs.h)
// ---------------------------------------------------------------------------
struct BsdfSample { Vec3 in_dir; float pdf, cos; Rgb color; };

float reflect_cosine(Vec3 in_dir, Vec3 n, Vec3 out_dir) { return -negative_dot(in_dir, reflect(out_dir, n)); }   // bsdfs.cpp:11-19
float fresnel_factor(float eta, float cos_i, float cos_t) {                                                       // bsdfs.cpp:21-27
    float rs = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    float rp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return (rs * rs + rp * rp) * 0.5f;
}
bool validate_sample(const SurfaceInfo& si, const BsdfSample& bs, bool expect_below, BsdfSample* out) {           // bsdfs.h:89-94
    bool is_below = dot(bs.in_dir, si.face_normal) < 0.0f;
    if (bs.pdf > 0.0f && is_below == expect_below) { *out = bs; return true; }
    return false;
}
int bsdf_type(const Scene& s, int32_t id) {
    const SolGpuBsdf& b = s.d->bsdfs[id];
    switch (b.type) {
        case SOL_GPU_BSDF_DIFFUSE: return 0;
        case SOL_GPU_BSDF_PHONG: return 1;
        case SOL_GPU_BSDF_MIRROR:
        case SOL_GPU_BSDF_GLASS: return 2;
        default: {                                                                                                 // bsdfs.cpp:226-230
            int a = bsdf_type(s, b.a), c = bsdf_type(s, b.b);
            return (a == 0 || c == 0) ? 0 : (a == 1 || c == 1) ? 1 : 2;
        }
    }
}
Rgb phong_eval(Vec3 in_dir, const SurfaceInfo& si, Vec3 out_dir, Rgb ks, float ns) {                              // bsdfs.cpp:102-104
    return ks * pow_(reflect_cosine(in_dir, si.normal(), out_dir), ns) * (ns + 2.0f) * (0.5f * std::numbers::inv_pi_v<float>);
}
Rgb bsdf_eval(const Scene& s, int32_t id, Vec3 in_dir, const SurfaceInfo& si, Vec3 out_dir) {
    const SolGpuBsdf& b = s.d->bsdfs[id];
    switch (b.type) {
        case SOL_GPU_BSDF_DIFFUSE: return sample_color(s, b.tex[0], si.tex_coords) * std::numbers::inv_pi_v<float>;       // bsdfs.cpp:35-37
        case SOL_GPU_BSDF_PHONG: return phong_eval(in_dir, si, out_dir, sample_color(s, b.tex[0], si.tex_coords),         // bsdfs.cpp:68-70
                                                   sample_scalar(s, b.tex[1], si.tex_coords));
        case SOL_GPU_BSDF_INTERP: return lerp(bsdf_eval(s, b.a, in_dir, si, out_dir), bsdf_eval(s, b.b, in_dir, si, out_dir), // bsdfs.cpp:185-190
                                              sample_scalar(s, b.tex[0], si.tex_coords));
        default: return rgb(0.0f);                                                                                         // bsdfs.h:52-58
    }
}
float bsdf_pdf(const Scene& s, int32_t id, Vec3 in_dir, const SurfaceInfo& si, Vec3 out_dir) {
    const SolGpuBsdf& b = s.d->bsdfs[id];
    switch (b.type) {
        case SOL_GPU_BSDF_DIFFUSE: return cosine_hemisphere_pdf(positive_dot(in_dir, si.normal()));                   // bsdfs.cpp:50-52
        case SOL_GPU_BSDF_PHONG: return cosine_power_hemisphere_pdf(sample_scalar(s, b.tex[1], si.tex_coords),       // bsdfs.cpp:87-89
                                                                    reflect_cosine(in_dir, si.normal(), out_dir));
        case SOL_GPU_BSDF_INTERP: return lerp(bsdf_pdf(s, b.a, in_dir, si, out_dir), bsdf_pdf(s, b.b, in_dir, si, out_dir),  // bsdfs.cpp:207-212
                                              sample_scalar(s, b.tex[0], si.tex_coords));
        default: return 0.0f;
    }
}
bool bsdf_sample(const Scene& s, int32_t id, Sampler& sampler, const SurfaceInfo& si, Vec3 out_dir, BsdfSample* out) {
    const SolGpuBsdf& b = s.d->bsdfs[id];
    switch (b.type) {
        case SOL_GPU_BSDF_DIFFUSE: {                          // bsdfs.cpp:39-48 (arguments drawn right to left)
            float v = sampler();
            float u = sampler();
            float pdf;
            Vec3 in_dir = sample_cosine_hemisphere(u, v, &pdf);
            Vec3 local_in_dir = mul(si.local, in_dir);
            return validate_sample(si, {local_in_dir, pdf, in_dir.z, bsdf_eval(s, id, local_in_dir, si, out_dir)}, false, out);
        }
        case SOL_GPU_BSDF_PHONG: {                            // bsdfs.cpp:72-85
            Rgb ks = sample_color(s, b.tex[0], si.tex_coords);
            float ns = sample_scalar(s, b.tex[1], si.tex_coords);
            Mat3 basis = ortho_basis(reflect(-out_dir, si.normal()));
            float v = sampler();
            float u = sampler();
            float pdf;
            Vec3 in_dir = sample_cosine_power_hemisphere(ns, u, v, &pdf);
            Vec3 local_in_dir = mul(basis, in_dir);
            float c = positive_dot(local_in_dir, si.normal());
            return validate_sample(si, {local_in_dir, pdf, c, phong_eval(local_in_dir, si, out_dir, ks, ns)}, false, out);
        }
        case SOL_GPU_BSDF_MIRROR:                             // bsdfs.cpp:112-119
            return validate_sample(si, {reflect(-out_dir, si.normal()), 1.0f, 1.0f, sample_color(s, b.tex[0], si.tex_coords)}, false, out);
        case SOL_GPU_BSDF_GLASS: {                            // bsdfs.cpp:138-165
            float eta = sample_scalar(s, b.tex[2], si.tex_coords);
            eta = si.is_front_side ? eta : 1.0f / eta;
            float cos_i = dot(out_dir, si.normal());
            float cos2_t = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
            if (cos2_t > 0.0f) {
                float cos_t = std::sqrt(cos2_t);
                if (sampler() > fresnel_factor(eta, cos_i, cos_t)) {
                    Vec3 refract_dir = (eta * cos_i - cos_t) * si.normal() - eta * out_dir;
                    return validate_sample(si, {refract_dir, 1.0f, 1.0f, sample_color(s, b.tex[1], si.tex_coords) * 1.0f}, true, out);
                }
            }
            return validate_sample(si, {reflect(-out_dir, si.normal()), 1.0f, 1.0f, sample_color(s, b.tex[0], si.tex_coords)}, false, out);
        }
        default: {                                            // bsdfs.cpp:192-205
            float k = sample_scalar(s, b.tex[0], si.tex_coords);
            int32_t target = b.b, other = b.a;
            if (sampler() > k) { std::swap(target, other); k = 1.0f - k; }
            BsdfSample bs;
            if (!bsdf_sample(s, target, sampler, si, out_dir, &bs)) return false;
            bs.pdf = lerp(bsdf_pdf(s, other, bs.in_dir, si, out_dir), bs.pdf, k);
            bs.color = lerp(bsdf_eval(s, other, bs.in_dir, si, out_dir), bs.color, k);
            *out = bs;
            return true;
        }
    }
}

// ---------------------------------------------------------------------------
// Lights (src/lights.cpp, src/shapes.cpp)
// ---------------------------------------------------------------------------
struct LightAreaSample { Vec3 pos; Rgb intensity; float pdf_from, cos; };

bool sample_area(const Scene& s, uint32_t li, Sampler& sampler, Vec3 from, LightAreaSample* out) {
    const SolGpuLight& l = s.d->lights[li];
    if (l.type == SOL_GPU_LIGHT_POINT) {                      // lights.cpp:15-24
        *out = {ld3(l.v0), rgb(l.intensity[0], l.intensity[1], l.intensity[2]), 1.0f, 1.0f};
        return true;
    }
    float v = sampler();                                      // shapes.cpp:13-16 (arguments drawn right to left)
    float u = sampler();
    Vec3 pos, normal;
    if (l.type == SOL_GPU_LIGHT_TRIANGLE) {                   // shapes.cpp:20-25
        if (u + v > 1.0f) { u = 1.0f - u; v = 1.0f - v; }
        pos = lerp3(ld3(l.v0), ld3(l.v1), ld3(l.v2), u, v);
        normal = s.light_normal[li];
    } else {                                                  // shapes.cpp:33-37
        float pdf;
        Vec3 dir = sample_uniform_sphere(u, v, &pdf);
        pos = ld3(l.v0) + dir * l.v1[0];
        normal = dir;
    }
    Vec3 dir = normalize(from - pos);                         // lights.cpp:64-77
    float c = positive_dot(dir, normal);
    if (!(c > 0.0f)) return false;
    *out = {pos, sample_color(s, l.intensity_tex, vec2(u, v)), s.light_inv_area[li], c};
    return true;
}

void emission(const Scene& s, uint32_t li, Vec3 dir, Vec2 uv, Rgb* intensity, float* pdf_from) {
    const SolGpuLight& l = s.d->lights[li];
    if (l.type == SOL_GPU_LIGHT_POINT) { *intensity = rgb(0.0f); *pdf_from = 1.0f; return; }   // lights.cpp:38-40
    Vec3 normal;                                              // lights.cpp:94-106
    if (l.type == SOL_GPU_LIGHT_TRIANGLE) normal = s.light_normal[li];
    else { float pdf; normal = sample_uniform_sphere(uv.x, uv.y, &pdf); }
    float c = dot(dir, normal);
    if (c <= 0.0f) { *intensity = rgb(0.0f); *pdf_from = 1.0f; return; }
    *intensity = sample_color(s, l.intensity_tex, uv);
    *pdf_from = s.light_inv_area[li];
}

// ---------------------------------------------------------------------------
// Path tracer (src/algorithms/path_tracer.cpp, include/sol/renderer.h)
// ---------------------------------------------------------------------------
struct Camera { Vec3 eye, dir, right, up; };

Camera make_camera(const OracleCamera& c) {                  // cameras.cpp:5-21
    Camera cam;
    cam.eye = ld3(c.eye);
    cam.dir = normalize(ld3(c.dir));
    cam.right = normalize(cross(ld3(c.dir), ld3(c.up)));
    cam.up = cross(cam.right, cam.dir);
    float w = std::tan(c.fov * std::numbers::pi_v<float> / 360.0f);
    float h = w / c.aspect;
    cam.right = cam.right * w;
    cam.up = cam.up * h;
    return cam;
}

/// Optional record of the rays one path traces (for debugging divergences).
struct PathLog {
    SolGpuRay* rays;     // extension and shadow rays in trace order
    int32_t* kinds;      // 0 = extension, 1 = shadow
    SolGpuHit* hits;     // result of each ray (shadow: tri >= 0 when occluded)
    uint32_t cap, n;
    void add(int kind, Vec3 o, Vec3 d, float t0, float t1, bool hit, const Hit& h) {
        if (!rays || n >= cap) { ++n; return; }
        rays[n] = SolGpuRay{{o.x, o.y, o.z}, t0, {d.x, d.y, d.z}, t1};
        kinds[n] = kind;
        hits[n] = hit ? SolGpuHit{(int32_t)h.tri, h.t, h.u, h.v} : SolGpuHit{-1, 0.0f, 0.0f, 0.0f};
        ++n;
    }
};

Rgb trace_path(const Scene& s, const SolGpuConfig& cfg, Sampler& sampler, Vec3 org, Vec3 dir, float tmin,
               PathLog* log = nullptr) {
    const uint32_t nl = s.d->num_lights;
    const float light_pick_prob = 1.0f / (float)nl;
    float pdf_prev_bounce = 0.0f;
    Rgb throughput = rgb(1.0f);
    Rgb color = rgb(0.0f);
    for (uint32_t path_len = 0; path_len < cfg.max_path_len; path_len++) {
        Hit hit;
        const bool found = cast(s, org, dir, tmin, kFloatMax, false, &hit);
        if (log) log->add(0, org, dir, tmin, kFloatMax, found, hit);
        if (!found) break;
        const float tmax = hit.t;
        SurfaceInfo si = surface(s, hit, org, dir);
        int32_t light = s.d->tri_light[hit.tri];
        int32_t bsdf = s.d->tri_bsdf[hit.tri];
        Vec3 out_dir = -dir;

        if (light >= 0 && si.is_front_side) {                // path_tracer.cpp:48-60
            float pdf_prev_bounce_area = pdf_prev_bounce * dot(out_dir, si.normal()) / (tmax * tmax);
            Rgb intensity; float pdf_from;
            emission(s, (uint32_t)light, out_dir, si.surf_coords, &intensity, &pdf_from);
            float mis_weight = pdf_prev_bounce != 0.0f ? 1.0f / (1.0f + (pdf_from * light_pick_prob) / pdf_prev_bounce_area) : 1.0f;
            color = color + throughput * intensity * mis_weight;
        }
        if (bsdf < 0) break;                                  // :62-63

        bool skip_nee = bsdf_type(s, bsdf) == 2;               // :66-97
        if (!skip_nee && nl > 0) {
            uint32_t li = std::min((uint32_t)(sampler() * (float)nl), nl - 1);   // :25-29
            const SolGpuLight& l = s.d->lights[li];
            LightAreaSample ls;
            if (sample_area(s, li, sampler, si.point, &ls)) {
                Vec3 in_dir = ls.pos - si.point;
                float cos_surf = dot(in_dir, si.normal());
                Hit occ;
                const bool occluded = cast(s, si.point, ls.pos - si.point, cfg.ray_offset, 1.0f - cfg.ray_offset, true, &occ);
                if (log) log->add(1, si.point, ls.pos - si.point, cfg.ray_offset, 1.0f - cfg.ray_offset, occluded, occ);
                if (!occluded) {
                    float inv_light_dist = 1.0f / length(in_dir);
                    cos_surf *= inv_light_dist;
                    in_dir = in_dir * inv_light_dist;
                    bool has_area = l.type != SOL_GPU_LIGHT_POINT;
                    float pdf_bounce = has_area ? bsdf_pdf(s, bsdf, in_dir, si, out_dir) : 0.0f;
                    float pdf_light = ls.pdf_from * light_pick_prob;
                    float geom_term = ls.cos * inv_light_dist * inv_light_dist;
                    float mis_weight = has_area ? 1.0f / (1.0f + (pdf_bounce * geom_term) / pdf_light) : 1.0f;
                    color = color + ls.intensity * throughput * bsdf_eval(s, bsdf, in_dir, si, out_dir) *
                                        (geom_term * cos_surf * mis_weight / pdf_light);
                }
            }
        }
        float survival_prob = 1.0f;                           // :99-108
        if (path_len >= cfg.min_rr_path_len) {
            float lum = luminance(throughput);
            survival_prob = lum < cfg.min_survival_prob ? cfg.min_survival_prob : (lum > cfg.max_survival_prob ? cfg.max_survival_prob : lum);
            if (sampler() >= survival_prob) break;
        }
        BsdfSample bs;                                         // :110-117
        if (!bsdf_sample(s, bsdf, sampler, si, out_dir, &bs)) break;
        throughput = throughput * (bs.color * (bs.cos / (bs.pdf * survival_prob)));
        org = si.point;
        dir = bs.in_dir;
        tmin = cfg.ray_offset;
        pdf_prev_bounce = skip_nee ? 0.0f : bs.pdf;
    }
    return color;
}

Scene prepare(const SolGpuSceneDesc* d) {
    Scene s;
    s.d = d;
    for (uint32_t i = 0; i < d->num_lights; ++i) {
        const SolGpuLight& l = d->lights[i];
        if (l.type == SOL_GPU_LIGHT_TRIANGLE) {               // shapes.h:53-55
            s.light_normal.push_back(triangle_normal(ld3(l.v0), ld3(l.v1), ld3(l.v2)));
            s.light_inv_area.push_back(1.0f / triangle_area(ld3(l.v0), ld3(l.v1), ld3(l.v2)));
        } else {
            s.light_normal.push_back(vec3(0.0f));
            s.light_inv_area.push_back(l.type == SOL_GPU_LIGHT_SPHERE ? 1.0f / sphere_area(l.v1[0]) : 1.0f);
        }
    }
    build_bvh(s);
    return s;
}

}  // namespace

extern "C" {

/// PathTracer::render (path_tracer.cpp:9-23) into planar films, `+=` per pixel.
int oracle_render(const SolGpuSceneDesc* d, const OracleCamera* c, const SolGpuConfig* cfg,
                  uint64_t sample_index, uint32_t sample_count, uint32_t w, uint32_t h,
                  float* r, float* g, float* b, int threads) {
    Scene s = prepare(d);
    Camera cam = make_camera(*c);
    if (threads > 0) omp_set_num_threads(threads);
    #pragma omp parallel for schedule(dynamic, 1)
    for (long y = 0; y < (long)h; ++y) {
        for (uint32_t x = 0; x < w; ++x) {
            Rgb color = rgb(0.0f);
            for (uint32_t i = 0; i < sample_count; ++i) {
                Sampler sampler(pixel_seed(sample_index + i, x, (uint64_t)y));   // renderer.h:44-46
                float ry = sampler();                                            // renderer.h:50-54, y drawn first
                float rx = sampler();
                float u = ((float)x + rx) * (2.0f / (float)w) - 1.0f;
                float v = 1.0f - ((float)y + ry) * (2.0f / (float)h);
                Vec3 dir = normalize(cam.dir + u * cam.right + v * cam.up);      // cameras.cpp:23-25
                color = color + trace_path(s, *cfg, sampler, cam.eye, dir, 0.0f);
            }
            size_t i = (size_t)y * w + x;                                        // image.h:54-60
            r[i] += color.r; g[i] += color.g; b[i] += color.b;
        }
    }
    return 0;
}

/// Closest-hit (any_hit == 0) or any-hit queries: hits[i].tri is the caller's
/// triangle index (-1 for a miss); closest hits also carry t, u, v.
int oracle_trace(const SolGpuSceneDesc* d, const SolGpuRay* rays, uint32_t count, int any_hit, SolGpuHit* hits) {
    Scene s = prepare(d);
    #pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < (long)count; ++i) {
        const SolGpuRay& q = rays[i];
        Hit h;
        SolGpuHit o{-1, 0.0f, 0.0f, 0.0f};
        if (cast(s, ld3(q.org), ld3(q.dir), q.tmin, q.tmax, any_hit != 0, &h)) {
            o.tri = (int32_t)h.tri;
            if (!any_hit) { o.t = h.t; o.u = h.u; o.v = h.v; }
        }
        hits[i] = o;
    }
    return 0;
}

/// Replays one (pixel, sample) path and records its rays, hits and colour.
/// Returns the number of rays the path traced (records beyond `cap` are dropped).
uint32_t oracle_debug_path(const SolGpuSceneDesc* d, const OracleCamera* c, const SolGpuConfig* cfg, uint64_t frame,
                           uint32_t x, uint32_t y, uint32_t w, uint32_t h, SolGpuRay* rays, int32_t* kinds,
                           SolGpuHit* hits, uint32_t cap, float* color) {
    Scene s = prepare(d);
    Camera cam = make_camera(*c);
    Sampler sampler(pixel_seed(frame, x, (uint64_t)y));
    float ry = sampler();
    float rx = sampler();
    float u = ((float)x + rx) * (2.0f / (float)w) - 1.0f;
    float v = 1.0f - ((float)y + ry) * (2.0f / (float)h);
    Vec3 dir = normalize(cam.dir + u * cam.right + v * cam.up);
    PathLog log{rays, kinds, hits, cap, 0};
    Rgb col = trace_path(s, *cfg, sampler, cam.eye, dir, 0.0f, &log);
    color[0] = col.r; color[1] = col.g; color[2] = col.b;
    return log.n;
}

/// `n` consecutive draws of PcgSampler(seed) in call order.
void oracle_pcg_floats(uint64_t seed, uint32_t n, float* out) {
    Sampler s(seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = s();
}

/// The shared pow_ (core/math.h) on the host, element-wise over n pairs.
void oracle_pow(const float* x, const float* y, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) out[i] = pow_(x[i], y[i]);
}

/// Renderer::pixel_seed for a batch of (frame, x, y) triples.
void oracle_pixel_seeds(const uint64_t* fxy, uint32_t n, uint32_t* out) {
    for (uint32_t i = 0; i < n; ++i) out[i] = pixel_seed(fxy[3 * i], fxy[3 * i + 1], fxy[3 * i + 2]);
}

}  // extern "C"
