// Per-path state and the per-vertex step of PathTracer::trace_path
// (src/algorithms/path_tracer.cpp:31-120), shared by the megakernel and the
// wavefront stages so that both schedules compute identical bits.
#pragma once

#include "../core/layout.h"
#include "../core/math.h"
#include "shading.cuh"
#include "traverse.cuh"

namespace sol_b200 {

/// Everything trace_path keeps between iterations, plus the ray to trace next.
struct PathState {
    Pcg rng;
    Vec3 org;
    Vec3 dir;
    float tmin;
    Rgb T;          // throughput
    Rgb color;      // radiance gathered so far
    float pdf_prev; // pdf_prev_bounce
    uint32_t path_len;
};

/// Shadow ray and contribution produced by one vertex, and whether the path ends.
struct VertexOut {
    bool end;
    bool has_shadow;
    Vec3 sh_org;
    Vec3 sh_dir;
    Rgb pending;
};

/// PathTracer::render's per-sample set-up (path_tracer.cpp:16-18): seeded
/// sampler, jittered camera ray, empty path.
__device__ __forceinline__ void start_path(PathState& ps, const DCamera& cam, uint64_t frame, uint32_t px, uint32_t py,
                                           uint32_t width, uint32_t height) {
    ps.rng = make_pcg(pixel_seed(frame, px, py));
    Vec2 uv = sample_pixel(ps.rng, px, py, width, height);
    ps.org = vec3(cam.eye[0], cam.eye[1], cam.eye[2]);
    ps.dir = camera_dir(cam, uv.x, uv.y);
    ps.tmin = 0.0f;
    ps.T = rgb(1.0f);
    ps.color = rgb(0.0f);
    ps.pdf_prev = 0.0f;
    ps.path_len = 0;
}

/// Builds SoL's SurfaceInfo for a closest hit (src/triangle_mesh.cpp:78-99)
/// from the triangle's shading record.  With `have_uv` the hit's barycentrics
/// are (hu, hv) from the traversal's triangle test; otherwise the test is
/// repeated here on the triangle's vertices (same inputs, same values).
__device__ __forceinline__ Surface make_surface(const SceneView& s, int slot, Vec3 org, Vec3 dir, float t,
                                                float tmin, int* bsdf, int* light, bool have_uv = false,
                                                float hu = 0.0f, float hv = 0.0f) {
    const DTriShade* sp = s.shade + slot;
    const float4 a = ldg4(sp->n0), b = ldg4(sp->n1), c = ldg4(sp->n2), d = ldg4(&sp->uv1y), e = ldg4(sp->fn);
    *bsdf = __float_as_int(d.w);
    *light = __float_as_int(e.w);
    float tt, u = hu, v = hv;
    if (!have_uv) {
        const DTri* tp = s.tris + slot;
        const float4 p0 = ldg4(tp->v0), p1 = ldg4(tp->v1), p2 = ldg4(tp->v2);
        intersect_triangle(make_shear(org, dir), tri_vertex(p0), tri_vertex(p1), tri_vertex(p2), tmin, kFloatMax, &tt,
                           &u, &v);
    }
    Vec3 face_normal = vec3(e.x, e.y, e.z);
    Vec3 normal = lerp3(vec3(a.x, a.y, a.z), vec3(b.x, b.y, b.z), vec3(c.x, c.y, c.z), u, v);
    Vec2 uv = lerp3(vec2(a.w, b.w), vec2(c.w, d.x), vec2(d.y, d.z), u, v);
    Surface sf;
    sf.front = dot(face_normal, dir) < 0.0f;
    if (!sf.front) { face_normal = -face_normal; normal = -normal; }
    sf.point = org + dir * t;
    sf.uv = uv;
    sf.surf = vec2(u, v);
    sf.face_normal = face_normal;
    sf.local = ortho_basis(normalize(normal));
    return sf;
}

/// Observer of shade_vertex that records nothing (the forward render).  The
/// path-replay adjoint passes an observer with the same hooks that keeps, per
/// vertex, the quantities its reverse sweep needs; the hooks see the values the
/// forward computes, so forward and replay cannot drift apart.
struct NoRecord {
    __device__ __forceinline__ void begin(const PathState&, const Surface&) {}
    __device__ __forceinline__ void emission(const SceneView&, const DLight&, Vec3, const Surface&, Rgb, float) {}
    __device__ __forceinline__ void before_light_sample(const DLight&, const Pcg&) {}
    __device__ __forceinline__ void light_sample(const SceneView&, int, const DLight&, const Surface&, Vec3, Vec3, Rgb,
                                                 Rgb, float) {}
    __device__ __forceinline__ void survival(float, bool) {}
    __device__ __forceinline__ void before_bounce(const SceneView&, int, const Surface&, const Pcg&) {}
    __device__ __forceinline__ void bounce(const SceneView&, int, const Surface&, Vec3, const BsdfSample&, float) {}
};

/// One iteration of trace_path after a closest hit at (`slot`, `t`): direct
/// emission with MIS (:48-60), light sample with MIS (:66-97, the shadow ray is
/// returned for the caller to trace), Russian roulette (:99-108) and the BSDF
/// bounce (:110-117), which replaces the state's ray.  `rec` observes the
/// vertex (see NoRecord).
template <class Rec, bool kBasic = false>
__device__ __forceinline__ void shade_vertex(const SceneView& s, const DConfig& cfg, float light_pick_prob,
                                             int slot, float t, PathState& ps, VertexOut& out, Rec& rec,
                                             bool have_uv = false, float hu = 0.0f, float hv = 0.0f) {
    out.end = false;
    out.has_shadow = false;
    int bsdf_id, light_id;
    const Surface sf = make_surface(s, slot, ps.org, ps.dir, t, ps.tmin, &bsdf_id, &light_id, have_uv, hu, hv);
    const Vec3 out_dir = -ps.dir;
    const uint32_t nl = s.num_lights;
    rec.begin(ps, sf);

    if (light_id >= 0 && sf.front) {
        const float pdf_prev_area = ps.pdf_prev * dot(out_dir, sf.normal()) / (t * t);
        Rgb le; float pdf_from;
        const DLight light = s.lights[light_id];
        light_emission<kBasic>(s, light, out_dir, sf.surf, &le, &pdf_from);
        const float mis = ps.pdf_prev != 0.0f ? balance_heuristic(pdf_prev_area, pdf_from * light_pick_prob) : 1.0f;
        ps.color = ps.color + ps.T * le * mis;
        rec.emission(s, light, out_dir, sf, le, mis);
    }
    if (bsdf_id < 0) { out.end = true; return; }

    const bool skip_nee = s.bsdfs[bsdf_id].type == kTypeSpecular;
    if (!skip_nee && nl > 0) {
        uint32_t li = (uint32_t)(ps.rng.next_float() * (float)nl);
        li = li < nl - 1 ? li : nl - 1;
        const DLight light = s.lights[li];
        rec.before_light_sample(light, ps.rng);
        LightSample ls;
        if (light_sample_area<kBasic>(s, light, ps.rng, sf.point, &ls)) {
            Vec3 in_dir = ls.pos - sf.point;
            float cos_surf = dot(in_dir, sf.normal());
            out.sh_org = sf.point;
            out.sh_dir = ls.pos - sf.point;
            const float inv_light_dist = ls.inv_dist;   // 1 / length(in_dir), from the light sample
            cos_surf = cos_surf * inv_light_dist;
            in_dir = in_dir * inv_light_dist;
            const bool has_area = light.kind != SOL_GPU_LIGHT_POINT;
            Rgb f;
            float pdf_bounce;
            bsdf_eval_pdf<kBasic>(s, bsdf_id, in_dir, sf, out_dir, has_area, &f, &pdf_bounce);
            const float pdf_light = ls.pdf_from * light_pick_prob;
            const float geom_term = ls.cos * inv_light_dist * inv_light_dist;
            const float mis = has_area ? balance_heuristic(pdf_light, pdf_bounce * geom_term) : 1.0f;
            const float scale = geom_term * cos_surf * mis / pdf_light;
            out.pending = ls.intensity * ps.T * f * scale;
            out.has_shadow = true;
            rec.light_sample(s, bsdf_id, light, sf, in_dir, out_dir, ls.intensity, f, scale);
        }
    }
    float survival = 1.0f;
    if (ps.path_len >= cfg.min_rr_path_len) {
        const float lum = luminance(ps.T);
        survival = clampf(lum, cfg.min_survival_prob, cfg.max_survival_prob);
        rec.survival(survival, lum > cfg.min_survival_prob && lum < cfg.max_survival_prob);
        if (ps.rng.next_float() >= survival) { out.end = true; return; }
    } else {
        rec.survival(1.0f, false);
    }
    rec.before_bounce(s, bsdf_id, sf, ps.rng);
    BsdfSample bs;
    if (!bsdf_sample<kBasic>(s, bsdf_id, ps.rng, sf, out_dir, &bs)) { out.end = true; return; }
    const float r = bs.cos / (bs.pdf * survival);
    ps.T = ps.T * (bs.color * r);
    ps.org = sf.point;
    ps.dir = bs.in_dir;
    ps.tmin = cfg.ray_offset;
    ps.pdf_prev = skip_nee ? 0.0f : bs.pdf;
    rec.bounce(s, bsdf_id, sf, out_dir, bs, r);
}

/// shade_vertex for the forward render (no observer); kBasic as in shading.cuh.
template <bool kBasic = false>
__device__ __forceinline__ void shade_vertex(const SceneView& s, const DConfig& cfg, float light_pick_prob,
                                             int slot, float t, PathState& ps, VertexOut& out, bool have_uv = false,
                                             float hu = 0.0f, float hv = 0.0f) {
    NoRecord none;
    shade_vertex<NoRecord, kBasic>(s, cfg, light_pick_prob, slot, t, ps, out, none, have_uv, hu, hv);
}

}  // namespace sol_b200
