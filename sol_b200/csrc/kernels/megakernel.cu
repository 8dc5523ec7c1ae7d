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
// One iteration of the loop traces one closest-hit ray, shades the hit (direct
// emission with MIS, light sample + MIS, Russian roulette, BSDF sample), then
// traces the shadow ray of that vertex.  The light contribution is added after
// the shadow ray returns and before the next vertex's emission, which is the
// order SoL adds them in; the random draws happen in SoL's order regardless of
// the shadow ray's outcome.
#include <cuda_runtime.h>

#include "kernels.h"
#include "shading.cuh"
#include "traverse.cuh"

namespace sol_b200 {

namespace {

struct PixelTile {
    uint32_t tiles_x;
    uint32_t total;  // tiles * 32
};

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

/// Builds SoL's SurfaceInfo for a closest hit (src/triangle_mesh.cpp:78-99).
__device__ __forceinline__ Surface make_surface(const SceneView& s, int slot, Vec3 org, Vec3 dir, float t,
                                                float tmin, int* bsdf, int* light) {
    const DTri* tp = s.tris + slot;
    const float4 p0 = ldg4(tp->v0), p1 = ldg4(tp->v1), p2 = ldg4(tp->v2);
    const Vec3 v0 = tri_vertex(p0), v1 = tri_vertex(p1), v2 = tri_vertex(p2);
    *bsdf = __float_as_int(p1.w);
    *light = __float_as_int(p2.w);
    // Barycentrics of the hit: the same test, same inputs, hence the same values.
    float tt, u = 0.0f, v = 0.0f;
    intersect_triangle(make_shear(org, dir), v0, v1, v2, tmin, kFloatMax, &tt, &u, &v);
    const DTriShade* sp = s.shade + slot;
    const float4 a = ldg4(sp->n0), b = ldg4(sp->n1), c = ldg4(sp->n2), d = ldg4(&sp->uv1y);
    Vec3 face_normal = triangle_normal(v0, v1, v2);
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

template <bool kCount>
__global__ void __launch_bounds__(kMegakernelBlock)
pt_megakernel(SceneView s, DCamera cam, DConfig cfg, uint64_t sample_index, uint32_t sample_count,
              uint32_t width, uint32_t height, float* __restrict__ film, DeviceCounters* __restrict__ ctr) {
    const uint32_t tiles_x = (width + 7u) / 8u;
    const uint32_t total = tiles_x * ((height + 3u) / 4u) * 32u;
    const size_t plane = (size_t)width * height;
    const uint32_t nl = s.num_lights;
    const float light_pick_prob = 1.0f / (float)nl;

    TraversalCounters tc{0u, 0u};
    uint32_t n_paths = 0, n_rays = 0, n_shadow = 0;

    bool have_pixel = false;
    uint32_t px = 0, py = 0, sample = 0;
    Rgb pix_sum = rgb(0.0f);

    Pcg rng;
    rng.state = 0;
    Vec3 org = vec3(0.0f), dir = vec3(0.0f, 0.0f, 1.0f);
    float tmin = 0.0f;
    Rgb T = rgb(1.0f), color = rgb(0.0f);
    float pdf_prev = 0.0f;
    uint32_t path_len = 0;
    bool done = false;

    while (true) {
        // --- make sure this lane has a live path (or stop) ------------------
        bool alive = false;
        while (!alive) {
            if (have_pixel && sample < sample_count) {
                // path_tracer.cpp:16-18: one sampler per (pixel, sample)
                rng = make_pcg(pixel_seed(sample_index + sample, px, py));
                Vec2 uv = sample_pixel(rng, px, py, width, height);
                org = vec3(cam.eye[0], cam.eye[1], cam.eye[2]);
                dir = camera_dir(cam, uv.x, uv.y);
                tmin = 0.0f;
                T = rgb(1.0f);
                color = rgb(0.0f);
                pdf_prev = 0.0f;
                path_len = 0;
                ++n_paths;
                if (cfg.max_path_len == 0) { pix_sum = pix_sum + color; ++sample; continue; }
                alive = true;
            } else {
                if (have_pixel) {
                    // image.h:54-60 accumulate
                    size_t i = (size_t)py * width + px;
                    film[i] += pix_sum.r;
                    film[i + plane] += pix_sum.g;
                    film[i + 2 * plane] += pix_sum.b;
                    have_pixel = false;
                }
                uint32_t item = claim_items(&ctr->next_item);
                if (item >= total) { done = true; break; }
                uint32_t tile = item >> 5, l = item & 31u;
                px = (tile % tiles_x) * 8u + (l & 7u);
                py = (tile / tiles_x) * 4u + (l >> 3);
                if (px < width && py < height) {
                    have_pixel = true;
                    sample = 0;
                    pix_sum = rgb(0.0f);
                }
            }
        }
        if (done) break;

        // --- closest hit (path_tracer.cpp:42) ------------------------------
        float t = kFloatMax;
        const int slot = traverse<false, kCount>(s.nodes, s.tris, org, dir, tmin, t, s.num_tris > 0, tc);
        ++n_rays;

        bool end = slot < 0;
        bool has_shadow = false;
        Vec3 sh_org = vec3(0.0f), sh_dir = vec3(0.0f);
        Rgb pending = rgb(0.0f);
        if (!end) {
            int bsdf_id, light_id;
            const Surface sf = make_surface(s, slot, org, dir, t, tmin, &bsdf_id, &light_id);
            const Vec3 out_dir = -dir;

            // Direct hit on a light (path_tracer.cpp:48-60)
            if (light_id >= 0 && sf.front) {
                const float pdf_prev_area = pdf_prev * dot(out_dir, sf.normal()) / (t * t);
                Rgb le; float pdf_from;
                light_emission(s, s.lights[light_id], out_dir, sf.surf, &le, &pdf_from);
                const float mis = pdf_prev != 0.0f ? balance_heuristic(pdf_prev_area, pdf_from * light_pick_prob) : 1.0f;
                color = color + T * le * mis;
            }

            if (bsdf_id < 0) {
                end = true;   // path_tracer.cpp:62-63
            } else {
                const bool skip_nee = s.bsdfs[bsdf_id].type == kTypeSpecular;
                // Next-event estimation (path_tracer.cpp:66-97)
                if (!skip_nee && nl > 0) {
                    uint32_t li = (uint32_t)(rng.next_float() * (float)nl);
                    li = li < nl - 1 ? li : nl - 1;
                    const DLight light = s.lights[li];
                    LightSample ls;
                    if (light_sample_area(s, light, rng, sf.point, &ls)) {
                        Vec3 in_dir = ls.pos - sf.point;
                        float cos_surf = dot(in_dir, sf.normal());
                        sh_org = sf.point;
                        sh_dir = ls.pos - sf.point;
                        const float inv_light_dist = 1.0f / length(in_dir);
                        cos_surf = cos_surf * inv_light_dist;
                        in_dir = in_dir * inv_light_dist;
                        const bool has_area = light.kind != SOL_GPU_LIGHT_POINT;
                        const float pdf_bounce = has_area ? bsdf_pdf(s, bsdf_id, in_dir, sf, out_dir) : 0.0f;
                        const float pdf_light = ls.pdf_from * light_pick_prob;
                        const float geom_term = ls.cos * inv_light_dist * inv_light_dist;
                        const float mis = has_area ? balance_heuristic(pdf_light, pdf_bounce * geom_term) : 1.0f;
                        pending = ls.intensity * T * bsdf_eval(s, bsdf_id, in_dir, sf, out_dir) *
                                  (geom_term * cos_surf * mis / pdf_light);
                        has_shadow = true;
                    }
                }
                // Russian roulette (path_tracer.cpp:99-108)
                float survival = 1.0f;
                if (path_len >= cfg.min_rr_path_len) {
                    survival = clampf(luminance(T), cfg.min_survival_prob, cfg.max_survival_prob);
                    if (rng.next_float() >= survival) end = true;
                }
                // Bounce (path_tracer.cpp:110-117)
                if (!end) {
                    BsdfSample bs;
                    if (!bsdf_sample(s, bsdf_id, rng, sf, out_dir, &bs)) {
                        end = true;
                    } else {
                        T = T * (bs.color * (bs.cos / (bs.pdf * survival)));
                        org = sf.point;
                        dir = bs.in_dir;
                        tmin = cfg.ray_offset;
                        pdf_prev = skip_nee ? 0.0f : bs.pdf;
                    }
                }
            }
        }

        // --- shadow ray of this vertex (path_tracer.cpp:72-74) -------------
        if (has_shadow) {
            float smax = 1.0f - cfg.ray_offset;
            const int occ = traverse<true, kCount>(s.nodes, s.tris, sh_org, sh_dir, cfg.ray_offset, smax, s.num_tris > 0, tc);
            ++n_rays;
            ++n_shadow;
            if (occ < 0) color = color + pending;
        }

        if (!end) {
            ++path_len;
            end = path_len >= cfg.max_path_len;
        }
        if (end) {
            pix_sum = pix_sum + color;   // path_tracer.cpp:19
            ++sample;
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

}  // namespace

int megakernel_blocks_per_sm(bool instrumented) {
    int n = 0;
    cudaError_t e = instrumented
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pt_megakernel<true>, kMegakernelBlock, 0)
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pt_megakernel<false>, kMegakernelBlock, 0);
    return e == cudaSuccess ? n : -1;
}

cudaError_t launch_megakernel(const SceneView& s, const DCamera& cam, const DConfig& cfg,
                              uint64_t sample_index, uint32_t sample_count, uint32_t width, uint32_t height,
                              float* film, DeviceCounters* counters, bool instrumented, int grid,
                              cudaStream_t stream) {
    if (instrumented)
        pt_megakernel<true><<<grid, kMegakernelBlock, 0, stream>>>(s, cam, cfg, sample_index, sample_count, width, height, film, counters);
    else
        pt_megakernel<false><<<grid, kMegakernelBlock, 0, stream>>>(s, cam, cfg, sample_index, sample_count, width, height, film, counters);
    return cudaGetLastError();
}

}  // namespace sol_b200
