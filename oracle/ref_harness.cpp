// Test infrastructure (oracle): drives SoL's own CPU path tracer, compiled from
// the SoL sources against the clean-room proto/par/bvh shims in oracle/shim.
//
// A flat scene (include/sol_gpu.h) is turned into a sol::Scene through SoL's
// public constructors (the same ones its OBJ loader uses, src/formats/obj.cpp:375-516),
// then rendered with sol::PathTracer::render.  Used as the checker of the
// restated oracle and of the GPU path, and as the timed CPU baseline.
#include <chrono>
#include <cstring>
#include <memory>
#include <optional>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include <omp.h>

#include "sol/algorithms/path_tracer.h"
#include "sol/bsdfs.h"
#include "sol/cameras.h"
#include "sol/image.h"
#include "sol/lights.h"
#include "sol/render_job.h"
#include "sol/scene.h"
#include "sol/textures.h"
#include "sol/triangle_mesh.h"

#include "oracle_camera.h"
#include "ref_harness.h"
#include "sol_gpu.h"

// SoL's EXR support needs tinyexr, which is not vendored; the path tracer never
// touches files, so image I/O is stubbed here.
namespace sol::exr {
std::optional<Image> load(const std::string_view&) { return std::nullopt; }
bool save(const Image&, const std::string_view&) { return false; }
}  // namespace sol::exr

namespace {

thread_local std::string g_err;

proto::Vec3f v3(const float* p) { return proto::Vec3f(p[0], p[1], p[2]); }

template <typename Filter>
std::unique_ptr<sol::Texture> image_texture(const sol::Image& img, int border) {
    switch (border) {
        case SOL_GPU_BORDER_CLAMP:  return std::make_unique<sol::ImageTexture<Filter, sol::BorderMode::Clamp>>(img);
        case SOL_GPU_BORDER_REPEAT: return std::make_unique<sol::ImageTexture<Filter, sol::BorderMode::Repeat>>(img);
        default:                    return std::make_unique<sol::ImageTexture<Filter, sol::BorderMode::Mirror>>(img);
    }
}

}  // namespace


extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

void ref_set_error(const char* what) { g_err = what; }

RefScene* ref_scene_create(const SolGpuSceneDesc* d, const OracleCamera* cam) {
    try {
        auto rs = std::make_unique<RefScene>();
        sol::Scene& s = rs->scene;
        std::vector<const sol::Image*> images;
        for (uint32_t i = 0; i < d->num_images; ++i) {
            const SolGpuImage& im = d->images[i];
            auto img = std::make_unique<sol::Image>(im.width, im.height, 3);
            for (int c = 0; c < 3; ++c)
                std::memcpy(img->channel(c).get(), im.channels[c], sizeof(float) * im.width * im.height);
            images.push_back(img.get());
            s.images.push_back(std::move(img));
        }
        std::vector<const sol::Texture*> textures;
        for (uint32_t i = 0; i < d->num_textures; ++i) {
            const SolGpuTexture& t = d->textures[i];
            std::unique_ptr<sol::Texture> tex;
            if (t.type == SOL_GPU_TEX_CONSTANT) tex = std::make_unique<sol::ConstantTexture>(t.value[0]);
            else if (t.type == SOL_GPU_TEX_CONSTANT_COLOR) tex = std::make_unique<sol::ConstantColorTexture>(sol::Color(t.value[0], t.value[1], t.value[2]));
            else if (t.filter == SOL_GPU_FILTER_NEAREST) tex = image_texture<sol::ImageFilter::Nearest>(*images.at(t.image), t.border);
            else tex = image_texture<sol::ImageFilter::Bilinear>(*images.at(t.image), t.border);
            textures.push_back(tex.get());
            s.textures.push_back(std::move(tex));
        }
        auto color_tex = [&](int32_t i) -> const sol::ColorTexture& { return static_cast<const sol::ColorTexture&>(*textures.at(i)); };
        std::vector<const sol::Bsdf*> bsdfs(d->num_bsdfs, nullptr);
        for (int pass = 0; pass < 2; ++pass) {
            for (uint32_t i = 0; i < d->num_bsdfs; ++i) {
                const SolGpuBsdf& b = d->bsdfs[i];
                if ((b.type == SOL_GPU_BSDF_INTERP) != (pass == 1)) continue;
                std::unique_ptr<sol::Bsdf> p;
                switch (b.type) {
                    case SOL_GPU_BSDF_DIFFUSE: p = std::make_unique<sol::DiffuseBsdf>(color_tex(b.tex[0])); break;
                    case SOL_GPU_BSDF_PHONG:   p = std::make_unique<sol::PhongBsdf>(color_tex(b.tex[0]), *textures.at(b.tex[1])); break;
                    case SOL_GPU_BSDF_MIRROR:  p = std::make_unique<sol::MirrorBsdf>(color_tex(b.tex[0])); break;
                    case SOL_GPU_BSDF_GLASS:   p = std::make_unique<sol::GlassBsdf>(color_tex(b.tex[0]), color_tex(b.tex[1]), *textures.at(b.tex[2])); break;
                    default:                   p = std::make_unique<sol::InterpBsdf>(bsdfs.at(b.a), bsdfs.at(b.b), *textures.at(b.tex[0])); break;
                }
                bsdfs[i] = p.get();
                s.bsdfs.push_back(std::move(p));
            }
        }
        std::vector<const sol::Light*> lights;
        for (uint32_t i = 0; i < d->num_lights; ++i) {
            const SolGpuLight& l = d->lights[i];
            std::unique_ptr<sol::Light> p;
            if (l.type == SOL_GPU_LIGHT_POINT)
                p = std::make_unique<sol::PointLight>(v3(l.v0), sol::Color(l.intensity[0], l.intensity[1], l.intensity[2]));
            else if (l.type == SOL_GPU_LIGHT_TRIANGLE)
                p = std::make_unique<sol::UniformTriangleLight>(sol::UniformTriangle(proto::Trianglef(v3(l.v0), v3(l.v1), v3(l.v2))), color_tex(l.intensity_tex));
            else
                p = std::make_unique<sol::UniformSphereLight>(sol::UniformSphere(proto::Spheref(v3(l.v0), l.v1[0])), color_tex(l.intensity_tex));
            lights.push_back(p.get());
            s.lights.push_back(std::move(p));
        }
        std::vector<size_t> indices(d->indices, d->indices + 3 * (size_t)d->num_triangles);
        std::vector<proto::Vec3f> vertices, normals;
        std::vector<proto::Vec2f> tex_coords;
        for (uint32_t i = 0; i < d->num_vertices; ++i) {
            vertices.push_back(v3(d->vertices + 3 * i));
            normals.push_back(v3(d->normals + 3 * i));
            tex_coords.push_back(proto::Vec2f(d->tex_coords[2 * i], d->tex_coords[2 * i + 1]));
        }
        std::vector<const sol::Bsdf*> tri_bsdfs(d->num_triangles);
        std::unordered_map<size_t, const sol::Light*> tri_lights;
        for (uint32_t i = 0; i < d->num_triangles; ++i) {
            tri_bsdfs[i] = d->tri_bsdf[i] >= 0 ? bsdfs.at(d->tri_bsdf[i]) : nullptr;
            if (d->tri_light[i] >= 0) tri_lights.emplace(i, lights.at(d->tri_light[i]));
        }
        s.root = std::make_unique<sol::TriangleMesh>(std::move(indices), std::move(vertices), std::move(normals),
                                                     std::move(tex_coords), std::move(tri_bsdfs), std::move(tri_lights));
        s.camera = std::make_unique<sol::PerspectiveCamera>(v3(cam->eye), v3(cam->dir), v3(cam->up), cam->fov, cam->aspect);
        return rs.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_scene_destroy(RefScene* s) { delete s; }

/// Replaces the scene's camera (a new sol::PerspectiveCamera from the same
/// constructor arguments), so one scene and its hierarchy serve many views.
int ref_scene_set_camera(RefScene* rs, const OracleCamera* cam) {
    if (!rs || !cam) { g_err = "null argument"; return -1; }
    rs->scene.camera = std::make_unique<sol::PerspectiveCamera>(v3(cam->eye), v3(cam->dir), v3(cam->up), cam->fov,
                                                                cam->aspect);
    return 0;
}

/// A scene file loaded by SoL's own loader (sol::Scene::load, src/scene_loader.cpp:
/// TOML scene description + OBJ/MTL import, src/formats/obj.cpp), with the
/// camera's aspect ratio defaulting to `aspect_ratio` as test/driver.cpp:197-199
/// sets it.  Returns nullptr with the loader's message in ref_last_error().
RefScene* ref_scene_load(const char* path, float aspect_ratio) {
    try {
        sol::Scene::Defaults defaults;
        defaults.aspect_ratio = aspect_ratio;
        std::ostringstream err;
        auto scene = sol::Scene::load(path, defaults, &err);
        if (!scene) { g_err = err.str(); return nullptr; }
        return new RefScene{std::move(*scene)};
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

/// Sizes of a loaded scene's tables: lights, BSDFs, textures, images.
void ref_scene_counts(const RefScene* rs, uint32_t* lights, uint32_t* bsdfs, uint32_t* textures, uint32_t* images) {
    *lights = (uint32_t)rs->scene.lights.size();
    *bsdfs = (uint32_t)rs->scene.bsdfs.size();
    *textures = (uint32_t)rs->scene.textures.size();
    *images = (uint32_t)rs->scene.images.size();
}

/// sol::PathTracer::render on a film that starts as the caller's channels and
/// is copied back afterwards (so the caller sees SoL's `+=`).  Returns the time
/// of the render call alone in `render_ms` (test/driver.cpp:232-238 times the
/// same region).
int ref_scene_render(RefScene* rs, const SolGpuConfig* cfg, uint64_t sample_index, uint32_t sample_count,
                     uint32_t width, uint32_t height, float* r, float* g, float* b, int threads, double* render_ms) {
    if (!rs || !cfg) { g_err = "null argument"; return -1; }
    if (threads > 0) omp_set_num_threads(threads);
    sol::PathTracer::Config c;
    c.max_path_len = cfg->max_path_len;
    c.min_rr_path_len = cfg->min_rr_path_len;
    c.min_survival_prob = cfg->min_survival_prob;
    c.max_survival_prob = cfg->max_survival_prob;
    c.ray_offset = cfg->ray_offset;
    sol::PathTracer tracer(rs->scene, c);
    sol::Image image(width, height, 3);
    float* film[3] = {r, g, b};
    const size_t n = (size_t)width * height;
    for (int ch = 0; ch < 3; ++ch) std::memcpy(image.channel(ch).get(), film[ch], sizeof(float) * n);
    auto t0 = std::chrono::steady_clock::now();
    tracer.render(image, sample_index, sample_count);
    auto t1 = std::chrono::steady_clock::now();
    if (render_ms) *render_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    for (int ch = 0; ch < 3; ++ch) std::memcpy(film[ch], image.channel(ch).get(), sizeof(float) * n);
    return 0;
}

/// sol::PathTracer driven by sol::RenderJob, for comparison with the above.
int ref_renderjob_render(RefScene* rs, const SolGpuConfig* cfg, uint32_t sample_count, uint32_t samples_per_frame,
                         uint32_t width, uint32_t height, float* r, float* g, float* b, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    sol::PathTracer::Config c;
    c.max_path_len = cfg->max_path_len;
    c.min_rr_path_len = cfg->min_rr_path_len;
    c.min_survival_prob = cfg->min_survival_prob;
    c.max_survival_prob = cfg->max_survival_prob;
    c.ray_offset = cfg->ray_offset;
    sol::PathTracer tracer(rs->scene, c);
    sol::Image image(width, height, 3);
    float* film[3] = {r, g, b};
    const size_t n = (size_t)width * height;
    for (int ch = 0; ch < 3; ++ch) std::memcpy(image.channel(ch).get(), film[ch], sizeof(float) * n);
    sol::RenderJob job(tracer, image);
    job.sample_count = sample_count;
    job.samples_per_frame = samples_per_frame;
    job.start();
    job.wait();
    for (int ch = 0; ch < 3; ++ch) std::memcpy(film[ch], image.channel(ch).get(), sizeof(float) * n);
    return 0;
}

/// Closest-hit / any-hit queries through sol::TriangleMesh (src/triangle_mesh.cpp:64-117).
/// Rays and hits use the layouts of SolGpuRay / SolGpuHit.
int ref_scene_trace(RefScene* rs, const SolGpuRay* rays, uint32_t count, int any_hit, SolGpuHit* hits) {
    const auto* mesh = dynamic_cast<const sol::TriangleMesh*>(rs->scene.root.get());
    if (!mesh) { g_err = "root is not a TriangleMesh"; return -1; }
    #pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < (long)count; ++i) {
        const SolGpuRay& q = rays[i];
        proto::Rayf ray(v3(q.org), v3(q.dir), q.tmin, q.tmax);
        SolGpuHit h{-1, 0.0f, 0.0f, 0.0f};
        if (any_hit) {
            if (mesh->intersect_any(ray)) h.tri = 0;
        } else if (auto hit = mesh->intersect_closest(ray)) {
            h.tri = 0;   // SoL's Hit does not expose the triangle index
            h.t = ray.tmax;
            h.u = hit->surf_info.surf_coords[0];
            h.v = hit->surf_info.surf_coords[1];
        }
        hits[i] = h;
    }
    return 0;
}

}  // extern "C"
