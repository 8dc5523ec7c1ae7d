// sol::GpuPathTracer: flattening of a sol::Scene into the C ABI's flat scene,
// and render() through sol_gpu_render.
//
// SoL keeps the parameters this needs in private members without accessors
// (bsdfs.h:110,128-129,142,158-160, lights.h:107-108,133-134,
// triangle_mesh.h:53-59, cameras.h:50-54).  Integrated into SoL, the class is
// declared a friend of those classes (`friend class GpuPathTracer;` in each,
// the header patch INTEGRATION.md gives) and this file is compiled with
// SOL_GPU_FRIEND_PATCH defined.  Without the patch -- the test build, against
// SoL's unmodified headers -- it gets the same access by widening
// `private`/`protected` while it includes them: the class layouts are
// unchanged, only access checking is (a stand-in for the friend declarations,
// not the integration).
// TriangleMesh's hierarchy holder is defined only inside triangle_mesh.cpp
// (src/triangle_mesh.cpp:27-28); its one-member definition is repeated here.

// Every header that the SoL headers pull in is included first, with normal access.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <numbers>
#include <optional>
#include <random>
#include <stdexcept>
#include <string>
#include <string_view>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <proto/hash.h>
#include <proto/mat.h>
#include <proto/random.h>
#include <proto/ray.h>
#include <proto/sphere.h>
#include <proto/triangle.h>
#include <proto/utils.h>
#include <proto/vec.h>
#include <bvh/bvh.h>

#ifndef SOL_GPU_FRIEND_PATCH
#define private public
#define protected public
#endif
#include "sol/bsdfs.h"
#include "sol/cameras.h"
#include "sol/image.h"
#include "sol/lights.h"
#include "sol/scene.h"
#include "sol/shapes.h"
#include "sol/textures.h"
#include "sol/triangle_mesh.h"
#ifndef SOL_GPU_FRIEND_PATCH
#undef private
#undef protected
#endif

#include "gpu_path_tracer.h"

namespace sol {

struct TriangleMesh::BvhData { bvh::Bvh<float> bvh; };

namespace {

template <typename T, typename P>
int32_t index_of(const std::vector<std::unique_ptr<T>>& v, const P* p) {
    for (size_t i = 0; i < v.size(); ++i)
        if (static_cast<const void*>(v[i].get()) == static_cast<const void*>(p)) return (int32_t)i;
    throw std::runtime_error("GpuPathTracer: object not owned by the scene");
}

void put3(float* dst, const proto::Vec3f& v) { dst[0] = v[0]; dst[1] = v[1]; dst[2] = v[2]; }

template <typename F>
const Image& image_of(const Texture& t, int border) {
    switch (border) {
        case 0: return static_cast<const ImageTexture<F, BorderMode::Clamp>&>(t).image();
        case 1: return static_cast<const ImageTexture<F, BorderMode::Repeat>&>(t).image();
        default: return static_cast<const ImageTexture<F, BorderMode::Mirror>&>(t).image();
    }
}

/// The image of an ImageTexture, by the filter / border decoded from its tag.
const Image& texture_image(const Texture& t, int filter, int border) {
    return filter == 0 ? image_of<ImageFilter::Nearest>(t, border) : image_of<ImageFilter::Bilinear>(t, border);
}

struct Flat {
    std::vector<float> vertices, normals, tex_coords;
    std::vector<uint32_t> indices, prims;
    std::vector<int32_t> tri_bsdf, tri_light;
    std::vector<SolGpuTexture> textures;
    std::vector<SolGpuImage> images;
    std::vector<SolGpuBsdf> bsdfs;
    std::vector<SolGpuLight> lights;
    std::vector<SolGpuBvhNode> nodes;
    SolGpuSceneDesc desc{};
};

void flatten(const Scene& scene, Flat& f) {
    const auto* mesh = dynamic_cast<const TriangleMesh*>(scene.root.get());
    if (!mesh) throw std::runtime_error("GpuPathTracer: the scene root must be a TriangleMesh");

    for (auto& img : scene.images) {
        if (img->channel_count() != 3) throw std::runtime_error("GpuPathTracer: images must have 3 channels");
        SolGpuImage g{};
        g.width = (uint32_t)img->width();
        g.height = (uint32_t)img->height();
        for (int c = 0; c < 3; ++c) g.channels[c] = img->channel(c).get();
        f.images.push_back(g);
    }
    constexpr size_t kBorders = BorderMode::tag_count();
    for (auto& t : scene.textures) {
        SolGpuTexture g{};
        g.image = -1;
        if (t->tag == Texture::Tag::ConstantTexture) {
            g.type = SOL_GPU_TEX_CONSTANT;
            g.value[0] = static_cast<const ConstantTexture&>(*t).constant_;
        } else if (t->tag == Texture::Tag::ConstantColorTexture) {
            g.type = SOL_GPU_TEX_CONSTANT_COLOR;
            const Color& c = static_cast<const ConstantColorTexture&>(*t).color_;
            g.value[0] = c.r; g.value[1] = c.g; g.value[2] = c.b;
        } else {
            // ImageTexture<Filter, Border>: tag = ImageTextureBegin + filter * borders + border (textures.h:79-85).
            size_t k = static_cast<size_t>(t->tag) - static_cast<size_t>(Texture::Tag::ImageTextureBegin);
            g.type = SOL_GPU_TEX_IMAGE;
            g.filter = (int32_t)(k / kBorders);
            g.border = (int32_t)(k % kBorders);
            g.image = index_of(scene.images, &texture_image(*t, g.filter, g.border));
        }
        f.textures.push_back(g);
    }
    auto tex = [&](const Texture& t) { return index_of(scene.textures, &t); };
    for (auto& b : scene.bsdfs) {
        SolGpuBsdf g{};
        g.tex[0] = g.tex[1] = g.tex[2] = -1;
        g.a = g.b = -1;
        switch (b->tag) {
            case Bsdf::Tag::DiffuseBsdf:
                g.type = SOL_GPU_BSDF_DIFFUSE;
                g.tex[0] = tex(static_cast<const DiffuseBsdf&>(*b).kd_);
                break;
            case Bsdf::Tag::PhongBsdf:
                g.type = SOL_GPU_BSDF_PHONG;
                g.tex[0] = tex(static_cast<const PhongBsdf&>(*b).ks_);
                g.tex[1] = tex(static_cast<const PhongBsdf&>(*b).ns_);
                break;
            case Bsdf::Tag::MirrorBsdf:
                g.type = SOL_GPU_BSDF_MIRROR;
                g.tex[0] = tex(static_cast<const MirrorBsdf&>(*b).ks_);
                break;
            case Bsdf::Tag::GlassBsdf:
                g.type = SOL_GPU_BSDF_GLASS;
                g.tex[0] = tex(static_cast<const GlassBsdf&>(*b).ks_);
                g.tex[1] = tex(static_cast<const GlassBsdf&>(*b).kt_);
                g.tex[2] = tex(static_cast<const GlassBsdf&>(*b).eta_);
                break;
            case Bsdf::Tag::InterpBsdf: {
                const auto& ib = static_cast<const InterpBsdf&>(*b);
                g.type = SOL_GPU_BSDF_INTERP;
                g.tex[0] = tex(ib.k_);
                g.a = index_of(scene.bsdfs, ib.a_);
                g.b = index_of(scene.bsdfs, ib.b_);
                break;
            }
        }
        f.bsdfs.push_back(g);
    }
    for (auto& l : scene.lights) {
        SolGpuLight g{};
        g.intensity_tex = -1;
        if (l->tag == Light::Tag::PointLight) {
            const auto& pl = static_cast<const PointLight&>(*l);
            g.type = SOL_GPU_LIGHT_POINT;
            put3(g.v0, pl.pos_);
            g.intensity[0] = pl.intensity_.r; g.intensity[1] = pl.intensity_.g; g.intensity[2] = pl.intensity_.b;
        } else if (l->tag == Light::Tag::UniformTriangleLight) {
            const auto& al = static_cast<const UniformTriangleLight&>(*l);
            g.type = SOL_GPU_LIGHT_TRIANGLE;
            put3(g.v0, al.shape_.shape.v0);
            put3(g.v1, al.shape_.shape.v1);
            put3(g.v2, al.shape_.shape.v2);
            g.intensity_tex = tex(al.intensity_);
        } else {
            const auto& al = static_cast<const UniformSphereLight&>(*l);
            g.type = SOL_GPU_LIGHT_SPHERE;
            put3(g.v0, al.shape_.shape.center);
            g.v1[0] = al.shape_.shape.radius;
            g.intensity_tex = tex(al.intensity_);
        }
        f.lights.push_back(g);
    }

    // Mesh: SoL keeps the triangles in BVH leaf order (triangles_[j] is
    // triangle prim_indices[j], src/triangle_mesh.cpp:148-160) and no vertex
    // array, so every triangle gets its own three vertices here.
    const auto& bvh = mesh->bvh_data_->bvh;
    const size_t nt = mesh->triangle_count();
    f.vertices.resize(9 * nt);
    f.normals.resize(9 * nt);
    f.tex_coords.resize(6 * nt);
    f.indices.resize(3 * nt);
    f.tri_bsdf.resize(nt);
    f.tri_light.assign(nt, -1);
    for (size_t j = 0; j < nt; ++j) {
        const size_t t = bvh.prim_indices[j];
        const auto& tri = mesh->triangles_[j];
        put3(&f.vertices[9 * t + 0], tri.v0);
        put3(&f.vertices[9 * t + 3], tri.v1);
        put3(&f.vertices[9 * t + 6], tri.v2);
    }
    for (size_t t = 0; t < nt; ++t) {
        auto [i0, i1, i2] = mesh->triangle_indices(t);
        const size_t iv[3] = {i0, i1, i2};
        for (int k = 0; k < 3; ++k) {
            put3(&f.normals[9 * t + 3 * k], mesh->normals_[iv[k]]);
            f.tex_coords[6 * t + 2 * k + 0] = mesh->tex_coords_[iv[k]][0];
            f.tex_coords[6 * t + 2 * k + 1] = mesh->tex_coords_[iv[k]][1];
            f.indices[3 * t + k] = (uint32_t)(3 * t + k);
        }
        const Bsdf* b = mesh->bsdfs_[t];
        f.tri_bsdf[t] = b ? index_of(scene.bsdfs, b) : -1;
    }
    for (auto& [t, l] : mesh->lights_) f.tri_light[t] = index_of(scene.lights, l);
    f.nodes.resize(bvh.nodes.size());
    for (size_t i = 0; i < bvh.nodes.size(); ++i) {
        const auto& n = bvh.nodes[i];
        for (int k = 0; k < 3; ++k) { f.nodes[i].lo[k] = n.box.lo[k]; f.nodes[i].hi[k] = n.box.hi[k]; }
        f.nodes[i].first = (uint32_t)n.first_index;
        f.nodes[i].count = (uint32_t)n.prim_count;
    }
    f.prims.assign(bvh.prim_indices.begin(), bvh.prim_indices.end());

    SolGpuSceneDesc& d = f.desc;
    d.num_vertices = (uint32_t)(3 * nt);
    d.num_triangles = (uint32_t)nt;
    d.vertices = f.vertices.data();
    d.normals = f.normals.data();
    d.tex_coords = f.tex_coords.data();
    d.indices = f.indices.data();
    d.tri_bsdf = f.tri_bsdf.data();
    d.tri_light = f.tri_light.data();
    d.num_bsdfs = (uint32_t)f.bsdfs.size(); d.bsdfs = f.bsdfs.data();
    d.num_textures = (uint32_t)f.textures.size(); d.textures = f.textures.data();
    d.num_images = (uint32_t)f.images.size(); d.images = f.images.data();
    d.num_lights = (uint32_t)f.lights.size(); d.lights = f.lights.data();
    d.num_bvh_nodes = (uint32_t)f.nodes.size(); d.bvh_nodes = f.nodes.data();
    d.bvh_prim_indices = f.prims.data();
}

[[noreturn]] void throw_status(int rc, const char* what) {
    throw std::runtime_error(std::string("GpuPathTracer: ") + what + " failed (" + std::to_string(rc) + "): " +
                             sol_gpu_last_error());
}

}  // namespace

GpuPathTracer::GpuPathTracer(const Scene& scene, const Config& config, int device)
    : Renderer("GpuPathTracer", scene), config_(config), device_(device) {}

GpuPathTracer::~GpuPathTracer() {
    if (gpu_scene_) sol_gpu_scene_destroy(gpu_scene_);
}

void GpuPathTracer::prepare() const {
    std::lock_guard<std::mutex> lock(mutex_);
    if (gpu_scene_) return;
    const auto* cam = dynamic_cast<const PerspectiveCamera*>(scene_.camera.get());
    if (!cam) throw std::runtime_error("GpuPathTracer: the camera must be a PerspectiveCamera");
    put3(camera_.eye, cam->eye_);
    put3(camera_.dir, cam->dir_);
    put3(camera_.right, cam->right_);
    put3(camera_.up, cam->up_);
    Flat f;
    flatten(scene_, f);
    SolGpuScene* s = nullptr;
    int rc = sol_gpu_scene_create(&f.desc, device_, &s);
    if (rc != SOL_GPU_OK) throw_status(rc, "sol_gpu_scene_create");
    gpu_scene_ = s;
}

void GpuPathTracer::render(Image& image, size_t sample_index, size_t sample_count) const {
    prepare();
    if (image.channel_count() != 3) throw std::runtime_error("GpuPathTracer: the image must have 3 channels");
    SolGpuConfig c{};
    c.max_path_len = (uint32_t)std::min<size_t>(config_.max_path_len, UINT32_MAX);
    c.min_rr_path_len = (uint32_t)std::min<size_t>(config_.min_rr_path_len, UINT32_MAX);
    c.min_survival_prob = config_.min_survival_prob;
    c.max_survival_prob = config_.max_survival_prob;
    c.ray_offset = config_.ray_offset;
    std::lock_guard<std::mutex> lock(mutex_);
    // Large requests are split so that the per-call sample count fits 32 bits.
    while (sample_count > 0) {
        uint32_t n = (uint32_t)std::min<size_t>(sample_count, 1u << 30);
        int rc = sol_gpu_render(gpu_scene_, &camera_, &c, sample_index, n, (uint32_t)image.width(),
                                (uint32_t)image.height(), image.channel(0).get(), image.channel(1).get(),
                                image.channel(2).get());
        if (rc != SOL_GPU_OK) throw_status(rc, "sol_gpu_render");
        sample_index += n;
        sample_count -= n;
    }
}

}  // namespace sol
