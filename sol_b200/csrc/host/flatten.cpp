// Scene validation and flattening into the device layout.
#include "flatten.h"

#include <chrono>
#include <cmath>
#include <numbers>

#include "../core/math.h"

namespace sol_b200 {

namespace {

Vec3 ld3(const float* p) { return vec3(p[0], p[1], p[2]); }

bool is_color_texture(const SolGpuSceneDesc& d, int32_t t) {
    return t >= 0 && (uint32_t)t < d.num_textures &&
           (d.textures[t].type == SOL_GPU_TEX_CONSTANT_COLOR || d.textures[t].type == SOL_GPU_TEX_IMAGE);
}
bool is_texture(const SolGpuSceneDesc& d, int32_t t) { return t >= 0 && (uint32_t)t < d.num_textures; }

int32_t leaf_ref(uint32_t first, uint32_t count) { return (int32_t)~((first << 3) | (count - 1u)); }

}  // namespace

bvh::Bvh build_mesh_bvh(const float* vertices, const uint32_t* indices, size_t ntri) {
    std::vector<bvh::BBox> boxes(ntri);
    std::vector<float> centers(3 * ntri);
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)ntri; ++i) {
        Vec3 v[3];
        bvh::BBox b = bvh::BBox::empty();
        for (int k = 0; k < 3; ++k) {
            const float* p = vertices + 3 * (size_t)indices[3 * i + k];
            v[k] = ld3(p);
            b.extend(p);
        }
        boxes[i] = b;
        Vec3 c = triangle_center(v[0], v[1], v[2]);
        centers[3 * i + 0] = c.x; centers[3 * i + 1] = c.y; centers[3 * i + 2] = c.z;
    }
    bvh::Bvh tree = bvh::build_sweep_sah(boxes.data(), centers.data(), ntri);
    bvh::ReinsertionOptimizer(tree).optimize();
    return tree;
}

SolGpuCamera perspective_camera(const float eye[3], const float dir_in[3], const float up_in[3], float fov, float aspect) {
    SolGpuCamera out;
    Vec3 dir = normalize(ld3(dir_in));
    Vec3 right = normalize(cross(ld3(dir_in), ld3(up_in)));
    Vec3 up = cross(right, dir);
    float w = std::tan(fov * std::numbers::pi_v<float> / 360.0f);
    float h = w / aspect;
    right = right * w;
    up = up * h;
    for (int k = 0; k < 3; ++k) {
        out.eye[k] = eye[k];
        out.dir[k] = comp(dir, k);
        out.right[k] = comp(right, k);
        out.up[k] = comp(up, k);
    }
    return out;
}

bool flatten_scene(const SolGpuSceneDesc& d, FlatScene& out, std::string& err, bool host_bvh) {
    auto t0 = std::chrono::steady_clock::now();
    const uint32_t nt = d.num_triangles, nv = d.num_vertices;
    if (nt > kMaxTriangles) { err = "too many triangles (max 2^28 - 2)"; return false; }
    if (nt > 0 && (!d.vertices || !d.normals || !d.tex_coords || !d.indices || !d.tri_bsdf || !d.tri_light)) {
        err = "mesh arrays must not be NULL"; return false;
    }
    for (size_t i = 0; i < 3 * (size_t)nt; ++i)
        if (d.indices[i] >= nv) { err = "vertex index out of range at index " + std::to_string(i); return false; }
    for (uint32_t i = 0; i < nt; ++i) {
        if (d.tri_bsdf[i] < -1 || (d.tri_bsdf[i] >= 0 && (uint32_t)d.tri_bsdf[i] >= d.num_bsdfs)) { err = "triangle BSDF out of range"; return false; }
        if (d.tri_light[i] < -1 || (d.tri_light[i] >= 0 && (uint32_t)d.tri_light[i] >= d.num_lights)) { err = "triangle light out of range"; return false; }
    }

    // Images: planar texel arena.
    out.images.resize(d.num_images);
    size_t texel_count = 0;
    for (uint32_t i = 0; i < d.num_images; ++i) {
        const SolGpuImage& im = d.images[i];
        if (im.width == 0 || im.height == 0 || !im.channels[0] || !im.channels[1] || !im.channels[2]) {
            err = "image " + std::to_string(i) + " is empty"; return false;
        }
        texel_count += 3 * (size_t)im.width * im.height;
    }
    out.texels.resize(texel_count);
    size_t off = 0;
    for (uint32_t i = 0; i < d.num_images; ++i) {
        const SolGpuImage& im = d.images[i];
        size_t plane = (size_t)im.width * im.height;
        out.images[i].offset = off;
        out.images[i].width = im.width;
        out.images[i].height = im.height;
        for (int c = 0; c < 3; ++c) std::copy(im.channels[c], im.channels[c] + plane, out.texels.begin() + (long)(off + c * plane));
        off += 3 * plane;
    }

    // Textures.
    out.textures.resize(d.num_textures);
    for (uint32_t i = 0; i < d.num_textures; ++i) {
        const SolGpuTexture& t = d.textures[i];
        DTexture& o = out.textures[i];
        o.kind = t.type; o.filter = t.filter; o.border = t.border; o.image = t.image;
        o.v[0] = t.value[0]; o.v[1] = t.value[1]; o.v[2] = t.value[2]; o.pad = 0;
        if (t.type < SOL_GPU_TEX_CONSTANT || t.type > SOL_GPU_TEX_IMAGE) { err = "bad texture type"; return false; }
        if (t.type == SOL_GPU_TEX_IMAGE) {
            if (t.image < 0 || (uint32_t)t.image >= d.num_images) { err = "texture image out of range"; return false; }
            if (t.filter < SOL_GPU_FILTER_NEAREST || t.filter > SOL_GPU_FILTER_BILINEAR) { err = "bad texture filter"; return false; }
            if (t.border < SOL_GPU_BORDER_CLAMP || t.border > SOL_GPU_BORDER_MIRROR) { err = "bad texture border"; return false; }
        }
    }

    // BSDFs.
    out.bsdfs.resize(d.num_bsdfs);
    for (uint32_t i = 0; i < d.num_bsdfs; ++i) {
        const SolGpuBsdf& b = d.bsdfs[i];
        DBsdf& o = out.bsdfs[i];
        o.kind = b.type; o.tex[0] = b.tex[0]; o.tex[1] = b.tex[1]; o.tex[2] = b.tex[2];
        o.a = b.a; o.b = b.b; o.pad = 0;
        switch (b.type) {
            case SOL_GPU_BSDF_DIFFUSE:
                if (!is_color_texture(d, b.tex[0])) { err = "diffuse kd must be a colour texture"; return false; }
                o.type = kTypeDiffuse; break;
            case SOL_GPU_BSDF_PHONG:
                if (!is_color_texture(d, b.tex[0]) || !is_texture(d, b.tex[1])) { err = "phong needs ks (colour) and ns"; return false; }
                o.type = kTypeGlossy; break;
            case SOL_GPU_BSDF_MIRROR:
                if (!is_color_texture(d, b.tex[0])) { err = "mirror ks must be a colour texture"; return false; }
                o.type = kTypeSpecular; break;
            case SOL_GPU_BSDF_GLASS:
                if (!is_color_texture(d, b.tex[0]) || !is_color_texture(d, b.tex[1]) || !is_texture(d, b.tex[2])) {
                    err = "glass needs ks, kt (colour) and eta"; return false;
                }
                o.type = kTypeSpecular; break;
            case SOL_GPU_BSDF_INTERP:
                break;
            default:
                err = "bad BSDF type"; return false;
        }
    }
    for (uint32_t i = 0; i < d.num_bsdfs; ++i) {
        const SolGpuBsdf& b = d.bsdfs[i];
        if (b.type != SOL_GPU_BSDF_INTERP) continue;
        if (!is_texture(d, b.tex[0]) || b.a < 0 || b.b < 0 || (uint32_t)b.a >= d.num_bsdfs || (uint32_t)b.b >= d.num_bsdfs) {
            err = "interp needs k and two BSDFs"; return false;
        }
        if (d.bsdfs[b.a].type == SOL_GPU_BSDF_INTERP || d.bsdfs[b.b].type == SOL_GPU_BSDF_INTERP) {
            err = "nested interp BSDFs are not supported"; return false;
        }
        // InterpBsdf::infer_type (src/bsdfs.cpp:226-230)
        int32_t ta = out.bsdfs[b.a].type, tb = out.bsdfs[b.b].type;
        out.bsdfs[i].type = (ta == kTypeDiffuse || tb == kTypeDiffuse) ? kTypeDiffuse
                          : (ta == kTypeGlossy || tb == kTypeGlossy) ? kTypeGlossy : kTypeSpecular;
    }

    // Lights.
    out.lights.resize(d.num_lights);
    for (uint32_t i = 0; i < d.num_lights; ++i) {
        const SolGpuLight& l = d.lights[i];
        DLight o{};
        o.kind = l.type;
        o.tex = l.intensity_tex;
        for (int k = 0; k < 3; ++k) {
            o.v0[k] = l.v0[k]; o.v1[k] = l.v1[k]; o.v2[k] = l.v2[k]; o.intensity[k] = l.intensity[k];
        }
        if (l.type == SOL_GPU_LIGHT_TRIANGLE) {
            if (!is_color_texture(d, l.intensity_tex)) { err = "triangle light needs a colour texture"; return false; }
            Vec3 a = ld3(l.v0), b = ld3(l.v1), c = ld3(l.v2);
            Vec3 n = triangle_normal(a, b, c);          // UniformTriangle (include/sol/shapes.h:53-55)
            o.n[0] = n.x; o.n[1] = n.y; o.n[2] = n.z;
            o.inv_area = 1.0f / triangle_area(a, b, c);
        } else if (l.type == SOL_GPU_LIGHT_SPHERE) {
            if (!is_color_texture(d, l.intensity_tex)) { err = "sphere light needs a colour texture"; return false; }
            o.radius = l.v1[0];
            o.inv_area = 1.0f / sphere_area(l.v1[0]);   // UniformSphere (shapes.h:66-68)
        } else if (l.type != SOL_GPU_LIGHT_POINT) {
            err = "bad light type"; return false;
        }
        out.lights[i] = o;
    }

    if (!host_bvh) {
        out.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return true;
    }

    // BVH: the caller's, or built here.
    bvh::Bvh tree;
    if (d.num_bvh_nodes > 0) {
        if (!d.bvh_nodes || !d.bvh_prim_indices) { err = "BVH arrays must not be NULL"; return false; }
        tree.nodes.resize(d.num_bvh_nodes);
        for (uint32_t i = 0; i < d.num_bvh_nodes; ++i) {
            const SolGpuBvhNode& n = d.bvh_nodes[i];
            bvh::Node& o = tree.nodes[i];
            for (int k = 0; k < 3; ++k) { o.box.lo[k] = n.lo[k]; o.box.hi[k] = n.hi[k]; }
            o.first = n.first; o.count = n.count;
            if (n.count == 0 && (uint64_t)n.first + 1 >= d.num_bvh_nodes) { err = "BVH child index out of range"; return false; }
            if (n.count > (uint32_t)kLeafMaxTris) { err = "BVH leaves may hold at most 8 primitives"; return false; }
            if (n.count > 0 && (uint64_t)n.first + n.count > nt) { err = "BVH leaf range out of range"; return false; }
        }
        tree.prim_indices.assign(d.bvh_prim_indices, d.bvh_prim_indices + nt);
        std::vector<uint8_t> seen(nt, 0);
        for (uint32_t p : tree.prim_indices) {
            if (p >= nt || seen[p]) { err = "BVH primitive indices are not a permutation"; return false; }
            seen[p] = 1;
        }
        // Every node must be reached once from the root (no cycles or sharing).
        std::vector<uint8_t> visited(d.num_bvh_nodes, 0);
        std::vector<uint32_t> stack{0};
        while (!stack.empty()) {
            uint32_t i = stack.back(); stack.pop_back();
            if (visited[i]) { err = "BVH is not a tree"; return false; }
            visited[i] = 1;
            if (tree.nodes[i].count == 0) { stack.push_back(tree.nodes[i].first); stack.push_back(tree.nodes[i].first + 1); }
        }
    } else if (nt > 0) {
        tree = build_mesh_bvh(d.vertices, d.indices, nt);
    }

    out.nodes.clear();
    out.tris.resize(nt);
    out.shade.resize(nt);
    if (nt > 0) {
        out.depth = tree.depth();
        if (out.depth > (uint32_t)kTraversalStack) {
            err = "BVH depth " + std::to_string(out.depth) + " exceeds the traversal stack (64)"; return false;
        }
        out.sah_cost = (float)tree.sah_cost();
        // Inner nodes in depth-first order (left subtree first).
        std::vector<int32_t> gpu_index(tree.nodes.size(), -1);
        auto ref_of = [&](uint32_t i) -> int32_t {
            const bvh::Node& n = tree.nodes[i];
            return n.is_leaf() ? leaf_ref(n.first, n.count) : gpu_index[i];
        };
        auto put_box = [](DNode& g, int c, const bvh::BBox& b) {
            float* xy = c == 0 ? g.b0 : g.b1;
            xy[0] = b.lo[0]; xy[1] = b.hi[0]; xy[2] = b.lo[1]; xy[3] = b.hi[1];
            g.b2[2 * c + 0] = b.lo[2]; g.b2[2 * c + 1] = b.hi[2];
        };
        if (tree.nodes[0].is_leaf()) {
            // A single leaf: a root whose two children are that leaf.
            DNode g{};
            put_box(g, 0, tree.nodes[0].box); put_box(g, 1, tree.nodes[0].box);
            g.ref[0] = g.ref[1] = ref_of(0);
            out.nodes.push_back(g);
            out.top_nodes = 1;
        } else {
            // Upper levels breadth first (whole levels while they fit in
            // kTopNodesMax), then every remaining subtree depth first (left
            // first).  Only the storage order changes: node 0 is the root and
            // each node keeps its children in the same order.
            std::vector<uint32_t> order;
            std::vector<uint32_t> level{0};
            while (!level.empty() && order.size() + level.size() <= kTopNodesMax) {
                std::vector<uint32_t> next;
                for (uint32_t i : level) {
                    gpu_index[i] = (int32_t)order.size();
                    order.push_back(i);
                    const bvh::Node& n = tree.nodes[i];
                    if (!tree.nodes[n.first].is_leaf()) next.push_back(n.first);
                    if (!tree.nodes[n.first + 1].is_leaf()) next.push_back(n.first + 1);
                }
                level.swap(next);
            }
            out.top_nodes = (uint32_t)order.size();
            for (uint32_t root : level) {
                std::vector<uint32_t> stack{root};
                while (!stack.empty()) {
                    uint32_t i = stack.back(); stack.pop_back();
                    gpu_index[i] = (int32_t)order.size();
                    order.push_back(i);
                    const bvh::Node& n = tree.nodes[i];
                    if (!tree.nodes[n.first + 1].is_leaf()) stack.push_back(n.first + 1);
                    if (!tree.nodes[n.first].is_leaf()) stack.push_back(n.first);
                }
            }
            out.nodes.resize(order.size());
            for (size_t k = 0; k < order.size(); ++k) {
                const bvh::Node& n = tree.nodes[order[k]];
                DNode& g = out.nodes[k];
                put_box(g, 0, tree.nodes[n.first].box);
                put_box(g, 1, tree.nodes[n.first + 1].box);
                g.ref[0] = ref_of(n.first);
                g.ref[1] = ref_of(n.first + 1);
                g.ref[2] = g.ref[3] = 0;
            }
        }
        // Triangles and shading records in leaf order.
        #pragma omp parallel for schedule(static)
        for (long j = 0; j < (long)nt; ++j) {
            uint32_t p = tree.prim_indices[j];
            uint32_t i0 = d.indices[3 * p], i1 = d.indices[3 * p + 1], i2 = d.indices[3 * p + 2];
            DTri& t = out.tris[j];
            for (int k = 0; k < 3; ++k) {
                t.v0[k] = d.vertices[3 * i0 + k]; t.v1[k] = d.vertices[3 * i1 + k]; t.v2[k] = d.vertices[3 * i2 + k];
            }
            t.prim = p;
            t.bsdf = d.tri_bsdf[p];
            t.light = d.tri_light[p];
            DTriShade& s = out.shade[j];
            for (int k = 0; k < 3; ++k) {
                s.n0[k] = d.normals[3 * i0 + k]; s.n1[k] = d.normals[3 * i1 + k]; s.n2[k] = d.normals[3 * i2 + k];
            }
            s.uv0x = d.tex_coords[2 * i0]; s.uv0y = d.tex_coords[2 * i0 + 1];
            s.uv1x = d.tex_coords[2 * i1]; s.uv1y = d.tex_coords[2 * i1 + 1];
            s.uv2x = d.tex_coords[2 * i2]; s.uv2y = d.tex_coords[2 * i2 + 1];
            s.bsdf = t.bsdf;
            s.light = t.light;
            const Vec3 fn = triangle_normal(vec3(t.v0[0], t.v0[1], t.v0[2]), vec3(t.v1[0], t.v1[1], t.v1[2]),
                                            vec3(t.v2[0], t.v2[1], t.v2[2]));
            s.fn[0] = fn.x; s.fn[1] = fn.y; s.fn[2] = fn.z;
        }
    } else {
        DNode g{};
        out.nodes.push_back(g);
    }
    out.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

}  // namespace sol_b200
