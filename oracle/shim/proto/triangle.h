// Test infrastructure (oracle): clean-room triangles.  PrecomputedTrianglef
// keeps the three vertices and intersects with the shared watertight test.
#pragma once

#include <optional>
#include <utility>

#include "proto/bbox.h"
#include "proto/ray.h"
#include "proto/vec.h"

namespace proto {

struct Trianglef {
    Vec3f v0, v1, v2;
    Trianglef() = default;
    Trianglef(const Vec3f& a, const Vec3f& b, const Vec3f& c) : v0(a), v1(b), v2(c) {}
    Vec3f normal() const { return from_m(sol_b200::triangle_normal(to_m(v0), to_m(v1), to_m(v2))); }
    float area() const { return sol_b200::triangle_area(to_m(v0), to_m(v1), to_m(v2)); }
    Vec3f center() const { return from_m(sol_b200::triangle_center(to_m(v0), to_m(v1), to_m(v2))); }
    BBoxf bbox() const { return BBoxf::empty().extend(v0).extend(v1).extend(v2); }
    bool operator==(const Trianglef& o) const { return v0 == o.v0 && v1 == o.v1 && v2 == o.v2; }
    template <typename Hasher>
    Hasher& hash(Hasher& h) const { return v2.hash(v1.hash(v0.hash(h))); }
};

struct PrecomputedTrianglef {
    Vec3f v0, v1, v2;
    PrecomputedTrianglef() = default;
    PrecomputedTrianglef(const Vec3f& a, const Vec3f& b, const Vec3f& c) : v0(a), v1(b), v2(c) {}

    Vec3f normal() const { return from_m(sol_b200::triangle_normal(to_m(v0), to_m(v1), to_m(v2))); }

    /// On a hit strictly inside (ray.tmin, ray.tmax): shrinks ray.tmax to the hit
    /// distance and returns the barycentrics (u for v1, v for v2).
    std::optional<std::pair<float, float>> intersect(Rayf& ray) const {
        float t, u, v;
        if (!sol_b200::intersect_triangle(ray.shear, to_m(v0), to_m(v1), to_m(v2), ray.tmin, ray.tmax, &t, &u, &v))
            return std::nullopt;
        ray.tmax = t;
        return std::make_optional(std::make_pair(u, v));
    }
};

} // namespace proto
