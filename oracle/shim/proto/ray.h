// Test infrastructure (oracle): clean-room ray.  Rays keep the shear constants
// of the watertight triangle test, computed once at construction.
#pragma once

#include "proto/vec.h"

namespace proto {

struct Rayf {
    Vec3f org, dir;
    float tmin, tmax;
    sol_b200::RayShear shear;

    Rayf() = default;
    Rayf(const Vec3f& o, const Vec3f& d, float t0 = 0.0f, float t1 = sol_b200::kFloatMax)
        : org(o), dir(d), tmin(t0), tmax(t1), shear(sol_b200::make_shear(to_m(o), to_m(d))) {}

    /// Segment from p to q, shortened by `offset` at both ends (in units of q - p).
    static Rayf between_points(const Vec3f& p, const Vec3f& q, float offset) {
        return Rayf(p, q - p, offset, 1.0f - offset);
    }

    Vec3f point_at(float t) const { return org + dir * t; }
};

} // namespace proto
