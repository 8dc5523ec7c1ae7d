// Test infrastructure (oracle): clean-room sphere.
#pragma once

#include "proto/random.h"
#include "proto/vec.h"

namespace proto {

struct Spheref {
    Vec3f center;
    float radius;
    Spheref() = default;
    Spheref(const Vec3f& c, float r) : center(c), radius(r) {}
    float area() const { return sol_b200::sphere_area(radius); }
    bool operator==(const Spheref& o) const { return center == o.center && radius == o.radius; }
    template <typename Hasher>
    Hasher& hash(Hasher& h) const { return center.hash(h).combine(radius); }
};

} // namespace proto
