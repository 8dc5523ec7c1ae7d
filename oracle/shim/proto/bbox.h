// Test infrastructure (oracle): clean-room axis-aligned box.
#pragma once

#include <algorithm>
#include <limits>

#include "proto/vec.h"

namespace proto {

struct BBoxf {
    Vec3f min, max;
    static BBoxf empty() {
        float inf = std::numeric_limits<float>::infinity();
        return BBoxf{Vec3f(inf), Vec3f(-inf)};
    }
    BBoxf& extend(const BBoxf& o) {
        for (int k = 0; k < 3; ++k) { min[k] = std::min(min[k], o.min[k]); max[k] = std::max(max[k], o.max[k]); }
        return *this;
    }
    BBoxf& extend(const Vec3f& p) {
        for (int k = 0; k < 3; ++k) { min[k] = std::min(min[k], p[k]); max[k] = std::max(max[k], p[k]); }
        return *this;
    }
};

} // namespace proto
