// Test infrastructure (oracle): SweepSahBuilder entry point over the product's
// full-sweep SAH builder.
#pragma once

#include <vector>

#include "bvh/bvh.h"
#include "proto/bbox.h"
#include "proto/vec.h"

namespace bvh {

template <typename B>
struct SweepSahBuilder {
    template <typename Scheduler, typename Executor>
    static B build(Scheduler&, Executor&, const proto::BBoxf&, const proto::BBoxf* bboxes,
                   const proto::Vec3f* centers, size_t count) {
        std::vector<sol_b200::bvh::BBox> boxes(count);
        std::vector<float> c(3 * count);
        for (size_t i = 0; i < count; ++i) {
            for (int k = 0; k < 3; ++k) {
                boxes[i].lo[k] = bboxes[i].min[k];
                boxes[i].hi[k] = bboxes[i].max[k];
                c[3 * i + k] = centers[i][k];
            }
        }
        return B::from(sol_b200::bvh::build_sweep_sah(boxes.data(), c.data(), count));
    }
};

} // namespace bvh
