// Test infrastructure (oracle): SequentialReinsertionOptimizer entry point over
// the product's reinsertion optimizer.
#pragma once

#include "bvh/topology_modifier.h"

namespace bvh {

template <typename B>
struct SequentialReinsertionOptimizer {
    template <typename M>
    static void optimize(M& modifier) {
        sol_b200::bvh::Bvh b = modifier.bvh.to_builder();
        sol_b200::bvh::ReinsertionOptimizer(b).optimize();
        modifier.bvh = B::from(b);
    }
};

} // namespace bvh
