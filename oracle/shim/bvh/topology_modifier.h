// Test infrastructure (oracle): holds the tree being optimised.
#pragma once

#include <vector>

#include "bvh/bvh.h"

namespace bvh {

template <typename B>
struct TopologyModifier {
    B& bvh;
    TopologyModifier(B& b, std::vector<size_t>&&) : bvh(b) {}
};
template <typename B> TopologyModifier(B&, std::vector<size_t>&&) -> TopologyModifier<B>;

} // namespace bvh
