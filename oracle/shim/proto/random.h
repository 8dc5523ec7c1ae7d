// Test infrastructure (oracle): clean-room sampling warps, delegating to the
// shared math so that the checker and the GPU draw identical directions.
#pragma once

#include <utility>

#include "proto/vec.h"

namespace proto {

inline std::pair<Vec3f, float> sample_cosine_hemisphere(float u, float v) {
    float pdf;
    Vec3f d = from_m(sol_b200::sample_cosine_hemisphere(u, v, &pdf));
    return {d, pdf};
}
inline float cosine_hemisphere_pdf(float c) { return sol_b200::cosine_hemisphere_pdf(c); }

inline std::pair<Vec3f, float> sample_cosine_power_hemisphere(float n, float u, float v) {
    float pdf;
    Vec3f d = from_m(sol_b200::sample_cosine_power_hemisphere(n, u, v, &pdf));
    return {d, pdf};
}
inline float cosine_power_hemisphere_pdf(float n, float c) { return sol_b200::cosine_power_hemisphere_pdf(n, c); }

inline std::pair<Vec3f, float> sample_uniform_sphere(float u, float v) {
    float pdf;
    Vec3f d = from_m(sol_b200::sample_uniform_sphere(u, v, &pdf));
    return {d, pdf};
}
template <typename T = float>
inline T uniform_sphere_pdf() { return sol_b200::uniform_sphere_pdf(); }

} // namespace proto
