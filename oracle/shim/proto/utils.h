// Test infrastructure (oracle): clean-room stand-in for the part of proto/utils.h
// that SoL uses.  proto (madmann91/proto) is not vendored with SoL; these shims
// only exist so that SoL's own sources compile here as the reference checker.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <type_traits>

#include "core/math.h"

#define proto_always_inline inline __attribute__((always_inline))

namespace proto {

template <size_t Bits> struct SizedIntegerTypeSel {};
template <> struct SizedIntegerTypeSel<8>  { using Type = int8_t; };
template <> struct SizedIntegerTypeSel<16> { using Type = int16_t; };
template <> struct SizedIntegerTypeSel<32> { using Type = int32_t; };
template <> struct SizedIntegerTypeSel<64> { using Type = int64_t; };
template <size_t Bits> using SizedIntegerType = typename SizedIntegerTypeSel<Bits>::Type;

/// x below a gives a, above b gives b, otherwise x (the comparison order of the shared math).
template <typename T>
inline T clamp(T x, T a, T b) { return x < a ? a : (x > b ? b : x); }

inline float lerp(float a, float b, float t) { return sol_b200::lerp(a, b, t); }
inline float lerp(float a, float b, float c, float u, float v) { return sol_b200::lerp3(a, b, c, u, v); }

} // namespace proto
