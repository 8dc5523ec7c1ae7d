// Forward-mode (dual number) versions of the shading math, for the tangent
// kernel.  Every dual value keeps its primal part `v` computed by the same float
// function the forward kernels call, so the replayed path takes exactly the
// forward render's decisions; the tangent part `d` carries the derivative along
// one direction in parameter space.
#pragma once

#include "../core/math.h"

namespace sol_b200 {

struct D  { float v, d; };
struct DV2 { Vec2 v, d; };
struct DV3 { Vec3 v, d; };
struct DRgb { Rgb v, d; };
struct DMat3 { Mat3 v, d; };

__device__ __forceinline__ D dconst(float x) { return D{x, 0.0f}; }
__device__ __forceinline__ DV3 dconst(Vec3 x) { return DV3{x, vec3(0.0f)}; }
__device__ __forceinline__ DRgb dconst(Rgb x) { return DRgb{x, rgb(0.0f)}; }

__device__ __forceinline__ D operator+(D a, D b) { return D{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ D operator-(D a, D b) { return D{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ D operator*(D a, D b) { return D{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ D operator/(D a, D b) { return D{a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
__device__ __forceinline__ D operator-(D a) { return D{-a.v, -a.d}; }

__device__ __forceinline__ DV3 operator+(DV3 a, DV3 b) { return DV3{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ DV3 operator-(DV3 a, DV3 b) { return DV3{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ DV3 operator-(DV3 a) { return DV3{-a.v, -a.d}; }
/// a * s with the primal as Vec3 * float.
__device__ __forceinline__ DV3 operator*(DV3 a, D s) { return DV3{a.v * s.v, a.d * s.v + a.v * s.d}; }
/// s * a with the primal as float * Vec3.
__device__ __forceinline__ DV3 operator*(D s, DV3 a) { return DV3{s.v * a.v, s.d * a.v + s.v * a.d}; }

__device__ __forceinline__ DRgb operator+(DRgb a, DRgb b) { return DRgb{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ DRgb operator*(DRgb a, DRgb b) { return DRgb{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ DRgb operator*(DRgb a, D s) { return DRgb{a.v * s.v, a.d * s.v + a.v * s.d}; }

__device__ __forceinline__ D ddot(DV3 a, DV3 b) { return D{dot(a.v, b.v), dot(a.d, b.v) + dot(a.v, b.d)}; }
__device__ __forceinline__ DV3 dcross(DV3 a, DV3 b) { return DV3{cross(a.v, b.v), cross(a.d, b.v) + cross(a.v, b.d)}; }
__device__ __forceinline__ D dlength(DV3 a) {
    const float l = length(a.v);
    return D{l, l > 0.0f ? dot(a.v, a.d) / l : 0.0f};
}
__device__ __forceinline__ DV3 dnormalize(DV3 a) {
    const Vec3 n = normalize(a.v);
    const float l = length(a.v);
    const Vec3 t = l > 0.0f ? (a.d - n * dot(n, a.d)) * (1.0f / l) : vec3(0.0f);
    return DV3{n, t};
}
__device__ __forceinline__ D dpositive_dot(DV3 a, DV3 b) {
    const D x = ddot(a, b);
    return x.v > 0.0f ? x : D{positive_dot(a.v, b.v), 0.0f};
}
__device__ __forceinline__ D dnegative_dot(DV3 a, DV3 b) {
    const D x = ddot(a, b);
    return x.v < 0.0f ? x : D{negative_dot(a.v, b.v), 0.0f};
}
__device__ __forceinline__ DV3 dreflect(DV3 d, DV3 n) {
    const D k = D{2.0f, 0.0f} * ddot(d, n);
    return DV3{reflect(d.v, n.v), d.d - (n.d * k.v + n.v * k.d)};
}
__device__ __forceinline__ D dsqrt(D x) {
    const float s = sqrt_(x.v);
    return D{s, s > 0.0f ? x.d * 0.5f / s : 0.0f};
}
__device__ __forceinline__ D dlog_(float x, float dx) { return D{0.0f, x > 0.0f ? dx / x : 0.0f}; }
/// x^y: the primal is pow_; d = x^y (y' ln x + y x'/x).
__device__ __forceinline__ D dpow(D x, D y) {
    const float p = pow_(x.v, y.v);
    if (!(x.v > 0.0f)) return D{p, 0.0f};
    const float lx = (float)log_pos_((double)x.v);
    return D{p, p * (y.d * lx + y.v * x.d / x.v)};
}
__device__ __forceinline__ D dluminance(DRgb c) { return D{luminance(c.v), luminance(c.d)}; }
__device__ __forceinline__ D dclamp(D x, float lo, float hi) {
    return x.v < lo ? D{lo, 0.0f} : (x.v > hi ? D{hi, 0.0f} : x);
}
__device__ __forceinline__ D dlerp(D a, D b, D t) {
    return D{lerp(a.v, b.v, t.v), a.d * (1.0f - t.v) + b.d * t.v + (b.v - a.v) * t.d};
}
__device__ __forceinline__ DRgb dlerp(DRgb a, DRgb b, D t) {
    return DRgb{lerp(a.v, b.v, t.v), rgb(a.d.r * (1.0f - t.v) + b.d.r * t.v + (b.v.r - a.v.r) * t.d,
                                         a.d.g * (1.0f - t.v) + b.d.g * t.v + (b.v.g - a.v.g) * t.d,
                                         a.d.b * (1.0f - t.v) + b.d.b * t.v + (b.v.b - a.v.b) * t.d)};
}
__device__ __forceinline__ DV3 dlerp3(Vec3 a, Vec3 b, Vec3 c, D u, D v) {
    // a (1 - u - v) + b u + c v, vertices constant
    return DV3{lerp3(a, b, c, u.v, v.v), (b - a) * u.d + (c - a) * v.d};
}
__device__ __forceinline__ DV2 dlerp3(Vec2 a, Vec2 b, Vec2 c, D u, D v) {
    return DV2{lerp3(a, b, c, u.v, v.v), vec2((b.x - a.x) * u.d + (c.x - a.x) * v.d, (b.y - a.y) * u.d + (c.y - a.y) * v.d)};
}

/// Duff et al.'s basis (math.h ortho_basis) with its derivative; the sign of n.z
/// is piecewise constant.
__device__ __forceinline__ DMat3 dortho_basis(DV3 n) {
    DMat3 m;
    m.v = ortho_basis(n.v);
    const float sign = copysign_(1.0f, n.v.z);
    const float a = -1.0f / (sign + n.v.z);
    const float da = n.d.z / ((sign + n.v.z) * (sign + n.v.z));
    const float b = n.v.x * n.v.y * a;
    const float db = n.d.x * n.v.y * a + n.v.x * n.d.y * a + n.v.x * n.v.y * da;
    m.d.c0 = vec3(sign * (2.0f * n.v.x * n.d.x * a + n.v.x * n.v.x * da), sign * db, -sign * n.d.x);
    m.d.c1 = vec3(db, 2.0f * n.v.y * n.d.y * a + n.v.y * n.v.y * da, -n.d.y);
    m.d.c2 = n.d;
    return m;
}
__device__ __forceinline__ DV3 dmul(const DMat3& m, DV3 x) {
    return DV3{mul(m.v, x.v), mul(m.d, x.v) + mul(m.v, x.d)};
}

}  // namespace sol_b200
