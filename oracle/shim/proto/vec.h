// Test infrastructure (oracle): clean-room vectors with the interface SoL uses.
// Arithmetic is delegated to the shared host/device math so that the checker
// and the GPU round identically.
#pragma once

#include <cstddef>

#include "proto/hash.h"
#include "proto/utils.h"

namespace proto {

template <typename T, size_t N>
struct Vec {
    T values[N];

    Vec() = default;
    explicit Vec(T s) { for (size_t i = 0; i < N; ++i) values[i] = s; }
    template <typename... Args, typename = std::enable_if_t<sizeof...(Args) == N && (N > 1)>>
    Vec(Args... args) : values{static_cast<T>(args)...} {}

    T& operator[](size_t i) { return values[i]; }
    const T& operator[](size_t i) const { return values[i]; }

    Vec& operator+=(const Vec& o) { return *this = *this + o; }
    Vec& operator-=(const Vec& o) { return *this = *this - o; }
    Vec& operator*=(const Vec& o) { return *this = *this * o; }
    Vec& operator*=(T s) { return *this = *this * s; }

    friend Vec operator+(const Vec& a, const Vec& b) { Vec r; for (size_t i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; }
    friend Vec operator-(const Vec& a, const Vec& b) { Vec r; for (size_t i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; }
    friend Vec operator*(const Vec& a, const Vec& b) { Vec r; for (size_t i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; }
    friend Vec operator*(const Vec& a, T s) { Vec r; for (size_t i = 0; i < N; ++i) r[i] = a[i] * s; return r; }
    friend Vec operator*(T s, const Vec& a) { Vec r; for (size_t i = 0; i < N; ++i) r[i] = s * a[i]; return r; }
    friend Vec operator-(const Vec& a) { Vec r; for (size_t i = 0; i < N; ++i) r[i] = -a[i]; return r; }
    friend bool operator==(const Vec& a, const Vec& b) { for (size_t i = 0; i < N; ++i) if (!(a[i] == b[i])) return false; return true; }

    template <typename Hasher>
    Hasher& hash(Hasher& h) const { for (size_t i = 0; i < N; ++i) h.combine(values[i]); return h; }
};

using Vec2f = Vec<float, 2>;
using Vec3f = Vec<float, 3>;

inline sol_b200::Vec3 to_m(const Vec3f& v) { return sol_b200::vec3(v[0], v[1], v[2]); }
inline Vec3f from_m(const sol_b200::Vec3& v) { return Vec3f(v.x, v.y, v.z); }

inline float dot(const Vec3f& a, const Vec3f& b) { return sol_b200::dot(to_m(a), to_m(b)); }
inline Vec3f cross(const Vec3f& a, const Vec3f& b) { return from_m(sol_b200::cross(to_m(a), to_m(b))); }
inline float length(const Vec3f& a) { return sol_b200::length(to_m(a)); }
inline Vec3f normalize(const Vec3f& a) { return from_m(sol_b200::normalize(to_m(a))); }
inline float positive_dot(const Vec3f& a, const Vec3f& b) { return sol_b200::positive_dot(to_m(a), to_m(b)); }
inline float negative_dot(const Vec3f& a, const Vec3f& b) { return sol_b200::negative_dot(to_m(a), to_m(b)); }
inline Vec3f reflect(const Vec3f& d, const Vec3f& n) { return from_m(sol_b200::reflect(to_m(d), to_m(n))); }

inline Vec3f lerp(const Vec3f& a, const Vec3f& b, const Vec3f& c, float u, float v) {
    return from_m(sol_b200::lerp3(to_m(a), to_m(b), to_m(c), u, v));
}
inline Vec2f lerp(const Vec2f& a, const Vec2f& b, const Vec2f& c, float u, float v) {
    return Vec2f(sol_b200::lerp3(a[0], b[0], c[0], u, v), sol_b200::lerp3(a[1], b[1], c[1], u, v));
}
inline Vec2f clamp(const Vec2f& x, const Vec2f& a, const Vec2f& b) {
    return Vec2f(clamp(x[0], a[0], b[0]), clamp(x[1], a[1], b[1]));
}

/// 3x3 matrix stored by columns.
struct Mat3x3f {
    sol_b200::Mat3 m;
    Vec3f col(size_t i) const { return from_m(i == 0 ? m.c0 : (i == 1 ? m.c1 : m.c2)); }
    friend Vec3f operator*(const Mat3x3f& a, const Vec3f& v) { return from_m(sol_b200::mul(a.m, to_m(v))); }
};

inline Mat3x3f ortho_basis(const Vec3f& n) { return Mat3x3f{sol_b200::ortho_basis(to_m(n))}; }

} // namespace proto
