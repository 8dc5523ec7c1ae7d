// Shared host/device math for the path-tracing hot path.
//
// SoL takes its vector, ray, triangle, sampling and hashing vocabulary from the
// external `proto` library (madmann91/proto), which is not vendored with SoL
// and whose version is not pinned anywhere in SoL's tree (src/CMakeLists.txt:27,
// README.md:13-15).  This header restates the subset that SoL's path tracer uses,
// written from the mathematics and from the published methods named beside each
// function.  The same source is compiled for the host (g++ -ffp-contract=off) and
// for sm_100a (nvcc -fmad=false, IEEE div/sqrt), so that the CPU checker and the
// GPU kernels produce bit-identical results: only +, -, *, /, sqrt, explicit
// double fused multiply-adds and float<->int conversions are used, all of which
// are correctly rounded on both sides.  Transcendentals (sin/cos/pow) are
// evaluated by our own polynomial and series code below rather than by a math
// library.
#pragma once

#include <stdint.h>
#include <string.h>

#include "pow_tables.h"

#if defined(__CUDACC__)
#define SOL_HD __host__ __device__ __forceinline__
#else
#define SOL_HD inline
#endif

namespace sol_b200 {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;   // same float as std::numbers::inv_pi_v<float>
constexpr float kFloatMax = 3.40282346638528859812e+38f;

SOL_HD uint32_t float_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}
SOL_HD float bits_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}
SOL_HD double bits_double(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d; memcpy(&d, &u, 8); return d;
#endif
}
SOL_HD uint64_t double_bits(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t u; memcpy(&u, &d, 8); return u;
#endif
}

SOL_HD float fmin_(float a, float b) { return a < b ? a : b; }
SOL_HD float fmax_(float a, float b) { return a > b ? a : b; }
SOL_HD float fabs_(float a) { return bits_float(float_bits(a) & 0x7fffffffu); }
SOL_HD float copysign_(float mag, float sgn) {
    return bits_float((float_bits(mag) & 0x7fffffffu) | (float_bits(sgn) & 0x80000000u));
}
SOL_HD float sqrt_(float x) {
#if defined(__CUDA_ARCH__)
    return __fsqrt_rn(x);
#else
    return __builtin_sqrtf(x);
#endif
}
SOL_HD float floor_(float x) {
#if defined(__CUDA_ARCH__)
    return floorf(x);
#else
    return __builtin_floorf(x);
#endif
}
/// Clamp with the comparison order used throughout: below `lo` gives `lo`, above
/// `hi` gives `hi`, otherwise (including NaN) the value itself.
SOL_HD float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
SOL_HD int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

// ---------------------------------------------------------------------------
// Vectors
// ---------------------------------------------------------------------------

struct Vec2 { float x, y; };
struct Vec3 { float x, y, z; };

SOL_HD Vec2 vec2(float x, float y) { Vec2 r; r.x = x; r.y = y; return r; }
SOL_HD Vec3 vec3(float x, float y, float z) { Vec3 r; r.x = x; r.y = y; r.z = z; return r; }
SOL_HD Vec3 vec3(float s) { return vec3(s, s, s); }

SOL_HD Vec3 operator+(Vec3 a, Vec3 b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
SOL_HD Vec3 operator-(Vec3 a, Vec3 b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
SOL_HD Vec3 operator-(Vec3 a) { return vec3(-a.x, -a.y, -a.z); }
SOL_HD Vec3 operator*(Vec3 a, Vec3 b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
SOL_HD Vec3 operator*(Vec3 a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
SOL_HD Vec3 operator*(float s, Vec3 a) { return vec3(s * a.x, s * a.y, s * a.z); }

SOL_HD float dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SOL_HD Vec3 cross(Vec3 a, Vec3 b) {
    return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SOL_HD float length(Vec3 a) { return sqrt_(dot(a, a)); }
SOL_HD Vec3 normalize(Vec3 a) { return a * (1.0f / length(a)); }
SOL_HD float positive_dot(Vec3 a, Vec3 b) { return fmax_(dot(a, b), 0.0f); }
SOL_HD float negative_dot(Vec3 a, Vec3 b) { return fmin_(dot(a, b), 0.0f); }
SOL_HD float comp(Vec3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

/// Mirror of `d` about the plane orthogonal to `n`: d - 2 (d.n) n.
SOL_HD Vec3 reflect(Vec3 d, Vec3 n) { return d - n * (2.0f * dot(d, n)); }

/// Linear interpolation a + (b - a) t, written as a (1 - t) + b t.
SOL_HD float lerp(float a, float b, float t) { return a * (1.0f - t) + b * t; }
/// Barycentric interpolation a (1 - u - v) + b u + c v.
SOL_HD float lerp3(float a, float b, float c, float u, float v) {
    return a * (1.0f - u - v) + b * u + c * v;
}
SOL_HD Vec3 lerp3(Vec3 a, Vec3 b, Vec3 c, float u, float v) {
    return vec3(lerp3(a.x, b.x, c.x, u, v), lerp3(a.y, b.y, c.y, u, v), lerp3(a.z, b.z, c.z, u, v));
}
SOL_HD Vec2 lerp3(Vec2 a, Vec2 b, Vec2 c, float u, float v) {
    return vec2(lerp3(a.x, b.x, c.x, u, v), lerp3(a.y, b.y, c.y, u, v));
}

/// 3x3 matrix stored by columns; `mul(m, v)` = c0 v.x + c1 v.y + c2 v.z.
struct Mat3 { Vec3 c0, c1, c2; };
SOL_HD Vec3 mul(const Mat3& m, Vec3 v) {
    return vec3(m.c0.x * v.x + m.c1.x * v.y + m.c2.x * v.z,
                m.c0.y * v.x + m.c1.y * v.y + m.c2.y * v.z,
                m.c0.z * v.x + m.c1.z * v.y + m.c2.z * v.z);
}

/// Orthonormal basis whose third column is the unit vector `n`
/// (Duff, Burgess, Christensen, Hery, Kensler, Liani, Villemin:
/// "Building an Orthonormal Basis, Revisited", JCGT 6(1), 2017).
SOL_HD Mat3 ortho_basis(Vec3 n) {
    float sign = copysign_(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    Mat3 m;
    m.c0 = vec3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    m.c1 = vec3(b, sign + n.y * n.y * a, -n.y);
    m.c2 = n;
    return m;
}

// ---------------------------------------------------------------------------
// Colour (RGB, FP32) — SoL's RgbColor arithmetic (include/sol/color.h:11-80)
// ---------------------------------------------------------------------------

struct Rgb { float r, g, b; };
SOL_HD Rgb rgb(float r, float g, float b) { Rgb c; c.r = r; c.g = g; c.b = b; return c; }
SOL_HD Rgb rgb(float s) { return rgb(s, s, s); }
SOL_HD Rgb operator+(Rgb a, Rgb b) { return rgb(a.r + b.r, a.g + b.g, a.b + b.b); }
SOL_HD Rgb operator*(Rgb a, Rgb b) { return rgb(a.r * b.r, a.g * b.g, a.b * b.b); }
SOL_HD Rgb operator*(Rgb a, float s) { return rgb(a.r * s, a.g * s, a.b * s); }
/// include/sol/color.h:58 — Rec.709 luminance.
SOL_HD float luminance(Rgb c) { return c.r * 0.2126f + c.g * 0.7152f + c.b * 0.0722f; }
SOL_HD Rgb lerp(Rgb a, Rgb b, float t) { return rgb(lerp(a.r, b.r, t), lerp(a.g, b.g, t), lerp(a.b, b.b, t)); }

// ---------------------------------------------------------------------------
// Transcendentals (own implementations; identical on host and device)
// ---------------------------------------------------------------------------

/// sin(2 pi t) and cos(2 pi t) for t in [0, 1] (the only angles SoL's samplers
/// produce).  4t is split exactly into a quadrant q and a remainder r in
/// [-1/2, 1/2]; sin/cos of r pi/2 come from their Taylor series (degree 9 and
/// 10, truncation error below 4e-8 on that interval), evaluated by Horner's rule.
SOL_HD void sincos_turns(float t, float* s, float* c) {
    float x = 4.0f * t;
    float qf = floor_(x + 0.5f);
    float r = x - qf;
    int q = ((int)qf) & 3;
    float r2 = r * r;
    float sp = r * (1.5707963705062866f + r2 * (-0.6459640860557556f + r2 * (0.07969262450933456f +
               r2 * (-0.004681753925979137f + r2 * 0.00016044118092395365f))));
    float cp = 1.0f + r2 * (-1.2337005138397217f + r2 * (0.25366950035095215f + r2 * (-0.020863480865955353f +
               r2 * (0.0009192602592520416f + r2 * -2.520204179745633e-05f))));
    float ss, cc;
    switch (q) {
        case 0:  ss = sp;  cc = cp;  break;
        case 1:  ss = cp;  cc = -sp; break;
        case 2:  ss = -sp; cc = -cp; break;
        default: ss = -cp; cc = sp;  break;
    }
    *s = ss; *c = cc;
}

/// Fused multiply-add a * b + c with one rounding (IEEE 754 fusedMultiplyAdd):
/// the same bits on the host (the FMA instruction, or libm's correctly rounded
/// fma) and on the device.
SOL_HD double fma_(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return __builtin_fma(a, b, c);
#endif
}

// Constant tables of pow_ (generated by gen_pow_tables.py, which states how
// each value is computed); the device reads its copies through the read-only
// data cache.
#if defined(__CUDACC__)
__device__ const double kPowInvDev[64] = SOL_POW_INV;
__device__ const double kPowLogInvDev[64] = SOL_POW_LOG_INV;
__device__ const double kPowExp2Dev[64] = SOL_POW_EXP2;
#endif
inline constexpr double kPowInvHost[64] = SOL_POW_INV;
inline constexpr double kPowLogInvHost[64] = SOL_POW_LOG_INV;
inline constexpr double kPowExp2Host[64] = SOL_POW_EXP2;
#if defined(__CUDA_ARCH__)
#define SOL_POW_TAB(name, j) __ldg(&name##Dev[j])
#else
#define SOL_POW_TAB(name, j) name##Host[j]
#endif

/// e^z for z in [-800, 800] (clamped outside; 0 below): z = (64 n + j) ln2/64 + r
/// with k = 64 n + j the nearest integer to 64 z / ln 2 (found by adding
/// 1.5 * 2^52, which leaves k in the low bits) and |r| <= ln2/128; then
/// e^z = 2^n * 2^(j/64) * e^r, with e^r - 1 from its Taylor series to degree 6
/// (truncation below 2^-54) and ln2/64 split in two so that k ln2/64 is exact.
SOL_HD double exp_(double z) {
    if (z < -800.0) return 0.0;
    if (z > 800.0) z = 800.0;
    const double shifter = 6755399441055744.0;   // 1.5 * 2^52
    const double shifted = z * SOL_POW_INV_LN2_64 + shifter;
    const double kd = shifted - shifter;
    const int k = (int)(uint32_t)double_bits(shifted);
    double r = fma_(-kd, SOL_POW_LN2_64_HI, z);
    r = fma_(-kd, SOL_POW_LN2_64_LO, r);
    double q = fma_(r, 1.0 / 720.0, 1.0 / 120.0);
    q = fma_(q, r, 1.0 / 24.0);
    q = fma_(q, r, 1.0 / 6.0);
    q = fma_(q, r, 0.5);
    const double em1 = fma_(q, r * r, r);
    const double t = SOL_POW_TAB(kPowExp2, k & 63);
    const double p = fma_(t, em1, t);
    // 2^n in two halves so that neither factor under- or overflows.
    const int n = k >> 6;
    const int n1 = n / 2, n2 = n - n1;
    return p * bits_double((uint64_t)(n1 + 1023) << 52) * bits_double((uint64_t)(n2 + 1023) << 52);
}

/// ln x for a positive, finite float, in double precision: x = 2^e m with m in
/// [1, 2) taken from the float's bits; m times the reciprocal of the midpoint
/// of its 64th of [1, 2) is 1 + r with |r| <= 2^-7, so ln m = ln(1 + r) -
/// ln(that reciprocal) (tabulated), ln(1 + r) from its series to degree 7
/// (truncation below 2^-59), and e ln2 with ln2 split in two so that e ln2 is
/// exact in its head.
SOL_HD double log_float_(float x) {
    uint32_t bits = float_bits(x);
    int e = (int)(bits >> 23) - 127;
    if ((bits >> 23) == 0u) {   // subnormal: scale into the normal range (exact)
        bits = float_bits(x * 8388608.0f);
        e = (int)(bits >> 23) - 150;
    }
    const uint32_t mant = bits & 0x7fffffu;
    const int j = (int)(mant >> 17);
    const double m = bits_double(0x3ff0000000000000ull | ((uint64_t)mant << 29));
    const double r = fma_(m, SOL_POW_TAB(kPowInv, j), -1.0);
    double q = fma_(r, 1.0 / 7.0, -1.0 / 6.0);
    q = fma_(q, r, 1.0 / 5.0);
    q = fma_(q, r, -0.25);
    q = fma_(q, r, 1.0 / 3.0);
    q = fma_(q, r, -0.5);
    const double l1p = fma_(q, r * r, r);
    const double ed = (double)e;
    return (ed * SOL_POW_LN2_HI + SOL_POW_TAB(kPowLogInv, j)) + fma_(ed, SOL_POW_LN2_LO, l1p);
}

/// x^y for x >= 0 (negative zero treated as zero), evaluated as e^(y ln x) in
/// double precision (relative error near 2^-50 for |y ln x| < 100) and rounded
/// once to float.  Special cases follow C's pow for non-negative bases: x^0 = 1,
/// 1^y = 1, 0^y = 0 (y > 0) or +inf (y < 0).
SOL_HD float pow_(float x, float y) {
    if (y == 0.0f || x == 1.0f) return 1.0f;
    if (x != x || y != y) return x + y;
    if (x <= 0.0f) {
        if (x == 0.0f) return y > 0.0f ? 0.0f : bits_float(0x7f800000u);
        return bits_float(0x7fc00000u);
    }
    if (float_bits(x) == 0x7f800000u) return y > 0.0f ? x : 0.0f;
    return (float)exp_((double)y * log_float_(x));
}

// ---------------------------------------------------------------------------
// Sampling warps (SoL calls these through proto/random.h)
// ---------------------------------------------------------------------------

SOL_HD float cosine_hemisphere_pdf(float c) { return c * kInvPi; }

/// Cosine-weighted hemisphere direction around +z (Malley's method):
/// phi = 2 pi u, cos(theta) = sqrt(1 - v), pdf = cos(theta)/pi.
SOL_HD Vec3 sample_cosine_hemisphere(float u, float v, float* pdf) {
    float s, c;
    sincos_turns(u, &s, &c);
    float cos_t = sqrt_(1.0f - v);
    float sin_t = sqrt_(v);
    *pdf = cosine_hemisphere_pdf(cos_t);
    return vec3(c * sin_t, s * sin_t, cos_t);
}

/// pdf of the cosine-power lobe: (n + 1)/(2 pi) cos^n.
SOL_HD float cosine_power_hemisphere_pdf(float n, float c) {
    return (n + 1.0f) * pow_(c, n) * (0.5f * kInvPi);
}

/// Cosine-power lobe around +z: cos(theta) = v^(1/(n+1)), phi = 2 pi u.
SOL_HD Vec3 sample_cosine_power_hemisphere(float n, float u, float v, float* pdf) {
    float s, c;
    sincos_turns(u, &s, &c);
    float cos_t = pow_(v, 1.0f / (n + 1.0f));
    float sin_t = sqrt_(fmax_(0.0f, 1.0f - cos_t * cos_t));
    *pdf = cosine_power_hemisphere_pdf(n, cos_t);
    return vec3(c * sin_t, s * sin_t, cos_t);
}

SOL_HD float uniform_sphere_pdf() { return 0.25f * kInvPi; }

/// Uniform direction on the unit sphere: cos(theta) = 2v - 1, phi = 2 pi u.
SOL_HD Vec3 sample_uniform_sphere(float u, float v, float* pdf) {
    float s, c;
    sincos_turns(u, &s, &c);
    float cos_t = 2.0f * v - 1.0f;
    float sin_t = sqrt_(fmax_(0.0f, 1.0f - cos_t * cos_t));
    *pdf = uniform_sphere_pdf();
    return vec3(c * sin_t, s * sin_t, cos_t);
}

// ---------------------------------------------------------------------------
// Random numbers: SoL's PcgGenerator (include/sol/samplers.h:20-46) behind
// std::uniform_real_distribution<float>(0, 1) (samplers.h:49-62)
// ---------------------------------------------------------------------------

struct Pcg {
    uint64_t state;
    /// PCG-XSH-RR 64/32 step with multiplier 6364136223846793005 and increment 1.
    SOL_HD uint32_t next_u32() {
        uint64_t old = state;
        state = old * 6364136223846793005ull + 1ull;
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
    }
    /// samplers.h:30-35: zero state, one step, add the seed, one step.
    SOL_HD void seed(uint64_t init) {
        state = 0;
        next_u32();
        state += init;
        next_u32();
    }
    /// One 32-bit output mapped to [0, 1): float(u) * 2^-32 with round-to-nearest
    /// conversion, and results that round up to 1 replaced by the largest float
    /// below 1.  This is what libstdc++'s uniform_real_distribution<float> returns
    /// for a 32-bit generator; checked against the host library bit for bit.
    SOL_HD float next_float() {
        float f = (float)next_u32() * 2.3283064365386963e-10f;
        return f < 1.0f ? f : 0.99999994039535522461f;
    }
};

SOL_HD Pcg make_pcg(uint64_t seed) { Pcg p; p.seed(seed); return p; }

/// 32-bit FNV-1a (Fowler, Noll, Vo) over the eight little-endian bytes of each
/// 64-bit value, offset basis 2166136261, prime 16777619.  SoL derives one
/// seed per (pixel, sample) from `fnv::Hasher().combine(x).combine(y).combine(frame)`
/// (include/sol/renderer.h:44-46).
SOL_HD uint32_t fnv_combine_u64(uint32_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (uint32_t)((v >> (8 * i)) & 0xffu);
        h *= 16777619u;
    }
    return h;
}
SOL_HD uint32_t pixel_seed(uint64_t frame, uint64_t x, uint64_t y) {
    uint32_t h = 2166136261u;
    h = fnv_combine_u64(h, x);
    h = fnv_combine_u64(h, y);
    h = fnv_combine_u64(h, frame);
    return h;
}

// ---------------------------------------------------------------------------
// Rays and watertight ray/triangle intersection
// ---------------------------------------------------------------------------

/// Per-ray constants of the watertight test (Woop, Benthin, Wald: "Watertight
/// Ray/Triangle Intersection", JCGT 2(1), 2013): the dominant axis kz, the two
/// others kx, ky (swapped when dir[kz] < 0 to keep the winding), and the shear.
struct RayShear {
    Vec3 org;
    int kx, ky, kz;
    float sx, sy, sz;
};

SOL_HD RayShear make_shear(Vec3 org, Vec3 dir) {
    RayShear r;
    r.org = org;
    float ax = fabs_(dir.x), ay = fabs_(dir.y), az = fabs_(dir.z);
    int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    float dz = comp(dir, kz);
    if (dz < 0.0f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.sx = comp(dir, kx) / dz;
    r.sy = comp(dir, ky) / dz;
    r.sz = 1.0f / dz;
    return r;
}

/// Signed edge functions U (opposite v0), V (opposite v1), W (opposite v2) in
/// the sheared ray space; falls back to double precision when one is exactly
/// zero, as the watertight method prescribes.
SOL_HD void edge_functions(const RayShear& r, Vec3 a, Vec3 b, Vec3 c,
                           float* U, float* V, float* W,
                           float* az, float* bz, float* cz) {
    float a_kz = comp(a, r.kz), b_kz = comp(b, r.kz), c_kz = comp(c, r.kz);
    float Ax = comp(a, r.kx) - r.sx * a_kz;
    float Ay = comp(a, r.ky) - r.sy * a_kz;
    float Bx = comp(b, r.kx) - r.sx * b_kz;
    float By = comp(b, r.ky) - r.sy * b_kz;
    float Cx = comp(c, r.kx) - r.sx * c_kz;
    float Cy = comp(c, r.ky) - r.sy * c_kz;
    float u = Cx * By - Cy * Bx;
    float v = Ax * Cy - Ay * Cx;
    float w = Bx * Ay - By * Ax;
    if (u == 0.0f || v == 0.0f || w == 0.0f) {
        double cxby = (double)Cx * (double)By, cybx = (double)Cy * (double)Bx;
        double axcy = (double)Ax * (double)Cy, aycx = (double)Ay * (double)Cx;
        double bxay = (double)Bx * (double)Ay, byax = (double)By * (double)Ax;
        u = (float)(cxby - cybx);
        v = (float)(axcy - aycx);
        w = (float)(bxay - byax);
    }
    *U = u; *V = v; *W = w;
    *az = r.sz * a_kz; *bz = r.sz * b_kz; *cz = r.sz * c_kz;
}

/// Watertight intersection of a ray with triangle (v0, v1, v2), both sides.
/// On a hit strictly inside (tmin, tmax) returns true with the distance `t`
/// (in units of the ray direction) and barycentrics u (weight of v1) and v
/// (weight of v2).
SOL_HD bool intersect_triangle(const RayShear& r, Vec3 v0, Vec3 v1, Vec3 v2,
                               float tmin, float tmax, float* t_out, float* u_out, float* v_out) {
    Vec3 a = v0 - r.org, b = v1 - r.org, c = v2 - r.org;
    float U, V, W, az, bz, cz;
    edge_functions(r, a, b, c, &U, &V, &W, &az, &bz, &cz);
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float T = U * az + V * bz + W * cz;
    float rcp = 1.0f / det;
    float t = T * rcp;
    if (!(t > tmin && t < tmax)) return false;
    *t_out = t;
    *u_out = V * rcp;
    *v_out = W * rcp;
    return true;
}

/// Surface area of a sphere of radius r: 4 pi r^2.
SOL_HD float sphere_area(float r) { return 4.0f * kPi * r * r; }

/// Centroid of a triangle, (v0 + v1 + v2) / 3.
SOL_HD Vec3 triangle_center(Vec3 v0, Vec3 v1, Vec3 v2) { return (v0 + v1 + v2) * (1.0f / 3.0f); }

/// Geometric normal of a triangle: normalize((v1 - v0) x (v2 - v0)).
SOL_HD Vec3 triangle_normal(Vec3 v0, Vec3 v1, Vec3 v2) { return normalize(cross(v1 - v0, v2 - v0)); }
/// Area of a triangle: |(v1 - v0) x (v2 - v0)| / 2.
SOL_HD float triangle_area(Vec3 v0, Vec3 v1, Vec3 v2) { return 0.5f * length(cross(v1 - v0, v2 - v0)); }

/// Reciprocal direction for slab tests; zero components are replaced by a tiny
/// value of the same sign so that no 0 * inf products appear.
SOL_HD Vec3 safe_inverse(Vec3 d) {
    const float eps = 1e-30f;
    float x = fabs_(d.x) > eps ? d.x : copysign_(eps, d.x);
    float y = fabs_(d.y) > eps ? d.y : copysign_(eps, d.y);
    float z = fabs_(d.z) > eps ? d.z : copysign_(eps, d.z);
    return vec3(1.0f / x, 1.0f / y, 1.0f / z);
}

/// Widening factor applied to the exit distance of every slab test so that
/// rounding in the box test never culls a box that the exact ray touches
/// (Ize: "Robust BVH Ray Traversal", JCGT 2(2), 2013: 1 + 2 gamma(3)).
constexpr float kSlabWiden = 1.0000008f;

}  // namespace sol_b200
