// Float32 vector / quaternion arithmetic for the arena tick, host+device.
//
// Every operation is written out in the order the reference evaluates it (reference
// include/rocketgpu/detail/math.hpp:605-1400): the device build uses --fmad=false and IEEE division / square root, the
// host build -ffp-contract=off, so each float op rounds identically on both and matches the reference's CPU path bit
// for bit. Do not "simplify" expressions here: (a*b)*c and a*(b*c) differ.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define RG_HD __host__ __device__ __forceinline__
#define RG_HDI __host__ __device__ inline
// Large phase functions stay out of line so their stack frames share one region instead of each holding its own
// slice of the caller's frame: the tick touches fewer distinct local-memory lines per thread.
#define RG_NOINL static __host__ __device__ __noinline__
#else
#define RG_HD inline
#define RG_HDI inline
#define RG_NOINL static inline
#endif

namespace rg {

struct V3 {
    float x, y, z;
};
struct Q4 {
    float w, x, y, z;
};

RG_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
RG_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
RG_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
RG_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
RG_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
RG_HD V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
RG_HD V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
RG_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// (x*x + y*y) + z*z grouping used by several reference call sites
RG_HD float dot_l(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
RG_HD V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
RG_HD float len2(V3 a) { return dot(a, a); }
RG_HD float len(V3 a) { return sqrtf(dot(a, a)); }
RG_HD bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
RG_HD float fmin_(float a, float b) { return a < b ? a : b; }
RG_HD float fmax_(float a, float b) { return a > b ? a : b; }
RG_HD float fabs_(float v) { return v >= 0.0f ? v : -v; }
RG_HD V3 vmin(V3 a, V3 b) { return V3{fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)}; }
RG_HD V3 vmax(V3 a, V3 b) { return V3{fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)}; }

// x / 50 (uu -> bt). The reference's device build emulates this division with an FMA; an IEEE division is the
// correctly rounded value the CPU path computes, so the device simply divides.
RG_HD float div50(float x) { return x / 50.0f; }
RG_HD V3 uu_to_bt_div(V3 v) { return V3{div50(v.x), div50(v.y), div50(v.z)}; }

// Float-to-integer conversions as the reference's x86 build performs them (cvttss2si / cvttsd2si): truncation toward
// zero, and the "integer indefinite" INT32_MIN for NaN and for values outside int32. CUDA's conversions saturate and
// turn NaN into 0, so the tick converts through these wherever a value may be NaN or out of range (a car whose state
// went NaN, a huge angle); in range they are plain truncations on both.
RG_HD int32_t x86_f2i(float x) {
    return (x >= -2147483648.0f && x < 2147483648.0f) ? static_cast<int32_t>(x) : INT32_MIN;
}
RG_HD int32_t x86_d2i(double x) {
    return (x > -2147483649.0 && x < 2147483648.0) ? static_cast<int32_t>(x) : INT32_MIN;
}

// Index of the lowest set bit (x != 0).
RG_HD int ctz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs(static_cast<int>(x)) - 1;
#else
    return __builtin_ctz(x);
#endif
}

RG_HD int ctz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __ffsll(static_cast<long long>(x)) - 1;
#else
    return __builtin_ctzll(x);
#endif
}

RG_HD uint32_t f2u(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}
RG_HD float u2f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// 3x3 (rows) times vector, reference Mul3x3Vec: each row dotted (x*x + y*y) + z*z.
RG_HD V3 mul3(V3 r0, V3 r1, V3 r2, V3 v) {
    return V3{(r0.x * v.x + r0.y * v.y) + r0.z * v.z, (r1.x * v.x + r1.y * v.y) + r1.z * v.z,
              (r2.x * v.x + r2.y * v.y) + r2.z * v.z};
}

// --- sin / cos: the reference's UCRT-equivalent single precision sine and cosine for |x| below 2^24-ish, evaluated
// in double with fused multiply-adds (reference math.hpp:17-63). Arguments on the tick's paths stay far below the
// limits; larger ones fall back to the C library, as the reference's host build does.
RG_HDI double ucrt_sin_poly(double r) {
    const double r2 = r * r;
    double p = fma(r2, 0x1.71de3a556c734p-19, -0x1.a01a01a01a01ap-13);
    p = fma(p, r2, 0x1.1111111111111p-7);
    p = fma(p, r2, -0x1.5555555555555p-3);
    return fma(p, r * r2, r);
}
RG_HDI double ucrt_cos_poly(double r) {
    const double r2 = r * r;
    const double base = 1.0 - r2 * 0.5;
    double p = fma(r2, -0x1.27e4fb7789f5cp-22, 0x1.a01a01a01a019p-16);
    p = fma(p, r2, -0x1.6c16c16c16c16p-10);
    p = fma(p, r2, 0x1.5555555555555p-5);
    return fma(p, r2 * r2, base);
}
RG_HDI double ucrt_reduce(double a, int* quadrant) {
    const int n = x86_d2i(fma(a, 0x1.45f306dc9c883p-1, 0.5));
    const double nd = static_cast<double>(n);
    const double r1 = fma(-nd, 0x1.921fb54400000p+0, a);
    *quadrant = n & 3;
    return r1 - nd * 0x1.0b4611a626331p-34;
}
RG_HDI float ucrt_sinf(float x) {
    const uint32_t ax = f2u(x) & 0x7fffffffu;
    if (ax < 0x39000000u) return x;
    const double d = static_cast<double>(x);
    if (ax <= 0x3f490fdbu) {
        if (ax < 0x3c000000u) return static_cast<float>(fma(-((d * d) * d), 0x1.5555555555555p-3, d));
        return static_cast<float>(ucrt_sin_poly(d));
    }
    int q = 0;
    const double r = ucrt_reduce(fabs(d), &q);
    const double y = (q & 1) ? ucrt_cos_poly(r) : ucrt_sin_poly(r);
    return static_cast<float>(((q >= 2) != (x < 0.0f)) ? -y : y);
}
RG_HDI float ucrt_cosf(float x) {
    const uint32_t ax = f2u(x) & 0x7fffffffu;
    if (ax < 0x39000000u) return 1.0f;
    const double d = static_cast<double>(x);
    if (ax <= 0x3f490fdbu) {
        if (ax < 0x3c000000u) return static_cast<float>(fma(-(d * 0.5), d, 1.0));
        return static_cast<float>(ucrt_cos_poly(d));
    }
    int q = 0;
    const double r = ucrt_reduce(fabs(d), &q);
    const double y = (q & 1) ? ucrt_sin_poly(r) : ucrt_cos_poly(r);
    return static_cast<float>((q == 1 || q == 2) ? -y : y);
}
constexpr uint32_t kSinLimitBits = 0x4b800456u;
constexpr uint32_t kCosLimitBits = 0x4f490fdbu;
RG_HDI float game_sinf(float x) { return (f2u(x) & 0x7fffffffu) < kSinLimitBits ? ucrt_sinf(x) : sinf(x); }
RG_HDI float game_cosf(float x) { return (f2u(x) & 0x7fffffffu) < kCosLimitBits ? ucrt_cosf(x) : cosf(x); }

// --- quaternion <-> basis (reference math.hpp:1092-1200)
RG_HDI Q4 game_rot_from_basis(V3 fwd, V3 right, V3 up) {
    const float m00 = fwd.x, m01 = right.x, m02 = up.x;
    const float m10 = fwd.y, m11 = right.y, m12 = up.y;
    const float m20 = fwd.z, m21 = right.z, m22 = up.z;
    const float trace = (m00 + m11) + m22;
    if (trace > 0.0f) {
        float s = sqrtf(trace + 1.0f);
        const float w = s * 0.5f;
        s = 0.5f / s;
        return Q4{w, (m21 - m12) * s, (m02 - m20) * s, (m10 - m01) * s};
    }
    // the largest diagonal element picks the component computed from the square root
    if (m00 < m11 ? m11 < m22 : m00 < m22) {
        float s = sqrtf(((m22 - m00) - m11) + 1.0f);
        const float z = s * 0.5f;
        s = 0.5f / s;
        return Q4{(m10 - m01) * s, (m02 + m20) * s, (m12 + m21) * s, z};
    }
    if (m00 < m11) {
        float s = sqrtf(((m11 - m22) - m00) + 1.0f);
        const float y = s * 0.5f;
        s = 0.5f / s;
        return Q4{(m02 - m20) * s, (m01 + m10) * s, y, (m21 + m12) * s};
    }
    float s = sqrtf(((m00 - m11) - m22) + 1.0f);
    const float x = s * 0.5f;
    s = 0.5f / s;
    return Q4{(m21 - m12) * s, x, (m10 + m01) * s, (m20 + m02) * s};
}
RG_HDI void game_basis_from_rot(Q4 q, V3& fwd, V3& right, V3& up) {
    const float d = ((q.x * q.x + q.y * q.y) + q.z * q.z) + q.w * q.w;
    const float s = 2.0f / d;
    const float xs = q.x * s, ys = q.y * s, zs = q.z * s;
    const float wx = q.w * xs, wy = q.w * ys, wz = q.w * zs;
    const float xx = q.x * xs, xy = q.x * ys, xz = q.x * zs;
    const float yy = q.y * ys, yz = q.y * zs, zz = q.z * zs;
    fwd = V3{1.0f - (yy + zz), xy + wz, xz - wy};
    right = V3{xy - wz, 1.0f - (xx + zz), yz + wx};
    up = V3{xz + wy, yz - wx, 1.0f - (xx + yy)};
}
// The basis a freshly uploaded orientation is read as (reference GetOfficialUploadBasisVectors, math.hpp:956-982).
RG_HDI void upload_basis_from_rot(Q4 q, V3& fwd, V3& right, V3& up) {
    const float len_sq = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    if (len_sq <= 1e-12f) {
        fwd = V3{1.0f, 0.0f, 0.0f};
        right = V3{0.0f, 1.0f, 0.0f};
        up = V3{0.0f, 0.0f, 1.0f};
        return;
    }
    const float s = 2.0f / len_sq;
    const float xs = q.x * s, ys = q.y * s, zs = q.z * s;
    const float wx = q.w * xs, wy = q.w * ys, wz = q.w * zs;
    const float xx = q.x * xs, xy = q.x * ys, xz = q.x * zs;
    const float yy = q.y * ys, yz = q.y * zs, zz = q.z * zs;
    fwd = V3{1.0f - (yy + zz), xy + wz, xz - wy};
    right = V3{xy - wz, 1.0f - (xx + zz), yz + wx};
    up = V3{xz + wy, yz - wx, 1.0f - (xx + yy)};
}
RG_HDI Q4 game_quat_normalize(Q4 q, float min_len_sq) {
    const float len_sq = ((q.x * q.x + q.y * q.y) + q.z * q.z) + q.w * q.w;
    if (!(len_sq > min_len_sq)) return Q4{1.0f, 0.0f, 0.0f, 0.0f};
    const float s = 1.0f / sqrtf(len_sq);
    return Q4{q.w * s, q.x * s, q.y * s, q.z * s};
}
// One component of the game's replicated rotation: smallest-three encoding at 18 bits (reference math.hpp:1160-1170).
RG_HDI float game_quat_quant_component(float c) {
    constexpr int kMax = (1 << 18) - 1;
    const float max_f = static_cast<float>(kMax);
    float v = ((c * 1.41421354f) * 0.5f + 0.5f) * max_f;
    v = (v + v) + 0.5f;
    int k = x86_f2i(rintf(v));
    k = k < 0 ? (k - 1) / 2 : k / 2;
    k = k < 0 ? 0 : (k < kMax ? k : kMax);
    const float r = static_cast<float>(k) / max_f - 0.5f;
    return (r + r) * 0.707106769f;
}
RG_HDI Q4 game_quantize_quat(Q4 q_in) {
    const Q4 q = game_quat_normalize(q_in, 1e-8f);
    const float a0 = fabsf(q.x), a1 = fabsf(q.y), a2 = fabsf(q.z), a3 = fabsf(q.w);
    const int i01 = a0 < a1 ? 1 : 0;
    const int i23 = a2 < a3 ? 3 : 2;
    const int big = (i01 == 1 ? a1 : a0) >= (i23 == 3 ? a3 : a2) ? i01 : i23;
    const float c_big = big == 0 ? q.x : big == 1 ? q.y : big == 2 ? q.z : q.w;
    const float sign = c_big < 0.0f ? -1.0f : 1.0f;
    const float d0 = game_quat_quant_component((big == 0 ? q.y : q.x) * sign);
    const float d1 = game_quat_quant_component((big <= 1 ? q.z : q.y) * sign);
    const float d2 = game_quat_quant_component((big <= 2 ? q.w : q.z) * sign);
    const float rest = ((1.0f - d0 * d0) - d1 * d1) - d2 * d2;
    const float dropped = sqrtf(rest);
    const float ox = big == 0 ? dropped : d0;
    const float oy = big == 1 ? dropped : (big == 0 ? d0 : d1);
    const float oz = big == 2 ? dropped : (big <= 1 ? d1 : d2);
    const float ow = big == 3 ? dropped : d2;
    return game_quat_normalize(Q4{ow, ox, oy, oz}, 1e-8f);
}
// Re-quantises a basis to the replicated rotation and rebuilds the basis from it; returns the quaternion.
RG_HDI Q4 game_quantize_basis(V3& fwd, V3& right, V3& up) {
    const Q4 q = game_quantize_quat(game_rot_from_basis(fwd, right, up));
    game_basis_from_rot(q, fwd, right, up);
    return q;
}

// Game network quantisation of positions (0.01 uu, round half up) and velocities (truncate to 0.01 / 0.0001 and nudge
// by a tenth of a step away from zero) applied at every tick start (reference raycast_wheels_and_contact_prep.hpp:3851-3871).
RG_HDI float quant_trunc_offset(float x, float scale) {
    const float inv_scale = 1.0f / scale;
    const float k = static_cast<float>(x86_f2i(x * scale));
    const float rounded = k * inv_scale;
    const float offset_mag = 0.1f * inv_scale;
    const float sgn = rounded == 0.0f ? 0.0f : (rounded > 0.0f ? 1.0f : -1.0f);
    const float offset = sgn * offset_mag;
    return rounded + offset;
}
RG_HDI float quant_round_pos(float x, float scale) {
    const float scaled = x * scale;
    return floorf(scaled + 0.5f) * (1.0f / scale);
}

}  // namespace rg
