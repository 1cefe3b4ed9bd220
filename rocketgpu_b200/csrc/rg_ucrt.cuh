// Single-precision atan2 and pow with the results of the reference's UCRT-compatible routines
// (reference include/rocketgpu/detail/math.hpp:65-457), evaluated in double with table lookups. The tables are
// generated by gen_ucrt_tables.py from their mathematical definitions.
#pragma once

#include "rg_math.cuh"

namespace rg {
namespace ucrt_host {
#define RG_UCRT_TABLE(name, n) static const double name[n]
#include "rg_ucrt_tables.inc"
#undef RG_UCRT_TABLE
}  // namespace ucrt_host
#if defined(__CUDACC__)
namespace ucrt_dev {
#define RG_UCRT_TABLE(name, n) __device__ static const double name[n]
#include "rg_ucrt_tables.inc"
#undef RG_UCRT_TABLE
}  // namespace ucrt_dev
#define RG_UCRT_TAB(name) (RG_UCRT_SELECT(name))
#if defined(__CUDA_ARCH__)
#define RG_UCRT_SELECT(name) ::rg::ucrt_dev::name
#else
#define RG_UCRT_SELECT(name) ::rg::ucrt_host::name
#endif
#else
#define RG_UCRT_TAB(name) (::rg::ucrt_host::name)
#endif

RG_HDI uint64_t d2u(double d) {
    uint64_t u;
    memcpy(&u, &d, 8);
    return u;
}
RG_HDI double u2d(uint64_t u) {
    double d;
    memcpy(&d, &u, 8);
    return d;
}

// atan2f: special cases on the exponent difference, then atan of the ratio from a 1/256-spaced table plus a cubic
// correction, or a short odd polynomial for small ratios.
RG_HDI float ucrt_atan2f(float yf, float xf) {
    const double y = static_cast<double>(yf), x = static_cast<double>(xf);
    const uint64_t xb = d2u(x), yb = d2u(y);
    const uint64_t ax = xb & 0x7fffffffffffffffull, ay = yb & 0x7fffffffffffffffull;
    const uint64_t inf = 0x7ff0000000000000ull;
    const bool yneg = (yb >> 63) != 0, xneg = (xb >> 63) != 0;
    const int diff = static_cast<int>((yb >> 52) & 0x7ff) - static_cast<int>((xb >> 52) & 0x7ff);
    if (ax > inf) return u2f(f2u(xf) | 0x400000u);
    if (ay > inf) return u2f(f2u(yf) | 0x400000u);
    if (ay == 0) return xneg ? u2f(yneg ? 0xc0490fdbu : 0x40490fdbu) : yf;
    if (ax == 0 || diff > 26) return u2f(yneg ? 0xbfc90fdbu : 0x3fc90fdbu);
    if (diff < -13 && !xneg) {
        if (diff < -150) return yneg ? -0.0f : 0.0f;
        return static_cast<float>(y / x);
    }
    if (diff < -26) return u2f(yneg ? 0xc0490fdbu : 0x40490fdbu);
    if (ay == inf) {
        if (!xneg) return u2f(yneg ? 0xbf490fdbu : 0x3f490fdbu);
        return u2f(yneg ? 0xc016cbe4u : 0x4016cbe4u);
    }
    double u = fabs(y), v = fabs(x);
    const bool swapped = u > v;
    if (swapped) {
        const double t = u;
        u = v;
        v = t;
    }
    const double ratio = u / v;
    double res;
    if (ratio > 0x1p-4) {
        const int i = x86_d2i(fma(256.0, ratio, 0.5));
        const double id = static_cast<double>(i);
        const double r = fma(u, 256.0, -(id * v)) / fma(u, id, v * 256.0);
        res = fma(-((r * r) * r), 0x1.5555555550877p-2, r + RG_UCRT_TAB(kAtanTab)[i - 16]);
    } else if (ratio < 0x1.a36e2eb1c432dp-14) {
        res = ratio;
    } else {
        const double r2 = ratio * ratio;
        double p = fma(-0x1.2492482bd6be1p-3, r2, 0x1.99999999643a3p-3);
        p = fma(-p, r2, 0x1.5555555555538p-2);
        res = fma(-(r2 * ratio), p, ratio);
    }
    if (swapped) res = 0x1.921fb54442d18p+0 - res;
    if (xneg) res = 0x1.921fb54442d18p+1 - res;
    return static_cast<float>(yneg ? -res : res);
}

// exp(t) for powf: t = n ln2/64 + r, 2^(n/64) from the table, a cubic in r.
RG_HDI float ucrt_powf_exp(double t, uint32_t sign, bool fused) {
    if (t > 0x1.62e43p6) return u2f(0x7f800000u | sign);
    if (!(t > -0x1.9d1dap6)) return u2f(sign);
    const int n = x86_d2i(rint(t * 0x1.71547652b82fep+6));
    const double tab = RG_UCRT_TAB(kPowExp2)[n & 63];
    double res;
    if (fused) {
        const double r = fma(-static_cast<double>(n), 0x1.62e42fefa39efp-7, t);
        res = fma(r * fma(fma(0x1.5555555555555p-3, r, 0.5), r, 1.0), tab, tab);
    } else {
        const double r = t - static_cast<double>(n) * 0x1.62e42fefa39efp-7;
        res = ((r * r) * (0x1.5555555555555p-3 * r + 0.5) + r) * tab + tab;
    }
    uint64_t rb = d2u(res);
    rb += static_cast<uint64_t>(static_cast<int64_t>(n >> 6)) << 52;
    res = u2d(rb);
    return u2f(f2u(static_cast<float>(res)) | sign);
}

// powf(x, y) = exp(y ln x): ln x from a 1/256-spaced table of ln c and 1/c plus a cubic in the reduced argument, or a
// dedicated series near x = 1.
RG_HDI float ucrt_powf(float x, float y) {
    const uint32_t ux = f2u(x), uy = f2u(y);
    const uint32_t ax = ux & 0x7fffffffu, ay = uy & 0x7fffffffu;
    const auto odd_int = [&]() {
        if ((ay & 0x7f800000u) > 0x4b000000u) return false;
        const float yr = rintf(y);
        return yr == y && (static_cast<int>(yr) & 1) != 0;
    };
    if (ay >= 0x7f800000u) {
        if (ay > 0x7f800000u)
            return ux == 0x3f800000u ? (ay < 0x7fc00000u ? 1.5f : 1.0f)
                                     : u2f((ax > 0x7f800000u ? ux : uy) | 0x400000u);
        if (ax > 0x7f800000u) return u2f(ux | 0x400000u);
        if (ax == 0x3f800000u) return 1.0f;
        return u2f((static_cast<int32_t>(uy) < 0) == (ax < 0x3f800000u) ? 0x7f800000u : 0u);
    }
    if (ay == 0) return (ax > 0x7f800000u && ax < 0x7fc00000u) ? u2f(ux | 0x400000u) : 1.0f;
    if (uy == 0x3f800000u) return ax > 0x7f800000u ? u2f(ux | 0x400000u) : x;
    if (ax > 0x7f800000u) return u2f(ux | 0x400000u);
    if (ax == 0x7f800000u || ax == 0) {
        const uint32_t mag = ((static_cast<int32_t>(uy) < 0) == (ax == 0)) ? 0x7f800000u : 0u;
        return u2f(mag | (odd_int() ? (ux & 0x80000000u) : 0u));
    }
    uint32_t sign = 0;
    if (static_cast<int32_t>(ux) < 0 && (ay & 0x7f800000u) <= 0x4b000000u) {
        if (rintf(y) != y) return u2f(0xffc00000u);
        if (odd_int()) sign = 0x80000000u;
    }
    const double dx = static_cast<double>(x), dy = static_cast<double>(y);
    if (static_cast<int32_t>(ux) < 0x3f880000) {
        const double f = dx - 1.0;
        if (fabs(f) < 0x1p-4) {
            const double u = f / (f + 2.0);
            const double w = u + u;
            const double v = w * w;
            const double w3 = w * v;
            const double a = v * 0x1.9999999bac6d4p-7 + 0x1.55555555554e6p-4;
            const double b = v * 0x1.c8034c85dfff0p-12 + 0x1.2492307f1519fp-9;
            const double s = (((v * v) * w3) * b + w3 * a) - u * f;
            return ucrt_powf_exp(dy * (f + s), sign, false);
        }
    }
    const uint64_t bx = d2u(dx);
    const uint64_t mant = bx & 0x000fffffffffffffull;
    const uint32_t idx = static_cast<uint32_t>(mant >> 44) + static_cast<uint32_t>((mant >> 43) & 1);
    const double c = u2d(static_cast<uint64_t>(0x3fe00u | idx) << 44);
    const double m = u2d(mant | 0x3fe0000000000000ull);
    const int e = static_cast<int>((bx >> 52) & 0x7ff) - 0x3ff;
    const double r = (c - m) * RG_UCRT_TAB(kPowInvC)[idx];
    const double rq = r * fma(fma(0x1.5555555555555p-2, r, 0.5), r, 1.0);
    const double log_x = (static_cast<double>(e) * 0x1.62e42fefa39efp-1 + RG_UCRT_TAB(kPowLogC)[idx]) - rq;
    return ucrt_powf_exp(dy * log_x, sign, true);
}

// acosf as the reference computes it (reference RocketGpuUcrtAcosf, math.hpp:458-491): for |x| < 0.5 a rational
// approximation in x^2 added to pi/2 in double, for larger |x| the half-angle identity acos(x) = 2 asin(sqrt((1-x)/2))
// with a split square root; the coefficients are the reference's, written here as their float bit patterns.
RG_HDI float ucrt_acosf(float x) {
    const uint32_t ux = f2u(x);
    const uint32_t ax = ux & 0x7fffffffu, ex = (ux >> 23) & 0xffu;
    if (ax > 0x7f800000u) return u2f(ux | 0x400000u);
    if (ex < 0x65u) return u2f(0x3fc90fdbu);
    if (ex >= 0x7fu) {
        if (x == 1.0f) return 0.0f;
        if (x == -1.0f) return u2f(0x40490fdbu);
        return u2f(0xffc00000u);
    }
    const float a = fabsf(x);
    const bool big = ex >= 0x7eu;
    const float z = big ? (1.0f - a) * 0.5f : a * a;
    const float s = big ? sqrtf(z) : 0.0f;
    float t = u2f(0x3b81ce6bu);
    t = fmaf(-t, z, u2f(0xbc5b3fe1u));
    t = fmaf(t, z, -u2f(0x3d678bddu));
    t = fmaf(t, z, u2f(0x3e3c94dcu));
    const float r = (t * z) / fmaf(-u2f(0x3f561f0du), z, u2f(0x3f8d6fa5u));
    if (!big) {
        const double lo = 0x1.1a62633145c07p-54 - static_cast<double>(r * x);
        return static_cast<float>(0x1.921fb54442d18p+0 - (static_cast<double>(x) - lo));
    }
    if (static_cast<int32_t>(ux) < 0) {
        const double h = (static_cast<double>(s * r) - 0x1.1a62633145c07p-54) + static_cast<double>(s);
        return static_cast<float>(0x1.921fb54442d18p+1 - (h + h));
    }
    const float hi = u2f(f2u(s) & 0xffff0000u);
    const float c = fmaf(-hi, hi, z) / (s + hi);
    return fmaf(r, s + s, c + c) + (hi + hi);
}

}  // namespace rg
