// Deterministic transcendental functions for the SSIMULACRA 2.1 path.
//
// VQM computes its cube root as pow(v, 1/3) and its transfer functions with
// pow/exp/sin in 32-bit float (src/metrics/ssimulacra2/shaders/prepare.comp:78,
// src/vulkan/shaders/color.glsl:117-205); the precision of those built-ins is
// left to each device's shader compiler. The metric's small 1-norms are
// sensitive to single-ulp changes in the XYB planes, so this file pins the
// functions down: each is built only from IEEE-754 basic operations
// (add, multiply, fused multiply-add, divide, conversions, integer bit
// manipulation), which round identically on every conforming CPU and GPU.
// The CUDA kernels, the host-side 8-bit decode tables and the CPU checker all
// evaluate these same functions, so the pyramid planes agree bit for bit.
//
// Accuracy (checked by tests/test_detmath.py against double-precision libm):
// every function but powf_gamma reaches a relative error below ~3e-13 (pow,
// exp and sin in double; the cube root in single precision with an exact
// residual) and rounds once to float, so the float result is the correctly
// rounded value except in the rare cases where the exact value lies within
// that error of a rounding boundary. powf_gamma, the power of the pure
// power-law transfers, works in float pairs to ~2^-30 and is faithfully
// rounded: within one ulp, and on the correctly rounded float for all but
// 0.3-0.4 % of the floats in [2^-30, 2^16) (exhaustive for y = 2.4); below
// 2^-30 it gives 0.
//
// Compiled as host C++ (g++, -ffp-contract=off) or as CUDA (nvcc,
// -fmad=false): no expression below may be contracted differently.
#pragma once

#include <cstdint>
#include <cstring>

#include "ss2_detmath_tables.h"

#if defined(__CUDACC__)
#define SS2_DM __host__ __device__ __forceinline__
#else
#define SS2_DM inline
#include <cmath>
#endif

namespace ss2dm {

SS2_DM double fmad(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
SS2_DM float fmaf_(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
SS2_DM uint32_t bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}
SS2_DM float from_bits(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}
SS2_DM uint64_t bits(double f) {
#if defined(__CUDA_ARCH__)
    return static_cast<uint64_t>(__double_as_longlong(f));
#else
    uint64_t u;
    std::memcpy(&u, &f, 8);
    return u;
#endif
}
SS2_DM double from_bits64(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(static_cast<long long>(u));
#else
    double f;
    std::memcpy(&f, &u, 8);
    return f;
#endif
}

SS2_DM double floord(double x) {
#if defined(__CUDA_ARCH__)
    return ::floor(x);
#else
    return std::floor(x);
#endif
}

// 2^n for integer n in [-1022, 1023].
SS2_DM double pow2i(int n) {
    return from_bits64(static_cast<uint64_t>(n + 1023) << 52);
}

// Cube root of x >= 0, in single precision only:
//   1. r = x^(-1/3) from a bit-level seed and three Newton steps (each
//      roughly squares the relative error: 0.04 -> 3e-3 -> 2e-5 -> ~1e-7);
//   2. y0 = x * r^2, within a few ulps of cbrt(x);
//   3. one Newton step on the root, y = y0 + (x - y0^3) / (3 y0^2), whose
//      residual x - y0^3 is formed without rounding error that matters:
//      y0^3 = hi3 + lo3 by fused-multiply-add error-free products (the
//      TwoProduct of Ogita, Rump and Oishi, "Accurate sum and dot product",
//      SIAM J. Sci. Comput. 26(6), 2005), and x - hi3 is exact (Sterbenz).
//      1 / (3 y0^2) is taken as r^2 / 3, and the step is applied with one
//      rounding (a fused multiply-add).
// The result is cbrt(x) with relative error below ~3e-13 before its single
// rounding, so it is the correctly rounded float except when cbrt(x) lies
// within that distance of a rounding boundary. Inputs outside [1e-20, 1e30]
// are scaled by 2^-90 or 2^90 first (cbrt(x 2^3k) = cbrt(x) 2^k, exact), which
// keeps every partial product above single precision's normal range. Returns
// 0 for x <= 0 and x for infinities and NaN.
SS2_DM float cbrt(float x) {
    if (!(x > 0.0f) || !(x < 3.402823466e38f)) return x > 0.0f ? x : 0.0f;
    float scale = 1.0f;
    if (x < 1.0e-20f) {
        x = x * 1.237940039285380274899e27f;  // 2^90
        scale = 9.313225746154785156e-10f;    // 2^-30
    } else if (x > 1.0e30f) {
        x = x * 8.077935669463160887e-28f;  // 2^-90
        scale = 1073741824.0f;              // 2^30
    }
    // x^(-1/3) seed from the exponent and mantissa bits (log-linear).
    const uint32_t i = bits(x);
    float r = from_bits(0x54a21d2au - i / 3u);
    const float third = 0.333333343267440796f;
    for (int k = 0; k < 3; ++k) {
        const float r3 = r * r * r;
        const float t = fmaf_(-x, r3, 1.0f);
        r = fmaf_(r * t, third, r);
    }
    const float rr = r * r;
    const float y0 = x * rr;
    const float hi = y0 * y0;
    const float lo = fmaf_(y0, y0, -hi);                  // y0^2 = hi + lo exactly
    const float hi3 = hi * y0;
    const float lo3 = fmaf_(lo, y0, fmaf_(hi, y0, -hi3));  // y0^3 = hi3 + lo3
    const float e = (x - hi3) - lo3;
    return fmaf_(e, rr * third, y0) * scale;
}

// The polynomial coefficients and conversion constants of log2d, exp2d and
// sinpi, indexed by the K* names below. Device code reads them from the
// constant bank, where a double-precision instruction takes them as an
// operand (a literal would first be assembled in registers); host code uses
// the same values.
#define SS2DM_CONSTANT_VALUES                                                  \
    1.0 / 7.0, -1.0 / 6.0, 1.0 / 5.0, -1.0 / 4.0, 1.0 / 3.0, -0.5,             \
        1.4426950408889634074, 0.69314718055994530942, 1.0 / 720.0,            \
        1.0 / 120.0, 1.0 / 24.0, 1.0 / 6.0, 0.5, 1.0
enum {
    kLogC7, kLogC6, kLogC5, kLogC4, kLogC3, kLogC2,  // log(1 + r) - r: r^7..r^2
    kLog2E, kLn2,
    kExpC6, kExpC5, kExpC4, kExpC3, kExpC2, kExpC1,  // e^z - 1: z^6..z (over z)
    kConstantCount
};
static const double kConstHost[kConstantCount] = {SS2DM_CONSTANT_VALUES};
#if defined(__CUDACC__)
static __constant__ double kConstDev[kConstantCount] = {SS2DM_CONSTANT_VALUES};
#endif
SS2_DM double K(int i) {
#if defined(__CUDA_ARCH__)
    return kConstDev[i];
#else
    return kConstHost[i];
#endif
}

// The tables of log2d and exp2d (ss2_detmath_tables.h, written by
// gen_detmath_tables.py): one copy for host code and one in device global
// memory, where lanes that index different entries are served by the L1
// cache rather than serialised as they would be from the constant bank.
static const double kInvCHost[128] = {SS2DM_KINVC_VALUES};
static const double kLog2InvCHost[128] = {SS2DM_KLOG2INVC_VALUES};
static const double kExp2JHost[64] = {SS2DM_KEXP2J_VALUES};
#if defined(__CUDACC__)
static __device__ const double kInvCDev[128] = {SS2DM_KINVC_VALUES};
static __device__ const double kLog2InvCDev[128] = {SS2DM_KLOG2INVC_VALUES};
static __device__ const double kExp2JDev[64] = {SS2DM_KEXP2J_VALUES};
#endif
SS2_DM double InvC(int i) {
#if defined(__CUDA_ARCH__)
    return __ldg(&kInvCDev[i]);
#else
    return kInvCHost[i];
#endif
}
SS2_DM double Log2InvC(int i) {
#if defined(__CUDA_ARCH__)
    return __ldg(&kLog2InvCDev[i]);
#else
    return kLog2InvCHost[i];
#endif
}
SS2_DM double Exp2J(int j) {
#if defined(__CUDA_ARCH__)
    return __ldg(&kExp2JDev[j]);
#else
    return kExp2JHost[j];
#endif
}

// The single-precision tables of powf_gamma (same generator), interleaved:
// kLogF4[4 i ..] = 1/c_i in float, then -log2 of it as a hi + lo pair, then
// 0; kExpF2[2 j ..] = 2^(j/64) as a hi + lo pair. One vector load each.
struct alignas(16) LogEntryF {
    float inv, hi, lo, pad;
};
struct alignas(8) ExpEntryF {
    float hi, lo;
};
static const float kLogF4Host[512] = {SS2DM_KLOGF4_VALUES};
static const float kExpF2Host[128] = {SS2DM_KEXPF2_VALUES};
#if defined(__CUDACC__)
static __device__ const float4 kLogF4Dev[128] = {SS2DM_KLOGF4_VALUES};
static __device__ const float2 kExpF2Dev[64] = {SS2DM_KEXPF2_VALUES};
#endif
SS2_DM LogEntryF LogF(int i) {
#if defined(__CUDA_ARCH__)
    const float4 v = __ldg(&kLogF4Dev[i]);
    return LogEntryF{v.x, v.y, v.z, v.w};
#else
    return LogEntryF{kLogF4Host[4 * i], kLogF4Host[4 * i + 1], kLogF4Host[4 * i + 2], 0.0f};
#endif
}
SS2_DM ExpEntryF ExpF(int j) {
#if defined(__CUDA_ARCH__)
    const float2 v = __ldg(&kExpF2Dev[j]);
    return ExpEntryF{v.x, v.y};
#else
    return ExpEntryF{kExpF2Host[2 * j], kExpF2Host[2 * j + 1]};
#endif
}

// log2 of a finite x > 0 in double, table-driven (the reduction of P. T. P.
// Tang, "Table-driven implementation of the logarithm function in IEEE
// floating-point arithmetic", ACM TOMS 16(4), 1990): x = m 2^e, m in [1, 2);
// the top 7 bits of m's fraction pick c near m, and
//   log2 x = e - log2(RN(1/c)) + log2(1 + r),  r = m RN(1/c) - 1 (one fused
// multiply-add, |r| < 2^-8), with ln(1 + r) by its Taylor series to r^7
// (remainder below 2^-67).
// The table-driven step for a normal double x with bits u, minus `shift`
// in the exponent (the body of log2d).
SS2_DM double log2d_normal(uint64_t u, int shift = 0) {
    const int e = static_cast<int>((u >> 52) & 0x7ff) - 1023 - shift;
    const uint64_t frac = u & 0x000fffffffffffffull;
    const int i = static_cast<int>(frac >> 45);
    const double m = from_bits64(frac | 0x3ff0000000000000ull);  // [1, 2)
    const double r = fmad(m, InvC(i), -1.0);
    double p = K(kLogC7);
    p = fmad(p, r, K(kLogC6));
    p = fmad(p, r, K(kLogC5));
    p = fmad(p, r, K(kLogC4));
    p = fmad(p, r, K(kLogC3));
    p = fmad(p, r, K(kLogC2));
    const double ln1r = fmad(r * r, p, r);
    return fmad(ln1r, K(kLog2E), Log2InvC(i) + static_cast<double>(e));
}

SS2_DM double log2d(double x) {
    uint64_t u = bits(x);
    if (((u >> 52) & 0x7ff) == 0) {  // subnormal: normalise, then correct the exponent
        return log2d_normal(bits(x * 18014398509481984.0), 54);  // x 2^54
    }
    return log2d_normal(u);
}

// 2^t in double for |t| < 1000, table-driven: t = (64 n + j) / 64 + f with
// j in [0, 64) and |f| <= 1/128 (f exact), 2^t = 2^n 2^(j/64) e^(f ln 2),
// e^z - 1 by its Taylor series to z^6 (|z| < 0.0055, remainder below 4e-20).
// The reduction and polynomial of exp2d for |t| <= 1000: 2^(j/64) e^(f ln 2)
// in [0.5, 2], and n with 2^t = that 2^n.
SS2_DM double exp2d_core(double t, int& n) {
    const double kd = floord(t * 64.0 + 0.5);
    const double f = t - kd * 0.015625;
    const int k = static_cast<int>(kd);
    const int j = k & 63;
    n = (k - j) >> 6;  // k - j is a multiple of 64
    const double z = f * K(kLn2);
    double p = K(kExpC6);
    p = fmad(p, z, K(kExpC5));
    p = fmad(p, z, K(kExpC4));
    p = fmad(p, z, K(kExpC3));
    p = fmad(p, z, K(kExpC2));
    p = fmad(p, z, K(kExpC1));
    const double tj = Exp2J(j);
    return fmad(tj, p * z, tj);  // 2^(j/64) (1 + (e^z - 1))
}

SS2_DM double exp2d(double t) {
    if (t > 1000.0) t = 1000.0;
    if (t < -1000.0) return 0.0;
    int n;
    const double v = exp2d_core(t, n);
    if (n > 1000) n = 1000;
    // v is in [0.5, 2]: one scaling when 2^n is a normal double; else split
    // it so every factor is (the product is the same: v 2^n1 is exact).
    if (n >= -1022) return v * pow2i(n);
    const int n1 = n / 2, n2 = n - n1;
    return v * pow2i(n1) * pow2i(n2);
}

// x^y for float x > 0 (0 for x == 0 and y > 0), both as float values.
SS2_DM float pow(float x, float y) {
    if (x == 1.0f || y == 0.0f) return 1.0f;
    if (!(x > 0.0f)) return x == 0.0f ? (y > 0.0f ? 0.0f : 3.402823466e38f * 10.0f) : x - x;
    // A positive float is a normal double, so log2d's subnormal step is not
    // needed.
    return static_cast<float>(
        exp2d(static_cast<double>(y) * log2d_normal(bits(static_cast<double>(x)))));
}

// x^y for float x >= 0 and y in [2, 4] (the power-law transfer functions,
// whose exponents are 2.2, 2.4 and 2.8), in single precision: faithfully
// rounded (never more than one ulp from the exact power; the correctly
// rounded float in all but about one case in a hundred) and built from float
// operations only, so it costs a fraction of pow. For x in [2^-30, 2^16):
//   x = 2^e m, m in [1, 2); the top 7 bits of m pick c_i = 1 + (i + 1/2)/128
//   and its float reciprocal inv_i, so r = m inv_i - 1 is exact as the pair
//   (m inv_i rounded - 1, the product's rounding error) with |r| < 2^-8;
//   log2 x = e + L_i + log2(1 + r), L_i = -log2 inv_i a hi + lo float pair,
//   log2(1 + r) by its Taylor series to r^4 (remainder below 2^-41);
//   t = y log2 x as a float pair (the product's error by a fused
//   multiply-add); 2^t = 2^n 2^(j/64) e^z with 64 n + j the nearest integer
//   to 64 t and |z| <= ln2 / 128, e^z - 1 to z^3 (remainder below 2^-34),
//   2^(j/64) a hi + lo pair.
// The absolute error of t stays below ~2^-30, so the value before the last
// rounding is within ~2^-30 relative of x^y (the method of the table-driven
// log and exp above, carried in float pairs: Tang 1990, and the pair
// arithmetic of Dekker 1971). For x in [0, 2^-30) the result is 0: the
// exact power is below 2^-60 there, far under any value the metric resolves,
// so the transfer's inputs need no branch below the fast range (the kernels'
// two-lane form selects 0 for them). For x of 2^16 and above (and negative
// or NaN x), and for y outside [2, 4], it is pow(x, y).
// powf_gamma's constants (shared with its two-lane form in the kernels):
// its fast range [2^-30, 2^16) and [2, 4], the Taylor coefficients of
// log2(1 + r), ln 2 and 1/6, each the float nearest the exact value.
constexpr float kGammaMinX = 9.31322574615478515625e-10f;  // 2^-30
constexpr float kGammaMaxX = 65536.0f;
constexpr float kGammaK1 = 1.44269502163f;     // 1 / ln 2
constexpr float kGammaK2 = -0.721347510815f;   // -1 / (2 ln 2)
constexpr float kGammaK3 = 0.480898350477f;    // 1 / (3 ln 2)
constexpr float kGammaK4 = -0.360673755407f;   // -1 / (4 ln 2)
constexpr float kGammaLn2 = 0.693147182465f;
constexpr float kGammaSixth = 0.166666671634f;
SS2_DM bool powf_gamma_exponent(float y) { return y >= 2.0f && y <= 4.0f; }
SS2_DM bool powf_gamma_fast(float x, float y) {
    return x >= kGammaMinX && x < kGammaMaxX && powf_gamma_exponent(y);
}

SS2_DM float powf_gamma(float x, float y) {
    if (powf_gamma_exponent(y) && x >= 0.0f && x < kGammaMinX) return 0.0f;
    if (!powf_gamma_fast(x, y)) return pow(x, y);
    const uint32_t ix = bits(x);
    const int e = static_cast<int>(ix >> 23) - 127;
    const int i = static_cast<int>((ix >> 16) & 127u);
    const float m = from_bits((ix & 0x007fffffu) | 0x3f800000u);
    const LogEntryF L = LogF(i);
    const float inv = L.inv;
    const float p = m * inv;
    const float pe = fmaf_(m, inv, -p);  // m inv = p + pe exactly
    const float rh = p - 1.0f;           // exact: p is within 2^-8 of 1
    // log2(1 + r) ~ k1 r + k2 r^2 + k3 r^3 + k4 r^4, k_n = (-1)^(n+1) / (n ln 2)
    const float poly = fmaf_(fmaf_(rh, kGammaK4, kGammaK3), rh, kGammaK2);
    const float lr = fmaf_(kGammaK1, rh, fmaf_(rh * rh, poly, kGammaK1 * pe));
    // log2 x = hi + lo: e + L_i exactly as a pair (|L_i| < 1 <= |e| or e = 0)
    const float ef = static_cast<float>(e);
    const float lh = L.hi;
    const float hi = ef + lh;
    const float lo = ((ef - hi) + lh) + (L.lo + lr);
    // t = y log2 x = th + tl
    const float th = y * hi;
    const float tl = fmaf_(y, lo, fmaf_(y, hi, -th));
    // 64 th to the nearest integer k (|64 th| < 2^22), then z = (t - k/64) ln 2
    const float kf = (th * 64.0f + 12582912.0f) - 12582912.0f;
    const float z = fmaf_(fmaf_(kf, -0.015625f, th), kGammaLn2, tl * kGammaLn2);
    const float q = fmaf_(fmaf_(z, kGammaSixth, 0.5f), z * z, z);  // e^z - 1
    const int k = static_cast<int>(kf);
    const int j = k & 63;
    const ExpEntryF T = ExpF(j);
    const float tj = T.hi;
    const float r = tj + fmaf_(tj, q, T.lo);
    return r * from_bits(static_cast<uint32_t>((k >> 6) + 127) << 23);
}

// a / b for b in [2^-20, 2^20] and |a| < 2^20 (the SSIM' and edge maps'
// quotients: their divisors are at least 0.0009 and 1), from basic
// operations only: a reciprocal from a bit seed (relative error below 0.051
// for every positive normal b) refined by three Newton steps r += r (1 - b r)
// (each squares the error: below 2^-34 after the third), then the quotient
// q0 = a r corrected once with its residual a - b q0 (exact in one fused
// multiply-add): q = q0 + r (a - b q0), the final step of Markstein's
// division ("IA-64 and Elementary Functions", 2000). Faithfully rounded, and
// the correctly rounded a / b unless the quotient lies within ~2^-44 of a
// rounding boundary (checked against IEEE division by tests/test_detmath.py).
// divf's reciprocal of b: the bit seed and its three Newton steps.
SS2_DM float recipf(float b) {
    float r = from_bits(0x7ef311c7u - bits(b));
    r = fmaf_(r, fmaf_(-b, r, 1.0f), r);
    r = fmaf_(r, fmaf_(-b, r, 1.0f), r);
    r = fmaf_(r, fmaf_(-b, r, 1.0f), r);
    return r;
}
SS2_DM float divf(float a, float b) {
    const float r = recipf(b);
    const float q0 = a * r;
    return fmaf_(fmaf_(-b, q0, a), r, q0);
}

// e^x for float x.
SS2_DM float exp(float x) {
    return static_cast<float>(exp2d(static_cast<double>(x) * K(kLog2E)));
}

// sin(pi x) for float x in [0, 8): reduced to [-1/2, 1/2] around the
// nearest integer, Taylor polynomial in double.
SS2_DM float sinpi(float xf) {
    const double x = static_cast<double>(xf);
    const double k = floord(x + 0.5);  // nearest integer
    const double f = x - k;             // [-1/2, 1/2]
    const double z = f * 3.14159265358979323846;
    const double z2 = z * z;
    double p = -1.0 / 1307674368000.0;  // -1/15!
    p = fmad(p, z2, 1.0 / 6227020800.0);
    p = fmad(p, z2, -1.0 / 39916800.0);
    p = fmad(p, z2, 1.0 / 362880.0);
    p = fmad(p, z2, -1.0 / 5040.0);
    p = fmad(p, z2, 1.0 / 120.0);
    p = fmad(p, z2, -1.0 / 6.0);
    const double s = fmad(z * z2, p, z);
    const long long ki = static_cast<long long>(k);
    return static_cast<float>((ki & 1) ? -s : s);
}

}  // namespace ss2dm
