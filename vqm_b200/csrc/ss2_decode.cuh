// Input decode on the device: one image's raw samples to linear Rec.709 RGB.
//
// The arithmetic follows VQM's input chain (src/vulkan/shaders/color.glsl,
// with the host constants of src/input.cc): raw sample times scale plus
// offset, chroma upsampling, the matrix / constant-luminance / ICtCp step,
// alpha, the transfer function and the primaries matrix. Every multiply-add
// the reference's shader compiler would contract is an explicit __fmaf_rn;
// the library is compiled with -fmad=false so nothing else is contracted.
//
// The 8-bit RGB / grey formats without alpha decode through a 256-entry table
// built on the host per image (transfer(code * scale + offset)): the table
// holds exactly the per-sample values, so both paths round identically.
// Integer YUV with a pure power-law transfer and at most 2x chroma
// subsampling takes BlockLinearYuv (below), the same values with the
// format's branches resolved; everything else BlockLinearGeneric.
#pragma once

#include <cuda_fp16.h>

#include "ss2_detmath.h"
#include "ss2_device.cuh"
#include "ss2_layout.h"

namespace vqm_b200 {

__device__ __forceinline__ float RawSample(const DevSourceHead& s, int plane,
                                           uint32_t x, uint32_t y) {
    const uint8_t* row = s.plane[plane] + static_cast<size_t>(y) * s.row_bytes[plane];
    float v;
    switch (s.type) {
        case 0: v = static_cast<float>(row[x]); break;
        case 1: v = static_cast<float>(reinterpret_cast<const uint16_t*>(row)[x]); break;
        case 2: v = __half2float(reinterpret_cast<const __half*>(row)[x]); break;
        default: v = reinterpret_cast<const float*>(row)[x]; break;
    }
    // color.glsl:86-89: class 0 luma/R (and RGB's G, B), 1 YUV chroma, 2 alpha.
    const int cls = plane == 3 ? 2 : (plane != 0 && s.family == 2 ? 1 : 0);
    return __fmaf_rn(v, s.scale[cls], s.offset[cls]);
}

// color.glsl:117-179.
__device__ __forceinline__ float Rec709InvOetf(float x) {
    x = fmaxf(x, 0.0f);
    const float alpha = 1.09929682680944f, beta = 0.018053968510807f;
    return x < __fmul_rn(4.5f, beta)
               ? __fdiv_rn(x, 4.5f)
               : ss2dm::pow(__fdiv_rn(__fadd_rn(x, __fsub_rn(alpha, 1.0f)), alpha),
                      __fdiv_rn(1.0f, 0.45f));
}
__device__ __forceinline__ float SrgbEotf(float v) {
    return v <= 0.04045f ? __fdiv_rn(v, 12.92f)
                         : ss2dm::pow(__fdiv_rn(__fadd_rn(v, 0.055f), 1.055f), 2.4f);
}
__device__ __forceinline__ float St2084Eotf(float x) {
    if (x <= 0.0f) return 0.0f;
    const float xp = ss2dm::pow(x, __fdiv_rn(1.0f, 78.84375f));
    const float num = fmaxf(__fsub_rn(xp, 0.8359375f), 0.0f);
    const float den = fmaxf(__fsub_rn(18.8515625f, __fmul_rn(18.6875f, xp)),
                            1.17549435e-38f);
    return ss2dm::pow(__fdiv_rn(num, den), __fdiv_rn(1.0f, 0.1593017578125f));
}
__device__ __forceinline__ float AribInvOetf(float x) {
    x = fmaxf(x, 0.0f);
    return x <= 0.5f ? __fmul_rn(__fmul_rn(x, x), __fdiv_rn(1.0f, 3.0f))
                     : __fdiv_rn(__fadd_rn(ss2dm::exp(__fdiv_rn(__fsub_rn(x, 0.55991073f),
                                                         0.17883277f)),
                                           0.28466892f),
                                 12.0f);
}
__device__ __forceinline__ float TransferDecode(const DevSourceHead& s, float v) {
    switch (s.transfer) {
        case 0: return v;
        case 1: return v < 0.0f ? 0.0f : ss2dm::powf_gamma(v, 2.4f);
        case 2: return v < 0.0f ? 0.0f : ss2dm::powf_gamma(v, 2.2f);
        case 3: return v < 0.0f ? 0.0f : ss2dm::powf_gamma(v, 2.8f);
        case 4: return SrgbEotf(v);
        case 5: return v <= 0.0f ? 0.01f : ss2dm::pow(10.0f, __fmul_rn(2.0f, __fsub_rn(v, 1.0f)));
        case 6:
            return v <= 0.0f ? 0.00316227766f
                             : ss2dm::pow(10.0f, __fmul_rn(2.5f, __fsub_rn(v, 1.0f)));
        case 7:
            return v >= 0.0f && v <= 1.0f
                       ? ss2dm::pow(v, 2.4f)
                       : (v < 0.0f ? -Rec709InvOetf(-v) : Rec709InvOetf(v));
        case 8:
            if (v >= 0.0f && v <= 1.0f) return ss2dm::pow(v, 2.4f);
            return v >= 0.0f ? Rec709InvOetf(v)
                             : __fdiv_rn(-Rec709InvOetf(__fmul_rn(-4.0f, v)), 4.0f);
        case 9: return __fmul_rn(s.to_linear, St2084Eotf(v));
        case 10:
            return v < 0.0f ? 0.0f
                            : __fmul_rn(__fdiv_rn(52.37f, 48.0f), ss2dm::pow(v, 2.6f));
    }
    return v;
}
// color.glsl:181-205.
__device__ __forceinline__ void TransferRgb(const DevSourceHead& s, float c[3]) {
    if (s.transfer == 11) {
        for (int i = 0; i < 3; ++i) c[i] = AribInvOetf(c[i]);
        const float luma =
            fmaxf(__fmaf_rn(s.kb, c[2], __fmaf_rn(s.kg, c[1], __fmul_rn(s.kr, c[0]))),
                  1.17549435e-38f);
        const float f = __fmul_rn(ss2dm::pow(luma, 0.2f), s.to_linear);
        for (int i = 0; i < 3; ++i) c[i] = __fmul_rn(c[i], f);
        return;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) c[i] = TransferDecode(s, c[i]);
}
// color.glsl:209-218.
__device__ __forceinline__ void ApplyMatrix(const float* m, float v[3]) {
    float r[3];
    for (int row = 0; row < 3; ++row)
        r[row] = __fmaf_rn(m[row * 3 + 2], v[2],
                           __fmaf_rn(m[row * 3 + 1], v[1], __fmul_rn(m[row * 3], v[0])));
    v[0] = r[0];
    v[1] = r[1];
    v[2] = r[2];
}
// ApplyMatrix on two pixels, two lanes per instruction: the same values.
__device__ __forceinline__ void ApplyMatrix2(const float* m, float2 v[3]) {
    float2 r[3];
#pragma unroll
    for (int row = 0; row < 3; ++row) {
        const float2 a = make_float2(m[row * 3], m[row * 3]);
        const float2 b = make_float2(m[row * 3 + 1], m[row * 3 + 1]);
        const float2 c = make_float2(m[row * 3 + 2], m[row * 3 + 2]);
        r[row] = __ffma2_rn(c, v[2], __ffma2_rn(b, v[1], __fmul2_rn(a, v[0])));
    }
    v[0] = r[0];
    v[1] = r[1];
    v[2] = r[2];
}
// color.glsl:223-236.
__device__ __forceinline__ void ClToRgb(const DevSourceHead& s, float e[3]) {
    const float u = e[1], v = e[2];
    const float kbv = u < 0.0f ? s.cl[0] : s.cl[1];
    const float krv = v < 0.0f ? s.cl[2] : s.cl[3];
    const float b = Rec709InvOetf(__fmaf_rn(__fmul_rn(u, 2.0f), kbv, e[0]));
    const float r = Rec709InvOetf(__fmaf_rn(__fmul_rn(v, 2.0f), krv, e[0]));
    const float luma = Rec709InvOetf(e[0]);
    const float g = __fdiv_rn(__fmaf_rn(-s.kb, b, __fmaf_rn(-s.kr, r, luma)), s.kg);
    e[0] = r;
    e[1] = g;
    e[2] = b;
}

// color.glsl:271-283.
__device__ __forceinline__ float RoundHalfup(float x) {
    return x < 0.0f ? floorf(__fadd_rn(x, 0.5f)) : floorf(__fadd_rn(x, 0.49999997f));
}
__device__ __forceinline__ int MirrorIndex(float xpos, uint32_t dim) {
    const float extent = static_cast<float>(dim);
    const float m = xpos < 0.0f ? -xpos
                                : (xpos >= extent ? __fsub_rn(__fmul_rn(2.0f, extent), xpos)
                                                  : xpos);
    return static_cast<int>(fminf(fmaxf(m, 0.0f), __fsub_rn(extent, 1.0f)));
}
__device__ __forceinline__ float FilterKernel(int filter, float x) {
    x = fabsf(x);
    if (filter == 0) return fmaxf(__fsub_rn(1.0f, x), 0.0f);
    if (filter == 1) {
        if (x < 1.0f)
            return __fmaf_rn(__fmul_rn(x, x), __fmaf_rn(x, 1.5f, -2.5f), 1.0f);
        if (x < 2.0f)
            return __fmaf_rn(x, __fmaf_rn(x, __fmaf_rn(-0.5f, x, 2.5f), -4.0f), 2.0f);
        return 0.0f;
    }
    // sin(pi v) / (pi v), the sine from the shared deterministic functions,
    // the denominator with the reference's float pi.
    const float pi = 3.14159265358979323846f;
    if (!(x < 3.0f)) return 0.0f;
    const float a = x == 0.0f ? 1.0f : __fdiv_rn(ss2dm::sinpi(x), __fmul_rn(pi, x));
    const float x3 = __fdiv_rn(x, 3.0f);
    const float b = x3 == 0.0f ? 1.0f : __fdiv_rn(ss2dm::sinpi(x3), __fmul_rn(pi, x3));
    return __fmul_rn(a, b);
}

// color.glsl:288-299. `scale` is 1, 2 or 4, so dividing by it is the exact
// product with its reciprocal.
__device__ __forceinline__ void BilinearPhase(uint32_t out_pos, float inv_scale, float shift,
                                              int centre, int& s0, float& w0, float& w1) {
    const float pos =
        __fadd_rn(__fmul_rn(__fadd_rn(static_cast<float>(out_pos), 0.5f), inv_scale), shift);
    const float base = __fadd_rn(RoundHalfup(__fsub_rn(pos, 1.0f)), 0.5f);
    const float t = __fsub_rn(pos, base);
    s0 = static_cast<int>(floorf(base)) - centre + 1;
    w0 = __fsub_rn(1.0f, t);
    w1 = t;
}

// Rows s and s + 1 of a 3x3 window, by selection rather than an index, so
// the window stays in registers. s is 0, 1 or 2: along an axis that is not
// subsampled the second tap of a phase can fall one slot past the window,
// always with weight exactly 0, and reads 0 here.
struct WinRows {
    float top[3], bottom[3];
};
__device__ __forceinline__ WinRows PickRows(const float (&win)[9], int s) {
    WinRows r;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r.top[k] = s == 0 ? win[k] : (s == 1 ? win[3 + k] : win[6 + k]);
        r.bottom[k] = s == 0 ? win[3 + k] : (s == 1 ? win[6 + k] : 0.0f);
    }
    return r;
}
// The bilinear value from rows r at columns s, s + 1 (s in 0..2, a column
// past the window reading 0), in the reference's accumulation order.
__device__ __forceinline__ float BilinearTap(const WinRows& r, int s, float xw0, float xw1,
                                             float yw0, float yw1) {
    const float w00 = __fmul_rn(xw0, yw0), w10 = __fmul_rn(xw1, yw0);
    const float w01 = __fmul_rn(xw0, yw1), w11 = __fmul_rn(xw1, yw1);
    const float t0 = s == 0 ? r.top[0] : (s == 1 ? r.top[1] : r.top[2]);
    const float t1 = s == 0 ? r.top[1] : (s == 1 ? r.top[2] : 0.0f);
    const float b0 = s == 0 ? r.bottom[0] : (s == 1 ? r.bottom[1] : r.bottom[2]);
    const float b1 = s == 0 ? r.bottom[1] : (s == 1 ? r.bottom[2] : 0.0f);
    return __fmaf_rn(w11, b1, __fmaf_rn(w01, b0, __fmaf_rn(w10, t1, __fmul_rn(w00, t0))));
}

// color.glsl:324-367: bilinear chroma of the block's four samples.
__device__ __forceinline__ void ChromaBilinear(const DevSourceHead& s, int plane, const uint32_t px[4],
                                               const uint32_t py[4], float out[4]) {
    const uint32_t dx = s.plane_w[plane], dy = s.plane_h[plane];
    const int cx = static_cast<int>(px[0] >> s.sub_w);
    const int cy = static_cast<int>(py[0] >> s.sub_h);
    float win[9];
    const bool interior =
        cx > 0 && cx + 1 < static_cast<int>(dx) && cy > 0 && cy + 1 < static_cast<int>(dy);
    if (interior && s.type <= 1) {
        // Integer samples away from the edges: three row addresses, nine
        // loads, then the class-1 scale and offset (RawSample's arithmetic).
        const size_t rb = s.row_bytes[plane];
        const uint8_t* row = s.plane[plane] + static_cast<size_t>(cy - 1) * rb;
#pragma unroll
        for (int j = 0; j < 3; ++j, row += rb)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const uint32_t x = static_cast<uint32_t>(cx - 1 + i);
                const float v = s.type == 0
                                    ? static_cast<float>(__ldg(row + x))
                                    : static_cast<float>(__ldg(reinterpret_cast<const uint16_t*>(row) + x));
                win[j * 3 + i] = __fmaf_rn(v, s.scale[1], s.offset[1]);
            }
    } else {
#pragma unroll
        for (int j = -1; j <= 1; ++j)
#pragma unroll
            for (int i = -1; i <= 1; ++i) {
                uint32_t sx, sy;
                if (interior) {
                    sx = static_cast<uint32_t>(cx + i);
                    sy = static_cast<uint32_t>(cy + j);
                } else {
                    sx = static_cast<uint32_t>(
                        MirrorIndex(__fadd_rn(static_cast<float>(cx + i), 0.5f), dx));
                    sy = static_cast<uint32_t>(
                        MirrorIndex(__fadd_rn(static_cast<float>(cy + j), 0.5f), dy));
                }
                win[(j + 1) * 3 + (i + 1)] = RawSample(s, plane, sx, sy);
            }
    }
    const float iscx = 1.0f / static_cast<float>(1u << s.sub_w);
    const float iscy = 1.0f / static_cast<float>(1u << s.sub_h);
    int xa, xb, ya, yb;
    float xwa0, xwa1, xwb0, xwb1, ywa0, ywa1, ywb0, ywb1;
    BilinearPhase(px[0], iscx, s.shift_x, cx, xa, xwa0, xwa1);
    BilinearPhase(px[1], iscx, s.shift_x, cx, xb, xwb0, xwb1);
    BilinearPhase(py[0], iscy, s.shift_y, cy, ya, ywa0, ywa1);
    BilinearPhase(py[2], iscy, s.shift_y, cy, yb, ywb0, ywb1);
    const WinRows ra = PickRows(win, ya), rb = PickRows(win, yb);
    out[0] = BilinearTap(ra, xa, xwa0, xwa1, ywa0, ywa1);
    out[1] = BilinearTap(ra, xb, xwb0, xwb1, ywa0, ywa1);
    out[2] = BilinearTap(rb, xa, xwa0, xwa1, ywb0, ywb1);
    out[3] = BilinearTap(rb, xb, xwb0, xwb1, ywb0, ywb1);
}

// color.glsl:371-432: bicubic (4 taps) or Lanczos-3 (6 taps) chroma.
__device__ void AxisTaps(const DevSourceHead& s, uint32_t out_pos, float scale, float shift,
                         uint32_t dim, int taps, float* w, int* idx) {
    const float pos =
        __fadd_rn(__fdiv_rn(__fadd_rn(static_cast<float>(out_pos), 0.5f), scale), shift);
    const float base =
        __fadd_rn(RoundHalfup(__fsub_rn(pos, __fdiv_rn(static_cast<float>(taps), 2.0f))), 0.5f);
    float total = 0.0f;
    for (int j = 0; j < taps; ++j)
        total = __fadd_rn(total, FilterKernel(s.filter,
                                              __fsub_rn(__fadd_rn(base, static_cast<float>(j)), pos)));
    for (int j = 0; j < taps; ++j) {
        w[j] = __fdiv_rn(
            FilterKernel(s.filter, __fsub_rn(__fadd_rn(base, static_cast<float>(j)), pos)),
            total);
        idx[j] = MirrorIndex(__fadd_rn(base, static_cast<float>(j)), dim);
    }
}
__device__ void ChromaTaps(const DevSourceHead& s, int plane, const uint32_t px[4],
                           const uint32_t py[4], float out[4]) {
    const int taps = s.filter == 1 ? 4 : 6;
    const float scx = static_cast<float>(1u << s.sub_w);
    const float scy = static_cast<float>(1u << s.sub_h);
    float wx0[6], wx1[6], wy0[6], wy1[6];
    int ix0[6], ix1[6], iy0[6], iy1[6];
    AxisTaps(s, px[0], scx, s.shift_x, s.plane_w[plane], taps, wx0, ix0);
    AxisTaps(s, px[1], scx, s.shift_x, s.plane_w[plane], taps, wx1, ix1);
    AxisTaps(s, py[0], scy, s.shift_y, s.plane_h[plane], taps, wy0, iy0);
    AxisTaps(s, py[2], scy, s.shift_y, s.plane_h[plane], taps, wy1, iy1);
    auto taps2d = [&](const float* wx, const int* ix, const float* wy, const int* iy) {
        float sum = 0.0f;
        for (int j = 0; j < taps; ++j) {
            float row = 0.0f;
            for (int k = 0; k < taps; ++k)
                row = __fmaf_rn(wx[k],
                                RawSample(s, plane, static_cast<uint32_t>(ix[k]),
                                          static_cast<uint32_t>(iy[j])),
                                row);
            sum = __fmaf_rn(wy[j], row, sum);
        }
        return sum;
    };
    out[0] = taps2d(wx0, ix0, wy0, iy0);
    out[1] = taps2d(wx1, ix1, wy0, iy0);
    out[2] = taps2d(wx0, ix0, wy1, iy1);
    out[3] = taps2d(wx1, ix1, wy1, iy1);
}

// color.glsl:447-541: the block's four samples, linear Rec.709, in
// (0,0), (1,0), (0,1), (1,1) order. The generic path: any format.
__device__ __forceinline__ void BlockLinearGeneric(const DevSourceHead& s, uint32_t bx, uint32_t by,
                                   float rgb[4][3]) {
    const uint32_t lx = s.width - 1, ly = s.height - 1;
    const uint32_t px[4] = {min(2 * bx, lx), min(2 * bx + 1, lx), min(2 * bx, lx),
                            min(2 * bx + 1, lx)};
    const uint32_t py[4] = {min(2 * by, ly), min(2 * by, ly), min(2 * by + 1, ly),
                            min(2 * by + 1, ly)};
    float cu[4] = {0, 0, 0, 0}, cv[4] = {0, 0, 0, 0};
    const bool sub = s.chroma_variant && s.family == 2;
    if (sub) {
        if (s.filter == 0) {
            ChromaBilinear(s, 1, px, py, cu);
            ChromaBilinear(s, 2, px, py, cv);
        } else {
            ChromaTaps(s, 1, px, py, cu);
            ChromaTaps(s, 2, px, py, cv);
        }
    }
    const bool has_alpha = s.alpha != 0;
    const bool premul = s.alpha == 2;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float alpha = has_alpha ? RawSample(s, 3, px[i], py[i]) : 1.0f;
        float e[3];
        e[0] = e[1] = e[2] = RawSample(s, 0, px[i], py[i]);
        if (s.family != 0) {
            if (sub) {
                e[1] = cu[i];
                e[2] = cv[i];
            } else {
                e[1] = RawSample(s, 1, px[i], py[i]);
                e[2] = RawSample(s, 2, px[i], py[i]);
            }
        }
        if (s.mode == 1) {
            ClToRgb(s, e);
        } else if (!s.identity1) {
            ApplyMatrix(s.m1, e);
        }
        if (premul) {
            const float cl = fminf(fmaxf(alpha, 0.0f), 1.0f);
            if (cl == 0.0f) {
                e[0] = e[1] = e[2] = 0.0f;
            } else {
                for (int k = 0; k < 3; ++k) e[k] = __fdiv_rn(e[k], cl);
            }
        }
        if (has_alpha) {
            const float target = __fmul_rn(__fsub_rn(1.0f, alpha), s.background);
            for (int k = 0; k < 3; ++k) e[k] = __fmaf_rn(alpha, e[k], target);
        }
        if (s.mode != 1) TransferRgb(s, e);
        if (!s.identity2) ApplyMatrix(s.m2, e);
        rgb[i][0] = e[0];
        rgb[i][1] = e[1];
        rgb[i][2] = e[2];
    }
}

// ss2dm::powf_gamma of two lanes with the same y, both inside the function's
// fast range (x in [2^-30, 2^16), y in [2, 4]; the caller selects the rest),
// the floating-point steps two lanes per instruction (FFMA2 / FMUL2 / FADD2),
// each the operation the scalar function performs on that lane: the same
// values. `pt` is a copy of the function's two tables (kLogF4, kExpF2) in
// shared memory, one array per field (PowTable): each lane's entry depends
// on its value, and divergent entries of a shared-memory table cost fewer
// cycles than the same loads through L1. One field per load puts the two
// lanes' values straight into the register pair of a two-lane instruction.
struct PowTable {
    static constexpr int kInv = 0, kHi = 128, kLo = 256, kExpHi = 384, kExpLo = 448;
    static constexpr int kFloats = 512;
};
__device__ __forceinline__ float2 PowfGamma2(float2 x, float y, const float* pt) {
    using namespace ss2dm;
    const auto P = [](float v) { return make_float2(v, v); };
    const auto N = [](float2 v) { return make_float2(-v.x, -v.y); };
    const uint32_t ix0 = __float_as_uint(x.x), ix1 = __float_as_uint(x.y);
    const int i0 = static_cast<int>((ix0 >> 16) & 127u), i1 = static_cast<int>((ix1 >> 16) & 127u);
    const float2 m = make_float2(__uint_as_float((ix0 & 0x007fffffu) | 0x3f800000u),
                                 __uint_as_float((ix1 & 0x007fffffu) | 0x3f800000u));
    const float2 inv = make_float2(pt[PowTable::kInv + i0], pt[PowTable::kInv + i1]);
    const float2 p = __fmul2_rn(m, inv);
    const float2 pe = __ffma2_rn(m, inv, N(p));
    const float2 rh = __fadd2_rn(p, P(-1.0f));
    const float2 poly = __ffma2_rn(__ffma2_rn(rh, P(kGammaK4), P(kGammaK3)), rh, P(kGammaK2));
    const float2 lr = __ffma2_rn(P(kGammaK1), rh,
                                 __ffma2_rn(__fmul2_rn(rh, rh), poly, __fmul2_rn(P(kGammaK1), pe)));
    // e = (ix >> 23) - 127 as a float without a conversion: 2^23 + (ix >> 23)
    // is a float's bit pattern, and subtracting 2^23 + 127 is exact.
    const float2 ef = __fadd2_rn(make_float2(__uint_as_float(0x4b000000u | (ix0 >> 23)),
                                             __uint_as_float(0x4b000000u | (ix1 >> 23))),
                                 P(-8388735.0f));
    const float2 lh = make_float2(pt[PowTable::kHi + i0], pt[PowTable::kHi + i1]);
    const float2 ll = make_float2(pt[PowTable::kLo + i0], pt[PowTable::kLo + i1]);
    const float2 hi = __fadd2_rn(ef, lh);
    const float2 lo = __fadd2_rn(__fadd2_rn(__fadd2_rn(ef, N(hi)), lh), __fadd2_rn(ll, lr));
    const float2 th = __fmul2_rn(P(y), hi);
    const float2 tl = __ffma2_rn(P(y), lo, __ffma2_rn(P(y), hi, N(th)));
    // big = 1.5 2^23 + k, k = round(64 th), |k| < 2^13: its bit pattern is
    // 0x4b400000 + k, so k's table index and exponent come from the bits (no
    // conversion), and the table load issues before z and q are formed.
    const float2 big = __ffma2_rn(th, P(64.0f), P(12582912.0f));
    const uint32_t u0 = __float_as_uint(big.x), u1 = __float_as_uint(big.y);
    const int j0 = static_cast<int>(u0 & 63u), j1 = static_cast<int>(u1 & 63u);
    const float2 kf = __fadd2_rn(big, P(-12582912.0f));
    const float2 z = __ffma2_rn(__ffma2_rn(kf, P(-0.015625f), th), P(kGammaLn2),
                                __fmul2_rn(tl, P(kGammaLn2)));
    const float2 q = __ffma2_rn(__ffma2_rn(z, P(kGammaSixth), P(0.5f)), __fmul2_rn(z, z), z);
    const float2 tj = make_float2(pt[PowTable::kExpHi + j0], pt[PowTable::kExpHi + j1]);
    const float2 tjl = make_float2(pt[PowTable::kExpLo + j0], pt[PowTable::kExpLo + j1]);
    const float2 r = __fadd2_rn(tj, __ffma2_rn(tj, q, tjl));
    // 2^(k >> 6) = bits ((k >> 6) + 127) << 23, with k + 127 * 64 = u -
    // 0x4b3fe040 in [448, 12224] over the fast range (t in [-120, 64)).
    return __fmul2_rn(r, make_float2(__uint_as_float(((u0 - 0x4b3fe040u) << 17) & 0xff800000u),
                                     __uint_as_float(((u1 - 0x4b3fe040u) << 17) & 0xff800000u)));
}

// The YUV fast path (DevSource::yuv_fast): the CTA's chroma window of both
// planes staged once in shared memory (kPrepTile >> sub samples per axis plus
// one on each side, edge-clamped: for the one-past-the-edge positions a block
// can touch that is the reference's mirror index), already scaled like
// RawSample. `plane` floats per plane: kChromaStage covers every
// subsampling the path takes, kChromaStage420 4:2:0 alone.
constexpr int kChromaStage = ((kPrepTile >> 1) + 2) * (kPrepTile + 2);
constexpr int kChromaStage420 = ((kPrepTile >> 1) + 2) * ((kPrepTile >> 1) + 2);
__device__ __forceinline__ void StageChroma(const DevSourceHead& s, uint32_t gx, uint32_t gy,
                                            float* stage, int plane) {
    const uint32_t sw = (kPrepTile >> s.sub_w) + 2, sh = (kPrepTile >> s.sub_h) + 2;
    const int c0x = static_cast<int>((gx * kPrepTile) >> s.sub_w) - 1;
    const int c0y = static_cast<int>((gy * kPrepTile) >> s.sub_h) - 1;
    // A row of the window per sw threads, blockDim.x / sw rows per pass
    // (sw <= 66, so at least 3 rows of the CTA's 256 threads).
    const uint32_t rows_per_pass = blockDim.x / sw;
    const uint32_t i = threadIdx.x % sw, j0 = threadIdx.x / sw;
    if (j0 >= rows_per_pass) return;
    // Both chroma planes have the same size; each pass loads a sample of
    // each (unrolled, so several passes' loads are in flight at once).
    const int dx = static_cast<int>(s.plane_w[1]), dy = static_cast<int>(s.plane_h[1]);
    const uint32_t x = static_cast<uint32_t>(min(max(c0x + static_cast<int>(i), 0), dx - 1));
    const auto sample = [&](int p, uint32_t y) {
        const uint8_t* row = s.plane[p] + static_cast<size_t>(y) * s.row_bytes[p];
        return s.type == 0 ? static_cast<float>(__ldg(row + x))
                           : static_cast<float>(__ldg(reinterpret_cast<const uint16_t*>(row) + x));
    };
#pragma unroll 3
    for (uint32_t j = j0; j < sh; j += rows_per_pass) {
        const uint32_t y = static_cast<uint32_t>(min(max(c0y + static_cast<int>(j), 0), dy - 1));
        const float u = sample(1, y), v = sample(2, y);
        stage[j * sw + i] = __fmaf_rn(u, s.scale[1], s.offset[1]);
        stage[plane + j * sw + i] = __fmaf_rn(v, s.scale[1], s.offset[1]);
    }
}

// The two 4:2:0 axis phases the host recognises (DevSource::chroma_pattern):
// type 0 (siting offset 0): slots 0, 1 with weights (1/4, 3/4), (3/4, 1/4);
// type 1 (offset 1/4): slots 1, 1 with (1, 0), (1/2, 1/2). Per output the
// four taps are BilinearTap's, in its order, with the weight products
// folded at compile time (exact: the factors are multiples of 1/4), so the
// values equal the runtime path's; the window reads become fixed offsets.
template <int kType>
struct AxisPhase {
    static __device__ constexpr int Slot(int par) { return par ? 1 : (kType ? 1 : 0); }
    static __device__ constexpr float W0(int par) {
        return par ? (kType ? 0.5f : 0.75f) : (kType ? 1.0f : 0.25f);
    }
    static __device__ constexpr float W1(int par) {
        return par ? (kType ? 0.5f : 0.25f) : (kType ? 0.0f : 0.75f);
    }
};
template <int kX, int kY>
__device__ __forceinline__ void ChromaFixed(const float* stage, int plane, int bxs, int bys,
                                            float e[4][3]) {
    using X = AxisPhase<kX>;
    using Y = AxisPhase<kY>;
    constexpr int sw = (kPrepTile >> 1) + 2;
    // Both pixels of a row at once (xp = 0, 1 in the two lanes), each lane
    // the scalar chain.
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const float* base = stage + p * plane + bys * sw + bxs;
#pragma unroll
        for (int yp = 0; yp < 2; ++yp) {
            const float* t0 = base + Y::Slot(yp) * sw + X::Slot(0);
            const float* t1 = base + Y::Slot(yp) * sw + X::Slot(1);
            const auto w = [](float a, float b) { return make_float2(a, b); };
            const float2 v = __ffma2_rn(
                w(X::W1(0) * Y::W1(yp), X::W1(1) * Y::W1(yp)), make_float2(t0[sw + 1], t1[sw + 1]),
                __ffma2_rn(w(X::W0(0) * Y::W1(yp), X::W0(1) * Y::W1(yp)),
                           make_float2(t0[sw], t1[sw]),
                           __ffma2_rn(w(X::W1(0) * Y::W0(yp), X::W1(1) * Y::W0(yp)),
                                      make_float2(t0[1], t1[1]),
                                      __fmul2_rn(w(X::W0(0) * Y::W0(yp), X::W0(1) * Y::W0(yp)),
                                                 make_float2(t0[0], t1[0])))));
            e[2 * yp][1 + p] = v.x;
            e[2 * yp + 1][1 + p] = v.y;
        }
    }
}

// BlockLinearGeneric for a yuv_fast image's block (bx, by) of the CTA's tile
// (gx, gy) whose two columns and rows are inside the image: the same values,
// with the format's branches resolved and the chroma taps read from the
// staged window at the host's per-parity slots and weights.
__device__ __forceinline__ void BlockLinearYuv(const DevSourceHead& s, const float* stage,
                                               int plane, const float* pow_table,
                                               uint32_t gx, uint32_t gy, uint32_t bx,
                                               uint32_t by, bool aligned4, float rgb[4][3]) {
    const uint32_t x0 = 2 * bx, y0 = 2 * by;
    float e[4][3];
    {
        const uint8_t* r0 = s.plane[0] + static_cast<size_t>(y0) * s.row_bytes[0];
        const uint8_t* r1 = r0 + s.row_bytes[0];
        float v[4];
        if (aligned4) {
            // Both samples of a row in one load (x0 is even; planes and rows
            // are 4-byte aligned).
            uint32_t a, b;
            if (s.type == 0) {
                a = __ldg(reinterpret_cast<const uint16_t*>(r0 + x0));
                b = __ldg(reinterpret_cast<const uint16_t*>(r1 + x0));
                v[0] = static_cast<float>(a & 0xffu);
                v[1] = static_cast<float>(a >> 8);
                v[2] = static_cast<float>(b & 0xffu);
                v[3] = static_cast<float>(b >> 8);
            } else {
                a = __ldg(reinterpret_cast<const uint32_t*>(r0 + 2 * x0));
                b = __ldg(reinterpret_cast<const uint32_t*>(r1 + 2 * x0));
                v[0] = static_cast<float>(a & 0xffffu);
                v[1] = static_cast<float>(a >> 16);
                v[2] = static_cast<float>(b & 0xffffu);
                v[3] = static_cast<float>(b >> 16);
            }
        } else if (s.type == 0) {
            v[0] = __ldg(r0 + x0);
            v[1] = __ldg(r0 + x0 + 1);
            v[2] = __ldg(r1 + x0);
            v[3] = __ldg(r1 + x0 + 1);
        } else {
            const uint16_t* w0 = reinterpret_cast<const uint16_t*>(r0);
            const uint16_t* w1 = reinterpret_cast<const uint16_t*>(r1);
            v[0] = __ldg(w0 + x0);
            v[1] = __ldg(w0 + x0 + 1);
            v[2] = __ldg(w1 + x0);
            v[3] = __ldg(w1 + x0 + 1);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) e[i][0] = __fmaf_rn(v[i], s.scale[0], s.offset[0]);
    }
    if (s.chroma_variant && s.chroma_pattern) {
        const int bxs = static_cast<int>((x0 >> 1) - ((gx * kPrepTile) >> 1));
        const int bys = static_cast<int>((y0 >> 1) - ((gy * kPrepTile) >> 1));
        switch (s.chroma_pattern) {
            case 1: ChromaFixed<0, 0>(stage, plane, bxs, bys, e); break;
            case 2: ChromaFixed<1, 0>(stage, plane, bxs, bys, e); break;
            case 3: ChromaFixed<0, 1>(stage, plane, bxs, bys, e); break;
            default: ChromaFixed<1, 1>(stage, plane, bxs, bys, e); break;
        }
    } else if (s.chroma_variant) {
        const uint32_t sw = (kPrepTile >> s.sub_w) + 2;
        // Window slot 0 of this block is chroma sample (cx - 1, cy - 1), the
        // staged entry (cx - 1 - c0x, cy - 1 - c0y).
        const int bxs = static_cast<int>((x0 >> s.sub_w) - ((gx * kPrepTile) >> s.sub_w));
        const int bys = static_cast<int>((y0 >> s.sub_h) - ((gy * kPrepTile) >> s.sub_h));
#pragma unroll
        for (int p = 0; p < 2; ++p) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int xp = i & 1, yp = i >> 1;
                const float* t =
                    stage + p * plane + (bys + s.cslot[1][yp]) * static_cast<int>(sw) +
                    bxs + s.cslot[0][xp];
                const float* w = s.cweight[yp][xp];
                // A first slot of 2 puts the second tap past the window: 0.
                const bool xpast = s.cslot[0][xp] == 2, ypast = s.cslot[1][yp] == 2;
                const float t0 = t[0], t1 = xpast ? 0.0f : t[1];
                const float b0 = ypast ? 0.0f : t[sw];
                const float b1 = xpast || ypast ? 0.0f : t[sw + 1];
                e[i][1 + p] = __fmaf_rn(
                    w[3], b1, __fmaf_rn(w[2], b0, __fmaf_rn(w[1], t1, __fmul_rn(w[0], t0))));
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            e[i][1] = RawSample(s, 1, x0 + (i & 1), y0 + (i >> 1));
            e[i][2] = RawSample(s, 2, x0 + (i & 1), y0 + (i >> 1));
        }
    }
    // From here on the block's two rows run as pixel pairs (pixels 0, 1 and
    // 2, 3), two lanes per instruction, each lane the scalar operation.
    float2 q[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int c = 0; c < 3; ++c) q[h][c] = make_float2(e[2 * h][c], e[2 * h + 1][c]);
    if (!s.identity1) {
#pragma unroll
        for (int h = 0; h < 2; ++h) ApplyMatrix2(s.m1, q[h]);
    }
    // The transfer, powf_gamma two pixels per call: v below 2^-30 (negative
    // included) gives 0; every other v is inside the fast range, the host
    // having bounded the matrix's output below 2^16 for every sample code
    // (DevSource::yuv_fast).
    const float g = s.gamma;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float2 v = q[h][c];
            const bool ia = v.x >= ss2dm::kGammaMinX, ib = v.y >= ss2dm::kGammaMinX;
            const float2 r =
                PowfGamma2(make_float2(ia ? v.x : 1.0f, ib ? v.y : 1.0f), g, pow_table);
            q[h][c] = make_float2(ia ? r.x : 0.0f, ib ? r.y : 0.0f);
        }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (!s.identity2) ApplyMatrix2(s.m2, q[h]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            rgb[2 * h][c] = q[h][c].x;
            rgb[2 * h + 1][c] = q[h][c].y;
        }
    }
}

}  // namespace vqm_b200
