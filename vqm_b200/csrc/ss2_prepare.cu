// Prepare stage for sm_100a: decode -> linear Rec.709 -> XYB -> the whole
// 2x2-box pyramid of one image's 64x64 base tile, per CTA
// (reference: src/metrics/ssimulacra2/shaders/prepare.comp).
//
// A CTA is NT threads (128 or 256) over the tile's 32x32 base 2x2 blocks:
// thread (tx, ty) = (t & 15, t >> 4) owns blocks (2tx + hx, ty + (NT / 16) vy),
// hx in {0, 1}, vy < 32 / (NT / 16), i.e. four base pixels in a row of two
// rows, two or four times. Levels 0 and 1 come from the thread's own samples;
// level 1 goes through a shared-memory ladder from which levels 2.. are
// averaged, each level with a barrier among the threads it still needs.
// Because the 2x2 box nests exactly, no CTA ever needs a neighbour's samples.
//
// Two kernels: 8-bit grey/RGB without alpha decode through the image's
// 256-entry table in shared memory, reading four samples of a row with one
// 32-bit load where the planes allow it; every other format runs the decode
// of ss2_decode.cuh, whose YUV fast path (integer YUV, power-law transfer)
// stages the tile's chroma window in shared memory first. Images whose
// linear samples the host has proved non-negative run a body whose cube
// roots skip their range check (the same values). The XYB transform of two
// pixels runs on Blackwell's two-lane FP32 instructions, and its cube root is
// the shared deterministic one (ss2_detmath.h) evaluated lane by lane with
// the same operations, so the planes this kernel writes are bit-identical to
// the CPU checker's.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "ss2_decode.cuh"
#include "ss2_detmath.h"
#include "ss2_device.cuh"
#include "ss2_kernels.h"
#include "ss2_layout.h"

namespace vqm_b200 {
namespace {

constexpr uint32_t kBlocks = kPrepTile / 2;  // base 2x2 blocks per tile side

// CTAs per SM of a prepare kernel of 128 threads (large launches): ten for
// the table decode, eight for the YUV decode with its 4:2:0 chroma window
// (28 KB of shared memory); the 256-thread kernels run five or four (see
// PrepareKernel).
constexpr int kTableCtas128 = 10;
constexpr int kYuvCtas128 = 8;

// The last prefix entry <= index (start[0] == 0 <= index < start[count]).
__device__ __forceinline__ uint32_t FindSlot(const uint32_t* __restrict__ start, uint32_t count,
                                             uint32_t index) {
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&start[mid]) <= index) lo = mid;
        else hi = mid;
    }
    return lo;
}

// prepare.comp:40-54.
constexpr float kM00 = 0.30f, kM02 = 0.078f, kM01 = static_cast<float>(1.0 - 0.078 - 0.30);
constexpr float kM10 = 0.23f, kM12 = 0.078f, kM11 = static_cast<float>(1.0 - 0.078 - 0.23);
constexpr float kM20 = 0.24342268924547819f, kM21 = 0.20476744424496821f;
constexpr float kM22 = static_cast<float>(1.0 - 0.24342268924547819 - 0.20476744424496821);
constexpr float kBias = 0.0037930732552754493f;
constexpr float kCbrtBias = 0.15595419704914093f;

__device__ __forceinline__ float2 Pack(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 Neg(float2 v) { return make_float2(-v.x, -v.y); }

// x^(-1/3) to about 2^-21 relative as 2^(-log2(x) / 3), from the
// special-function unit's approximate base-2 logarithm and exponential.
__device__ __forceinline__ float RcbrtEstimate(float x) {
    float l, r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
    l = __fmul_rn(l, -0.333333343267440796f);
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(l));
    return r;
}

// The correctly rounded cube root of both lanes, ss2dm::cbrt's value, by a
// shorter route for lanes in [kCbrtRouteLo, kCbrtRouteHi) = [2^-16, 2^24)
// (every XYB mix of in-gamut light: the mix includes a bias of 0.0038); any
// other lane pair calls ss2dm::cbrt per lane. ss2dm::cbrt refines a
// bit-level estimate of x^(-1/3) (error ~0.04) with three Newton steps;
// here the estimate comes from the special-function unit (error ~2^-21), so
// one step brings r to the same float-rounding floor, and the remaining
// steps are ss2dm::cbrt's own: y0 = x r^2, then one Newton step on the root
// with its residual x - y0^3 formed exactly, rounded once. Both routes round
// a value within ~1e-13 of cbrt(x); on every float of the band they give the
// same float, which the library checks on the device (vqm_cu_ss2_check_cbrt,
// run by the GPU tests over the whole band). Outside it they can part: one
// mantissa, 0x7afd13, whose cube root lies almost on a rounding boundary,
// rounds differently every third octave below 2^-16 and above 2^24.
// Two lanes per instruction. kInRange: the caller knows both lanes are in
// the band (the host proves it per image: DevSource::in_range).
template <bool kInRange = false>
__device__ __forceinline__ float2 Cbrt2(float2 x) {
    if (!kInRange && !(x.x >= kCbrtRouteLo && x.x < kCbrtRouteHi && x.y >= kCbrtRouteLo &&
                       x.y < kCbrtRouteHi))
        return make_float2(ss2dm::cbrt(x.x), ss2dm::cbrt(x.y));
    float2 r = make_float2(RcbrtEstimate(x.x), RcbrtEstimate(x.y));
    const float2 third = Pack(0.333333343267440796f);
    {
        const float2 r3 = __fmul2_rn(__fmul2_rn(r, r), r);
        const float2 t = __ffma2_rn(Neg(x), r3, Pack(1.0f));
        r = __ffma2_rn(__fmul2_rn(r, t), third, r);
    }
    const float2 rr = __fmul2_rn(r, r);
    const float2 y0 = __fmul2_rn(x, rr);
    const float2 hi = __fmul2_rn(y0, y0);
    const float2 lo = __ffma2_rn(y0, y0, Neg(hi));
    const float2 hi3 = __fmul2_rn(hi, y0);
    const float2 lo3 = __ffma2_rn(lo, y0, __ffma2_rn(hi, y0, Neg(hi3)));
    const float2 e = __fadd2_rn(__fadd2_rn(x, Neg(hi3)), Neg(lo3));
    return __ffma2_rn(e, __fmul2_rn(rr, third), y0);
}

__device__ __forceinline__ float2 Max0(float2 v) {
    return make_float2(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f));
}

// prepare.comp:81-98 for two pixels. Only the channels in `mask` are
// meaningful; B's cube root is skipped when B is not stored. kInRange: the
// inputs are non-negative and finite (so every mix is at least the bias).
template <bool kInRange = false>
__device__ __forceinline__ void Xyb2(float2 r, float2 g, float2 b, uint32_t mask, float2 out[3]) {
    // In range, every mix is at least the bias, so the clamp at 0 is the
    // identity and is left out.
    const auto clamp = [](float2 v) { return kInRange ? v : Max0(v); };
    const float2 m0 = clamp(__ffma2_rn(Pack(kM00), r,
                                       __ffma2_rn(Pack(kM01), g, __ffma2_rn(Pack(kM02), b, Pack(kBias)))));
    const float2 m1 = clamp(__ffma2_rn(Pack(kM10), r,
                                       __ffma2_rn(Pack(kM11), g, __ffma2_rn(Pack(kM12), b, Pack(kBias)))));
    const float2 c0 = __fadd2_rn(Cbrt2<kInRange>(m0), Pack(-kCbrtBias));
    const float2 c1 = __fadd2_rn(Cbrt2<kInRange>(m1), Pack(-kCbrtBias));
    const float2 sum = __fadd2_rn(c0, c1);
    out[0] = __ffma2_rn(__fmul2_rn(Pack(0.5f), __fadd2_rn(c0, Neg(c1))), Pack(14.0f), Pack(0.42f));
    out[1] = __ffma2_rn(Pack(0.5f), sum, Pack(0.01f));
    out[2] = Pack(0.0f);
    if (mask & 4u) {
        const float2 m2 = clamp(__ffma2_rn(
            Pack(kM20), r, __ffma2_rn(Pack(kM21), g, __ffma2_rn(Pack(kM22), b, Pack(kBias)))));
        const float2 c2 = __fadd2_rn(Cbrt2<kInRange>(m2), Pack(-kCbrtBias));
        out[2] = __fadd2_rn(__ffma2_rn(Pack(-0.5f), sum, c2), Pack(0.55f));
    }
}

// One pixel: the pair form with a duplicated lane.
template <bool kInRange = false>
__device__ __forceinline__ void Xyb(float r, float g, float b, uint32_t mask, float out[3]) {
    float2 o[3];
    Xyb2<kInRange>(Pack(r), Pack(g), Pack(b), mask, o);
    out[0] = o[0].x;
    out[1] = o[1].x;
    out[2] = o[2].x;
}

// The half-plane build's rounding of a plane value (ssimu2_common.glsl:86-91).
template <bool kHalf>
__device__ __forceinline__ float PlaneRound(float v) {
    return kHalf ? __half2float(__float2half_rn(v)) : v;
}

// prepare.comp:103-111: ((((0 + a) + b) + c) + d) * 0.25, rounded like a
// plane value (the average used to reach the next level through the planes).
template <bool kHalf>
__device__ __forceinline__ float BoxAverage(float a, float b, float c, float d) {
    return PlaneRound<kHalf>(__fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(a, b), c), d), 0.25f));
}

// Per-level addressing of this image's planes, staged in shared memory:
// float elements, or binary16 ones with half planes.
struct LevelInfo {
    void* plane[kMaxLevels][3];  // nullptr when pruned
    uint32_t w[kMaxLevels], h[kMaxLevels], pitch[kMaxLevels], mask[kMaxLevels];
    uint32_t levels;
};

template <bool kHalf>
__device__ __forceinline__ void PutPlane(void* plane, size_t at, float v) {
    if (kHalf) static_cast<__half*>(plane)[at] = __float2half_rn(v);
    else static_cast<float*>(plane)[at] = v;
}

// Writes pixel (x, y) of `level` with XYB value `xyb` (kept channels): the
// value inside the level, 0 in the padding columns and row past an unaligned
// size (ss2_layout.h: to a multiple of 2 columns, 4 with half planes), nothing
// beyond. Every padding entry has a thread: a level's tile grid spans a
// multiple of 64 >> level (at least 4) columns and rows.
template <bool kHalf>
__device__ __forceinline__ void StorePixel(const LevelInfo& lv, uint32_t level, uint32_t x,
                                           uint32_t y, float x_, float y_, float b_) {
    const uint32_t mask = lv.mask[level];
    const uint32_t w = lv.w[level], h = lv.h[level];
    if (!mask || x >= PaddedColumns(w, kHalf) || y >= ((h + 1) & ~1u)) return;
    const bool inside = x < w && y < h;
    const size_t at = PlaneIndex(lv.pitch[level], x, y);
    if (mask & 1u) PutPlane<kHalf>(lv.plane[level][0], at, inside ? x_ : 0.0f);
    if (mask & 2u) PutPlane<kHalf>(lv.plane[level][1], at, inside ? y_ : 0.0f);
    if (mask & 4u) PutPlane<kHalf>(lv.plane[level][2], at, inside ? b_ : 0.0f);
}

// Level 0's 2x2 block at (x0, y0) as one aligned store of the row-pair plane:
// (x0, y0), (x0, y0+1), (x0+1, y0), (x0+1, y0+1).
template <bool kHalf>
__device__ __forceinline__ void PutBlock(void* plane, size_t at, float a, float b, float c,
                                         float d) {
    if (kHalf) {
        __half2* p = reinterpret_cast<__half2*>(static_cast<__half*>(plane) + at);
        uint2 v;
        const __half2 lo = __floats2half2_rn(a, b), hi = __floats2half2_rn(c, d);
        v.x = *reinterpret_cast<const uint32_t*>(&lo);
        v.y = *reinterpret_cast<const uint32_t*>(&hi);
        *reinterpret_cast<uint2*>(p) = v;
    } else {
        *reinterpret_cast<float4*>(static_cast<float*>(plane) + at) = make_float4(a, b, c, d);
    }
}

// The four samples of base block (bx, by) of an 8-bit image, as table
// entries, in (0,0), (1,0), (0,1), (1,1) order, edge-clamped like
// prepare.comp's loads. `w4[c]` holds the 32-bit words of rows 2by and
// 2by + 1 at column 4 * (bx / 2) when `fast`.
__device__ __forceinline__ void TableBlock(const DevSourceHead& s, const float* lut, bool fast,
                                           const uint32_t (&w4)[3][2], uint32_t hx, uint32_t bx,
                                           uint32_t by, float lin[4][3]) {
    const bool grey = s.family == 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        uint32_t code[4];
        if (fast) {
            // Bytes 2hx and 2hx + 1 of each row word, zero-extended.
            const uint32_t row0 = grey ? w4[0][0] : w4[c][0];
            const uint32_t row1 = grey ? w4[0][1] : w4[c][1];
            const uint32_t sel = 0x4440u | (2u * hx);
            code[0] = __byte_perm(row0, 0u, sel);
            code[1] = __byte_perm(row0, 0u, sel + 1u);
            code[2] = __byte_perm(row1, 0u, sel);
            code[3] = __byte_perm(row1, 0u, sel + 1u);
        } else {
            const int pl = grey ? 0 : c;
            const uint32_t x0 = 2 * bx, y0 = 2 * by;
            const uint32_t x1 = min(x0 + 1, s.width - 1), y1 = min(y0 + 1, s.height - 1);
            const uint8_t* r0 = s.plane[pl] + static_cast<size_t>(y0) * s.row_bytes[pl];
            const uint8_t* r1 = s.plane[pl] + static_cast<size_t>(y1) * s.row_bytes[pl];
            code[0] = __ldg(r0 + x0);
            code[1] = __ldg(r0 + x1);
            code[2] = __ldg(r1 + x0);
            code[3] = __ldg(r1 + x1);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) lin[i][c] = lut[code[i]];
    }
    if (!s.identity2) {
#pragma unroll
        for (int i = 0; i < 4; ++i) ApplyMatrix(s.m2, lin[i]);
    }
}

// CTAs per SM: five of 256 threads (40 warps) for the table and YUV
// decodes, four for the generic one; the table decode also runs as ten CTAs
// of 128 threads (see LaunchPrepareOf). The decodes' long dependency chains
// (the YUV power's table loads, the generic FP64 transfers) want the warps
// more than the registers (measured on 136 uneven pairs: the YUV kernel at
// 5 CTAs with some spilling took 8.48 ms, at 4 9.33 ms; the generic decode
// at 4 beats 2 by a quarter; the table kernel of 256 threads on 64 1080p
// pairs took 1.366 ms at 5, 1.374 ms at 6 and 1.399 ms at 4).
#ifndef VQM_GENERIC_PREPARE_CTAS
#define VQM_GENERIC_PREPARE_CTAS 4
#endif
#ifndef VQM_YUV_PREPARE_CTAS
#define VQM_YUV_PREPARE_CTAS 5
#endif
template <int kGroup, bool kHalf, int kNT>
__global__ void __launch_bounds__(kNT, kNT == 128     ? (kGroup == 0 ? kTableCtas128 : kYuvCtas128)
                                       : kGroup == 0 ? 5
                                       : kGroup == 1 ? VQM_YUV_PREPARE_CTAS
                                                     : VQM_GENERIC_PREPARE_CTAS)
    PrepareKernel(DevBatch batch) {
    constexpr uint32_t kThreads = kNT;
    constexpr uint32_t kRows = kThreads / 16;         // block rows per pass
    constexpr uint32_t kRowPasses = kBlocks / kRows;  // 2 or 4
    constexpr bool kTable = kGroup == 0;  // 8-bit RGB/grey by table
    constexpr bool kYuv = kGroup == 1;    // yuv_fast images
    // Level-1 tile (32x32) of each channel, then the levels after it in two
    // alternating buffers: odd levels in `ladder_a`, even ones in `ladder_b`.
    __shared__ __align__(16) float ladder_a[3][kBlocks * kBlocks];
    __shared__ float ladder_b[3][kBlocks * kBlocks / 4];
    __shared__ float lut[kTable ? 256 : 1];
    __shared__ DevSourceHead src_s;  // (the byte table goes to `lut`)
    __shared__ LevelInfo lv;
    __shared__ uint32_t aligned4;
    // Both chroma planes' window of the tile, for yuv_fast images, and the
    // power's tables.
    // The 128-thread YUV kernel stages 4:2:0 windows only (the host sends
    // it launches whose images all have 4:2:0 chroma or none subsampled).
    constexpr int kStagePlane = (kYuv && kNT == 128) ? kChromaStage420 : kChromaStage;
    __shared__ float chroma_stage[kYuv ? 2 * kStagePlane : 1];
    __shared__ float pow_table[kYuv ? PowTable::kFloats : 1];

    const uint32_t tid = threadIdx.x;
    const uint32_t n_items = batch.prep_items[kGroup];
    uint32_t before = 0;  // images in the groups ahead of this one
#pragma unroll
    for (int g = 0; g < kGroup; ++g) before += batch.prep_items[g];
    const DevPrepItem* items = batch.prep_item + before;
    const uint32_t* start = batch.prep_start + before + kGroup;
    const uint32_t it = FindSlot(start, n_items, blockIdx.x);
    const DevPrepItem item = items[it];
    const DevPair& P = batch.pair[item.pair];
    const uint32_t t = blockIdx.x - __ldg(&start[it]);
    const uint32_t gy = t / P.prep_tiles_x;
    const uint32_t gx = t - gy * P.prep_tiles_x;
    const int image = static_cast<int>(item.image);

    {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&P.src[image]);
        uint32_t* to = reinterpret_cast<uint32_t*>(&src_s);
        constexpr uint32_t words = sizeof(DevSourceHead) / 4;
        for (uint32_t i = tid; i < words; i += kThreads) to[i] = from[i];
        if (kTable)
            for (uint32_t i = tid; i < 256; i += kThreads) lut[i] = P.src[image].srgb_lut[i];
        if (kYuv && tid < 128) {
            const float4 l = __ldg(&ss2dm::kLogF4Dev[tid]);  // inv, hi, lo, 0
            pow_table[PowTable::kInv + tid] = l.x;
            pow_table[PowTable::kHi + tid] = l.y;
            pow_table[PowTable::kLo + tid] = l.z;
        }
        if (kYuv && tid < 64) {
            const float2 e = __ldg(&ss2dm::kExpF2Dev[tid]);  // hi, lo
            pow_table[PowTable::kExpHi + tid] = e.x;
            pow_table[PowTable::kExpLo + tid] = e.y;
        }
        if (tid < kMaxLevels * 3) {
            const uint32_t l = tid / 3, c = tid % 3;
            const bool kept = l < P.levels && (P.mask[l] & (1u << c));
            const size_t elem = static_cast<size_t>(image) * P.image_stride + P.plane_off[l][c];
            lv.plane[l][c] = !kept ? nullptr
                             : kHalf ? static_cast<void*>(reinterpret_cast<__half*>(P.pyramid) + elem)
                                     : static_cast<void*>(P.pyramid + elem);
        }
        if (tid < kMaxLevels) {
            lv.w[tid] = P.w[tid];
            lv.h[tid] = P.h[tid];
            lv.pitch[tid] = P.pitch[tid];
            lv.mask[tid] = tid < P.levels ? P.mask[tid] : 0u;
        }
        if (tid == 0) {
            lv.levels = P.levels;
            // 32-bit sample loads need every plane and row on a 4-byte boundary.
            const DevSource& ps = P.src[image];
            uint32_t ok = 1;
            for (int c = 0; c < (ps.family == 0 ? 1 : 3); ++c)
                ok &= ((reinterpret_cast<uintptr_t>(ps.plane[c]) | ps.row_bytes[c]) & 3u) == 0;
            aligned4 = ok;
        }
    }
    __syncthreads();
    // The rest of the kernel, for inputs whose every mix is known to be in
    // the cube root's direct range (kInRange) or not.
    const auto body = [=](auto in_range) {
    constexpr bool kInRange = decltype(in_range)::value;
    const DevSourceHead& s = src_s;
    if constexpr (kYuv) {
        if (s.chroma_variant) {
            // A window larger than the stage would overrun it: such an image
            // never reaches this kernel, and if it did its tiles are left
            // unwritten rather than read out of bounds.
            if (kStagePlane == kChromaStage420 && (s.sub_w != 1 || s.sub_h != 1)) return;
            StageChroma(s, gx, gy, chroma_stage, kStagePlane);
            __syncthreads();
        }
    }
    const uint32_t levels = lv.levels;
    const uint32_t width = s.width, height = s.height;
    const uint32_t wb = (width + 1) / 2, hb = (height + 1) / 2;  // base blocks
    // Blocks of level 0's plane, padding included (ss2_layout.h).
    const uint32_t wb_pad = PaddedColumns(width, kHalf) / 2;
    const uint32_t tx = tid & 15, ty = tid >> 4;
    const uint32_t mask0 = lv.mask[0];

    uint32_t last = 0;  // the deepest level that stores a channel
    for (uint32_t l = 1; l < levels; ++l)
        if (lv.mask[l]) last = l;

#pragma unroll 1
    for (uint32_t vy = 0; vy < kRowPasses; ++vy) {
        const uint32_t by = gy * kBlocks + ty + kRows * vy;
        const uint32_t bx0 = gx * kBlocks + 2 * tx;
        // Both blocks' samples of each plane as two 32-bit words when the
        // four columns and two rows are inside and aligned.
        uint32_t w4[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        bool fast = false;
        if (kTable) {
            fast = aligned4 && 2 * bx0 + 3 < width && 2 * by + 1 < height;
            if (fast) {
                const int np = s.family == 0 ? 1 : 3;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (c >= np) break;
                    const uint8_t* r0 =
                        s.plane[c] + static_cast<size_t>(2 * by) * s.row_bytes[c] + 2 * bx0;
                    w4[c][0] = __ldg(reinterpret_cast<const uint32_t*>(r0));
                    w4[c][1] = __ldg(reinterpret_cast<const uint32_t*>(r0 + s.row_bytes[c]));
                }
            }
        }
        float l1[2][3];
        // Unrolled for the table decode (the words and averages stay in
        // registers); rolled for the generic decode, whose body is large.
#pragma unroll(kTable ? 2 : 1)
        for (uint32_t hx = 0; hx < 2; ++hx) {
            const uint32_t bx = bx0 + hx;
            float lin[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            const bool in_block = bx < wb && by < hb;
            if (kHalf && !in_block && bx < wb_pad && by < hb && mask0) {
                // Padding blocks past the image's last column: zeros.
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    if (mask0 & (1u << c))
                        PutBlock<kHalf>(lv.plane[0][c], PlaneIndex(lv.pitch[0], 2 * bx, 2 * by),
                                        0.0f, 0.0f, 0.0f, 0.0f);
            }
            if (in_block) {
                if constexpr (kTable) {
                    TableBlock(s, lut, fast, w4, hx, bx, by, lin);
                } else if constexpr (kYuv) {
                    // Even width and height (PrepGroup): the block is whole.
                    BlockLinearYuv(s, chroma_stage, kStagePlane, pow_table, gx, gy, bx, by,
                                   aligned4 != 0, lin);
                } else {
                    BlockLinearGeneric(s, bx, by, lin);
                }
                // Level 0: the block is one aligned float4 of the row-pair
                // plane, (x0, y0), (x0, y0+1), (x0+1, y0), (x0+1, y0+1); a
                // column or row past the image is the plane's zero padding.
                if (mask0) {
                    float2 top[3], bottom[3];
                    Xyb2<kInRange>(make_float2(lin[0][0], lin[1][0]),
                                   make_float2(lin[0][1], lin[1][1]),
                                   make_float2(lin[0][2], lin[1][2]), mask0, top);
                    Xyb2<kInRange>(make_float2(lin[2][0], lin[3][0]),
                                   make_float2(lin[2][1], lin[3][1]),
                                   make_float2(lin[2][2], lin[3][2]), mask0, bottom);
                    const uint32_t x0 = 2 * bx, y0 = 2 * by;
                    const bool two = x0 + 1 < width;
                    const bool second_row = y0 + 1 < height;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        if (!(mask0 & (1u << c))) continue;
                        PutBlock<kHalf>(lv.plane[0][c], PlaneIndex(lv.pitch[0], x0, y0), top[c].x,
                                        second_row ? bottom[c].x : 0.0f, two ? top[c].y : 0.0f,
                                        two && second_row ? bottom[c].y : 0.0f);
                    }
                }
            }
            float avg[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                avg[c] = BoxAverage<kHalf>(lin[0][c], lin[1][c], lin[2][c], lin[3][c]);
            // Register copies, not an index, for the rolled form.
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (hx == 0) l1[0][c] = avg[c];
                else l1[1][c] = avg[c];
            }
        }
        // Level 1: pixels (bx0, by) and (bx0 + 1, by).
        if (last >= 1) {
            float2 xyb[3];
            Xyb2<kInRange>(make_float2(l1[0][0], l1[1][0]), make_float2(l1[0][1], l1[1][1]),
                           make_float2(l1[0][2], l1[1][2]), lv.mask[1], xyb);
            // Rows by and by ^ 1 of the row pair belong to lanes l and l ^ 16
            // of the same warp. Where the pair's 2x2 block is inside the
            // level and X and Y are its kept channels, each channel's block
            // is one float4 of the row-pair plane: the even row's thread
            // stores X and the odd row's Y, each taking the other row's
            // values of its channel from its partner lane.
            const bool odd = (by & 1u) != 0;
            const float2 send = odd ? xyb[0] : xyb[1];
            const float2 recv = make_float2(__shfl_xor_sync(0xffffffffu, send.x, 16),
                                            __shfl_xor_sync(0xffffffffu, send.y, 16));
            const uint32_t y0 = by & ~1u;
            if (!kHalf && lv.mask[1] == 3u && bx0 + 1 < lv.w[1] && y0 + 1 < lv.h[1]) {
                const float2 own = odd ? xyb[1] : xyb[0];
                const float4 v = odd ? make_float4(recv.x, own.x, recv.y, own.y)
                                     : make_float4(own.x, recv.x, own.y, recv.y);
                float* plane = static_cast<float*>(lv.plane[1][odd ? 1 : 0]);
                *reinterpret_cast<float4*>(plane + PlaneIndex(lv.pitch[1], bx0, y0)) = v;
            } else {
                StorePixel<kHalf>(lv, 1, bx0, by, xyb[0].x, xyb[1].x, xyb[2].x);
                StorePixel<kHalf>(lv, 1, bx0 + 1, by, xyb[0].y, xyb[1].y, xyb[2].y);
            }
            if (last >= 2) {
                const uint32_t at = (ty + kRows * vy) * kBlocks + 2 * tx;  // even
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    *reinterpret_cast<float2*>(&ladder_a[c][at]) = make_float2(l1[0][c], l1[1][c]);
            }
        }
    }
    if (last < 2) return;
    __syncthreads();

    // Levels 2..last: the first min(side^2, NT) threads average the
    // previous level's 2x2 blocks from the ladder (side^2 = 256, 64, 16, 4
    // pixels; prepare.comp:149-168, clamped to the previous level's last
    // column and row); threads that no longer take part leave, and the rest
    // meet at a barrier of their own.
#pragma unroll 1
    for (uint32_t level = 2; level <= last; ++level) {
        const uint32_t shift = 6 - level;             // side = 64 >> level
        const uint32_t side = 1u << shift;
        const uint32_t active = side * side;
        const uint32_t workers = active < kThreads ? active : kThreads;
        if (tid >= workers) return;
        const uint32_t prev_side = side * 2;
        const uint32_t pw = lv.w[level - 1], ph = lv.h[level - 1];
        const uint32_t ox = min(gx * prev_side, pw - 1);
        const uint32_t oy = min(gy * prev_side, ph - 1);
        const uint32_t lx = pw - 1 - ox, ly = ph - 1 - oy;
        const float* prev0 = (level & 1u) ? &ladder_b[0][0] : &ladder_a[0][0];
        const uint32_t prev_stride = (level & 1u) ? kBlocks * kBlocks / 4 : kBlocks * kBlocks;
        float* next0 = (level & 1u) ? &ladder_a[0][0] : &ladder_b[0][0];
        const uint32_t next_stride = (level & 1u) ? kBlocks * kBlocks : kBlocks * kBlocks / 4;
        const auto pixel = [&](uint32_t px) {
            const uint32_t jx = px & (side - 1);
            const uint32_t jy = px >> shift;
            const uint32_t cx0 = min(2 * jx, lx), cx1 = min(2 * jx + 1, lx);
            const uint32_t cy0 = min(2 * jy, ly), cy1 = min(2 * jy + 1, ly);
            float v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float* p = prev0 + c * prev_stride;
                v[c] = BoxAverage<kHalf>(p[cy0 * prev_side + cx0], p[cy0 * prev_side + cx1],
                                         p[cy1 * prev_side + cx0], p[cy1 * prev_side + cx1]);
            }
            float xyb[3];
            Xyb<kInRange>(v[0], v[1], v[2], lv.mask[level], xyb);
            StorePixel<kHalf>(lv, level, gx * side + jx, gy * side + jy, xyb[0], xyb[1],
                              xyb[2]);
            if (level < last) {
#pragma unroll
                for (int c = 0; c < 3; ++c) next0[c * next_stride + px] = v[c];
            }
        };
        if constexpr (kThreads >= 256) {
            pixel(tid);  // at most 256 pixels a level: one each
        } else {
            for (uint32_t px = tid; px < active; px += kThreads) pixel(px);
        }
        if (level < last) {
            if (workers > 32) {
                // 256, 128 or 64 threads: whole warps from warp 0.
                asm volatile("bar.sync 1, %0;" ::"r"(workers) : "memory");
            } else {
                __syncwarp((1u << workers) - 1u);
            }
        }
    }
    };
    if (src_s.in_range) body(std::true_type{});
    else body(std::false_type{});
}

}  // namespace

template <bool kHalf>
cudaError_t PreloadPrepareOf() {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, PrepareKernel<0, kHalf, 256>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, PrepareKernel<0, kHalf, 128>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, PrepareKernel<1, kHalf, 256>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, PrepareKernel<1, kHalf, 128>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, PrepareKernel<2, kHalf, 256>);
    return e;
}
cudaError_t PreloadPrepare() {
    const cudaError_t e = PreloadPrepareOf<false>();
    return e == cudaSuccess ? PreloadPrepareOf<true>() : e;
}

namespace {
// Compares Cbrt2's in-range route with ss2dm::cbrt on the `count` floats
// whose bit patterns follow `first`, two per thread step (the odd last one
// paired with itself); counts the differing patterns and keeps the smallest.
__global__ void CheckCbrtKernel(uint32_t first, uint32_t count, unsigned long long* mismatches,
                                uint32_t* first_bad) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t pairs = count / 2 + count % 2;
    unsigned long long bad = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += stride) {
        const uint32_t b0 = first + 2 * i;
        const bool two = 2 * i + 1 < count;
        const uint32_t b1 = two ? b0 + 1 : b0;
        const float2 x = make_float2(__uint_as_float(b0), __uint_as_float(b1));
        const float2 fast = Cbrt2<true>(x);
        const bool d0 = __float_as_uint(fast.x) != __float_as_uint(ss2dm::cbrt(x.x));
        const bool d1 = two && __float_as_uint(fast.y) != __float_as_uint(ss2dm::cbrt(x.y));
        bad += static_cast<unsigned long long>(d0) + static_cast<unsigned long long>(d1);
        if (d0 || d1) atomicMin(first_bad, d0 ? b0 : b1);
    }
    if (bad) atomicAdd(mismatches, bad);
}
}  // namespace

cudaError_t CheckCbrt(uint32_t first_bits, uint32_t last_bits, uint64_t* mismatches,
                      uint32_t* first_bad) {
    if (last_bits < first_bits || last_bits - first_bits == 0xffffffffu)
        return cudaErrorInvalidValue;
    unsigned long long* d_count = nullptr;
    cudaError_t e = cudaMalloc(&d_count, sizeof(unsigned long long) + sizeof(uint32_t));
    if (e != cudaSuccess) return e;
    uint32_t* d_first = reinterpret_cast<uint32_t*>(d_count + 1);
    const uint32_t none = 0xffffffffu;
    unsigned long long h_count = 0;
    uint32_t h_first = none;
    e = cudaMemset(d_count, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemcpy(d_first, &none, sizeof(none), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        CheckCbrtKernel<<<148 * 8, 256>>>(first_bits, last_bits - first_bits + 1, d_count,
                                          d_first);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h_count, d_count, sizeof(h_count), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&h_first, d_first, sizeof(h_first), cudaMemcpyDeviceToHost);
    cudaFree(d_count);
    if (e != cudaSuccess) return e;
    *mismatches = h_count;
    *first_bad = h_first;
    return cudaSuccess;
}

// SMs of the current device, looked up once per device.
static uint32_t DeviceSmCount() {
    static std::mutex mu;
    static int cached[64] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
        cudaGetLastError();
        return 148;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (cached[device] == 0 &&
        cudaDeviceGetAttribute(&cached[device], cudaDevAttrMultiProcessorCount, device) !=
            cudaSuccess) {
        cudaGetLastError();
        return 148;
    }
    return static_cast<uint32_t>(cached[device]);
}

template <bool kHalf>
void LaunchPrepareOf(const DevBatch& b, cudaStream_t stream) {
    // The table decode of a launch of at least two waves of 256-thread CTAs
    // runs as ten CTAs of 128 threads per SM: 64 1080p pairs 1.149 -> 1.075
    // ms. Smaller launches keep 256 threads, which finish a CTA's tile
    // sooner (one 1080p pair 27.0 against 28.7 us, one 256x256 pair 12.3
    // against 17.0 us).
    if (b.prep_blocks[0]) {
        if (b.prep_blocks[0] >= 2u * 5u * DeviceSmCount())
            PrepareKernel<0, kHalf, 128><<<b.prep_blocks[0], 128, 0, stream>>>(b);
        else
            PrepareKernel<0, kHalf, 256><<<b.prep_blocks[0], 256, 0, stream>>>(b);
    }
    // The YUV decode likewise, when every image of the launch has 4:2:0
    // chroma: eight 128-thread CTAs per SM with the smaller window (uneven
    // prepare 5.76 -> 5.56 ms).
    if (b.prep_blocks[1]) {
        if (b.yuv420 && b.prep_blocks[1] >= 2u * 5u * DeviceSmCount())
            PrepareKernel<1, kHalf, 128><<<b.prep_blocks[1], 128, 0, stream>>>(b);
        else
            PrepareKernel<1, kHalf, 256><<<b.prep_blocks[1], 256, 0, stream>>>(b);
    }
    if (b.prep_blocks[2]) PrepareKernel<2, kHalf, 256><<<b.prep_blocks[2], 256, 0, stream>>>(b);
}
cudaError_t LaunchPrepare(const DevBatch& b, cudaStream_t stream) {
    if (b.half)
        LaunchPrepareOf<true>(b, stream);
    else
        LaunchPrepareOf<false>(b, stream);
    return cudaGetLastError();
}

}  // namespace vqm_b200
