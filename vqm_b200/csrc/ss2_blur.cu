// Blur stage for sm_100a: the five 13-tap blurs, the SSIM' and edge maps and
// the compensated norm partials of every (pair, level, kept channel) output
// tile (reference: src/metrics/ssimulacra2/shaders/scale.comp).
//
// Rounding contract: the library is compiled with -fmad=false; every fused
// multiply-add is explicit and placed where VQM's shaders accumulate
// (scale.comp:149-333): each blurred value is w0*s0 followed by fused
// ascending taps, horizontal pass first. So the blurred quantities and map
// values are bit-identical to the CPU checker's FP32 path for bit-identical
// pyramid planes, whichever tile shape below computes them.
//
// One CTA computes a TW x TH output tile:
//   1. cp.async copies the (TW+12) x (TH+12) source window of both images in
//      16-byte chunks (2 columns x 2 rows of the row-pair planes, see
//      ss2_layout.h); chunks outside the plane are zero-filled, which is the
//      zero padding of scale.comp:107-124.
//   2. Horizontal pass: a thread takes one row pair and four output columns
//      and accumulates both rows at once with Blackwell's two-lane FP32
//      instructions (FFMA2); the five results go to row-major planes.
//   3. Vertical pass: a thread takes a column pair and four output rows,
//      again two lanes per instruction, then evaluates the maps of its eight
//      pixels and keeps six running sums.
//   4. The CTA's six sums are combined with two-sum compensation into one
//      partial per CTA (its tile, or its strip of tiles below).
//   5. The CTA that writes a segment's last partial adds the segment's
//      partials in FP64, and the one that completes a pair's last segment
//      turns the pair's sums into its 108 norms and FP64 score (the
//      reference's reduce.comp:21-63, ReadResult in vulkan.cc:545-583 and
//      Score in score.cc:118-163): no separate finalize launch. Counters
//      decide who is last; no CTA ever waits for another.
// A persistent form keeps each CTA resident and copies its next tile's
// window into a second buffer while it computes the current one; a strip
// form walks a few tiles down one column and reuses the horizontal results
// of the rows the windows share.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <mutex>
#include <queue>
#include <unordered_map>
#include <utility>
#include <vector>

#include "ss2_detmath.h"
#include "ss2_device.cuh"
#include "ss2_kernels.h"
#include "ss2_layout.h"

namespace vqm_b200 {
namespace {

// score.cc:38-87, flat rows channel * scales + scale.
__constant__ double c_weights[18][6];

// The last prefix entry <= index (start[0] == 0 <= index < start[count]).
__device__ __forceinline__ uint32_t FindSlot(const uint32_t* __restrict__ start,
                                             uint32_t count, uint32_t index) {
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&start[mid]) <= index) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Compensated (two-sum) addition of (s2, c2) into (s, c).
__device__ __forceinline__ void TwoSumAdd(float& s, float& c, float s2, float c2) {
    const float t = __fadd_rn(s, s2);
    const float bp = __fsub_rn(t, s);
    const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(s2, bp));
    s = t;
    c = __fadd_rn(__fadd_rn(c, c2), e);
}

template <int TW, int TH, int NT>
struct Tile {
    static constexpr int SW = TW + 2 * kRadius;  // source columns
    static constexpr int SH = TH + 2 * kRadius;  // source rows
    static constexpr int RP = SH / 2;            // source row pairs
    static constexpr int CP = SW / 2;            // 16-byte chunks per source row pair
    // Floats per source row pair: 2 * SW plus 4 of padding, so that the row
    // pair stride is 28 banks mod 32 (see HorizontalPass).
    static constexpr int SRS = 2 * SW + 4;
    static constexpr int IMG = RP * SRS;  // floats per source image
    static constexpr int KH = 4;          // output columns per horizontal task
    static constexpr int NG = TW / KH;    // column groups per row pair
    static constexpr int HT = RP * NG;    // horizontal tasks
    static constexpr int RV = 4;          // output rows per vertical task
    static constexpr int VT = (TW / 2) * (TH / RV);
    static constexpr size_t kSrcBytes = sizeof(float) * 2 * IMG;
    static constexpr size_t kHqBytes = sizeof(float) * 5 * SH * TW;
    static_assert(TW % 32 == 0, "whole warps of column pairs in the vertical pass");
    static_assert(TH % RV == 0 && RP % 2 == 0 && NG % 4 == 0, "tile shape");
    static_assert(SRS % 32 == 28, "bank spread of the horizontal loads");
    static_assert(NT % 32 == 0 && NT >= 96, "whole warps, 16 lanes per sum");
    static_assert(kSrcBytes >= sizeof(float) * 12 * NT, "the reduction reuses the source buffer");
};

// Where one output tile's planes, geometry and partial slot are.
struct TileRef {
    const float* pa;
    const float* pb;
    uint32_t pitch;    // floats per row pair
    uint32_t partial;  // index of the tile's partial
    uint32_t segment;  // index of its segment
    int w, h, x0, y0;
};

// Output tile (tx, ty) of a segment. With half planes pa and pb point at
// binary16 elements (typed float* only to share the struct).
template <int TW, int TH, bool kHalf = false>
__device__ __forceinline__ TileRef SegmentTile(const DevBatch& batch, const DevSegment& seg,
                                               uint32_t si, uint32_t tx, uint32_t ty) {
    const DevPair& P = batch.pair[seg.pair];
    TileRef t;
    if (kHalf) {
        const __half* a = reinterpret_cast<const __half*>(P.pyramid) + P.plane_off[seg.level][seg.channel];
        t.pa = reinterpret_cast<const float*>(a);
        t.pb = reinterpret_cast<const float*>(a + P.image_stride);
    } else {
        t.pa = P.pyramid + P.plane_off[seg.level][seg.channel];
        t.pb = t.pa + P.image_stride;
    }
    t.pitch = P.pitch[seg.level];
    t.w = static_cast<int>(P.w[seg.level]);
    t.h = static_cast<int>(P.h[seg.level]);
    t.x0 = static_cast<int>(tx * TW);
    t.y0 = static_cast<int>(ty * TH);
    t.partial = seg.partial_first + ty * seg.tiles_x + tx;
    t.segment = si;
    return t;
}

// Block `blk` of a one-tile-per-block launch (blur_start counts tiles).
template <int TW, int TH, bool kHalf = false>
__device__ __forceinline__ TileRef LocateTile(const DevBatch& batch, uint32_t blk) {
    const uint32_t si = FindSlot(batch.blur_start, batch.segments, blk);
    const DevSegment seg = batch.seg[si];
    const uint32_t tile = blk - __ldg(&batch.blur_start[si]);
    const uint32_t ty = tile / seg.tiles_x;
    return SegmentTile<TW, TH, kHalf>(batch, seg, si, tile - ty * seg.tiles_x, ty);
}

// Asynchronous 16-byte global-to-shared copy; a source size of 0 writes
// zeros and reads nothing.
__device__ __forceinline__ void CpAsync16(uint32_t dst, const float* src, bool valid) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void CpAsyncCommit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void CpAsyncWait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issues the copies of one tile's two source windows into `buf`: chunk
// (rp, cp) of the window is the 2x2 block at window column 2cp, row 2rp.
// Row pairs below `rp_begin` are left as they are. A thread keeps one chunk
// column, cp = tid mod CP, and steps down the rows NT / CP at a time, so its
// column test and addresses are set once and advance by constants.
template <int TW, int TH, int NT>
__device__ __forceinline__ void IssueTileLoads(float* buf, const TileRef& t, int rp_begin = 0) {
    using T = Tile<TW, TH, NT>;
    constexpr int kRowsPerPass = NT / T::CP;
    static_assert(kRowsPerPass >= 1, "a pass covers at least one row of chunks");
    const int cp = static_cast<int>(threadIdx.x) % T::CP;
    const int r = static_cast<int>(threadIdx.x) / T::CP;
    if (r >= kRowsPerPass) return;
    const uint32_t wp = static_cast<uint32_t>(t.w + 1) >> 1;  // chunks per row pair
    const uint32_t hp = static_cast<uint32_t>(t.h + 1) >> 1;  // row pairs
    const int gx = (t.x0 >> 1) - kRadius / 2 + cp, ry0 = (t.y0 >> 1) - kRadius / 2;
    const bool column_in = static_cast<uint32_t>(gx) < wp;
    const uint32_t col_off = 4u * static_cast<uint32_t>(gx);
    uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(buf)) +
                   4u * static_cast<uint32_t>((rp_begin + r) * T::SRS + 4 * cp);
    for (int rp = rp_begin + r; rp < T::RP; rp += kRowsPerPass) {
        const int gy = ry0 + rp;
        const bool in = column_in && static_cast<uint32_t>(gy) < hp;
        const uint32_t off = in ? static_cast<uint32_t>(gy) * t.pitch + col_off : 0u;
        CpAsync16(dst, t.pa + off, in);
        CpAsync16(dst + 4u * T::IMG, t.pb + off, in);
        dst += 4u * kRowsPerPass * T::SRS;
    }
}

// Half planes: 16-byte chunks are 4 columns x 2 rows of binary16 elements,
// so the copied window starts 8 columns left of the tile (4-column aligned,
// as x0 is) and spans TW + 16 columns; it is staged in `staging` (the
// horizontal planes' space, unused until the horizontal pass) and widened to
// the float window by ConvertHalfTile.
template <int TW, int TH, int NT>
struct HalfWindow {
    using T = Tile<TW, TH, NT>;
    static constexpr int CQ = (TW + 16) / 4;              // chunks per row pair
    static constexpr int CHUNKS = T::RP * CQ;             // per image
    static constexpr size_t kBytes = 2 * CHUNKS * 16;
    static_assert(kBytes <= T::kHqBytes, "the staging fits the horizontal planes");
};

template <int TW, int TH, int NT>
__device__ __forceinline__ void IssueTileLoadsHalf(unsigned char* staging, const TileRef& t) {
    using H = HalfWindow<TW, TH, NT>;
    const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(staging));
    const uint32_t wq = static_cast<uint32_t>(t.w + 3) >> 2;  // chunks per row pair
    const uint32_t hp = static_cast<uint32_t>(t.h + 1) >> 1;  // row pairs
    const int cq0 = (t.x0 >> 2) - 2, ry0 = (t.y0 >> 1) - kRadius / 2;
    const __half* pa = reinterpret_cast<const __half*>(t.pa);
    const __half* pb = reinterpret_cast<const __half*>(t.pb);
    for (int k = threadIdx.x; k < H::CHUNKS; k += NT) {
        const int rp = k / H::CQ, q = k - rp * H::CQ;
        const int gy = ry0 + rp, gq = cq0 + q;
        const bool in = static_cast<uint32_t>(gy) < hp && static_cast<uint32_t>(gq) < wq;
        const uint32_t off = in ? static_cast<uint32_t>(gy) * t.pitch + 8u * static_cast<uint32_t>(gq)
                                : 0u;
        const uint32_t dst = base + 16u * static_cast<uint32_t>(k);
        CpAsync16(dst, reinterpret_cast<const float*>(pa + off), in);
        CpAsync16(dst + 16u * H::CHUNKS, reinterpret_cast<const float*>(pb + off), in);
    }
}

// The staged binary16 window to the float row-pair window of `src`.
template <int TW, int TH, int NT>
__device__ __forceinline__ void ConvertHalfTile(const unsigned char* staging, float* src) {
    using T = Tile<TW, TH, NT>;
    using H = HalfWindow<TW, TH, NT>;
    for (int k = threadIdx.x; k < 2 * H::CHUNKS; k += NT) {
        const int img = k >= H::CHUNKS ? 1 : 0;
        const int kk = k - img * H::CHUNKS;
        const int rp = kk / H::CQ, q = kk - rp * H::CQ;
        const uint4 v = *reinterpret_cast<const uint4*>(staging + 16 * k);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        float* row = src + img * T::IMG + rp * T::SRS;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int col = 4 * q + i - 2;  // float window column (x0 - 6 based)
            if (col < 0 || col >= T::SW) continue;
            const __half2 h = *reinterpret_cast<const __half2*>(&w[i]);
            *reinterpret_cast<float2*>(row + 2 * col) = __half22float2(h);
        }
    }
}

__device__ __forceinline__ float2 Pack(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 Neg(float2 v) { return make_float2(-v.x, -v.y); }

// The reciprocal of both lanes' divisors for the maps' division: an estimate
// from the special-function unit (within 1 ulp) and one Newton step
// r += r (1 - b r), which leaves ~2^-46 of error before its single rounding;
// ss2dm::recipf takes three steps from a bit seed and leaves ~2^-34, so the
// two reciprocals differ by an ulp for about 1.6e-4 of divisors.
__device__ __forceinline__ float RcpEstimate(float b) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    return r;
}
__device__ __forceinline__ float2 Recip2(float2 b) {
    const float2 r = make_float2(RcpEstimate(b.x), RcpEstimate(b.y));
    return __ffma2_rn(r, __ffma2_rn(Neg(b), r, Pack(1.0f)), r);
}

// The maps' division of both lanes, two lanes per instruction: Recip2 and
// ss2dm::divf's final step, q0 = a r corrected once with the residual
// a - b q0 (exact in one fused multiply-add), which absorbs a 1-ulp
// difference in r: the quotient equals ss2dm::divf's unless it lies within
// ~2^-46 of a rounding boundary. The library checks every divisor of the
// maps' band [2^-11, 2^4] (the SSIM' denominator is at least 0.0009, the edge
// map's at least 1) at sixteen quotient values on the device
// (vqm_cu_ss2_check_division, run by the GPU tests).
__device__ __forceinline__ float2 Div2(float2 a, float2 b) {
    const float2 r = Recip2(b);
    const float2 q0 = __fmul2_rn(a, r);
    return __ffma2_rn(__ffma2_rn(Neg(b), q0, a), r, q0);
}

// Horizontal pass (scale.comp:149-207): row pair rp, output columns
// c0..c0+3, all five quantities, both rows per instruction, for the row
// pairs from `rp_begin` (even) on.
//
// Task -> (rp, column group): within every 8 lanes, lanes 0-3 take four
// column groups of row pair rp and lanes 4-7 the same groups of rp + 1. The
// source row pair stride is 28 banks mod 32, so the quarter warp's eight
// 16-byte loads cover all 32 banks once.
//
// The horizontal planes are row-pair blocks too: row pair rp is TW / 2
// 16-byte blocks, block b holding columns 2b, 2b + 1 of row 2rp and then of
// row 2rp + 1, so the vertical pass reads two rows of its column pair with
// one load. On odd row pairs block b is stored at b ^ 1, which keeps the
// quarter warp's stores (row pairs rp and rp + 1, even and odd) apart.
template <int TW, int TH, int NT>
__device__ __forceinline__ void HorizontalPass(const float2 (&taps)[kTaps], const float* src,
                                               float* hq, int rp_begin = 0) {
    using T = Tile<TW, TH, NT>;
    constexpr int KH = T::KH;
    const int tasks = T::HT - rp_begin * T::NG;
    for (int task = threadIdx.x; task < tasks; task += NT) {
        const int cg_lo = task & 3, rp_lo = (task >> 2) & 1, rest = task >> 3;
        const int cg = (rest % (T::NG / 4)) * 4 + cg_lo;
        const int rp = rp_begin + (rest / (T::NG / 4)) * 2 + rp_lo;
        const float* ra = src + rp * T::SRS + 2 * KH * cg;
        const float* rb = ra + T::IMG;
        float2 A[KH + 12], B[KH + 12];
#pragma unroll
        for (int j = 0; j < KH + 12; j += 2) {
            const float4 va = *reinterpret_cast<const float4*>(ra + 2 * j);
            const float4 vb = *reinterpret_cast<const float4*>(rb + 2 * j);
            A[j] = make_float2(va.x, va.y);
            A[j + 1] = make_float2(va.z, va.w);
            B[j] = make_float2(vb.x, vb.y);
            B[j + 1] = make_float2(vb.z, vb.w);
        }
        float* out = hq + rp * 2 * TW + 8 * cg;
        const int flip = (rp & 1) << 2;  // block 2cg + h at 2cg + (h ^ (rp & 1))
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            float2 S[KH + 12];
#pragma unroll
            for (int j = 0; j < KH + 12; ++j)
                S[j] = q == 0 ? A[j]
                     : q == 1 ? B[j]
                     : q == 2 ? __fmul2_rn(A[j], A[j])
                     : q == 3 ? __fmul2_rn(B[j], B[j])
                              : __fmul2_rn(A[j], B[j]);
            float2 acc[KH];
#pragma unroll
            for (int k = 0; k < KH; ++k) acc[k] = __fmul2_rn(taps[0], S[k]);
#pragma unroll
            for (int tap = 1; tap < kTaps; ++tap) {
                const float2 wt = taps[tap];
#pragma unroll
                for (int k = 0; k < KH; ++k) acc[k] = __ffma2_rn(wt, S[k + tap], acc[k]);
            }
            float* plane = out + q * T::SH * TW;
            *reinterpret_cast<float4*>(plane + flip) =
                make_float4(acc[0].x, acc[1].x, acc[0].y, acc[1].y);
            *reinterpret_cast<float4*>(plane + (4 ^ flip)) =
                make_float4(acc[2].x, acc[3].x, acc[2].y, acc[3].y);
        }
    }
}

// Vertical pass (scale.comp:211-301) on column pairs and the maps
// (scale.comp:305-333) of each task's eight pixels, added into `sum`. With
// kEdge, pixels outside the level contribute 0 (their inputs are the zero
// padding, so every map value is finite before it is dropped).
template <int TW, int TH, int NT, bool kEdge>
__device__ __forceinline__ void VerticalMaps(const float2 (&taps)[kTaps], const float* src,
                                             const float* hq, const TileRef& t,
                                             float2 (&sum)[6]) {
    using T = Tile<TW, TH, NT>;
    constexpr int RV = T::RV;
    for (int task = threadIdx.x; task < T::VT; task += NT) {
        const int c = (task % (TW / 2)) * 2;
        const int r0 = (task / (TW / 2)) * RV;
        // Row pair r0 / 2 + i holds column pair c in block c / 2, at
        // c / 2 ^ 1 when i is odd (r0 / 2 being even).
        const int blocks[2] = {2 * c, 2 * (c ^ 2)};
        float2 V[5][RV];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const float* plane = hq + q * T::SH * TW + r0 * TW;
            float2 M[RV + 12];
#pragma unroll
            for (int i = 0; i < (RV + 12) / 2; ++i) {
                const float4 v =
                    *reinterpret_cast<const float4*>(plane + i * 2 * TW + blocks[i & 1]);
                M[2 * i] = make_float2(v.x, v.y);
                M[2 * i + 1] = make_float2(v.z, v.w);
            }
#pragma unroll
            for (int j = 0; j < RV; ++j) {
                float2 acc = __fmul2_rn(taps[0], M[j]);
#pragma unroll
                for (int k = 1; k < kTaps; ++k) acc = __ffma2_rn(taps[k], M[j + k], acc);
                V[q][j] = acc;
            }
        }
        // The raw values of rows r0 + 6 .. r0 + 9, columns c + 6 and c + 7:
        // one 16-byte load per row pair and image.
        float4 raw1[RV / 2], raw2[RV / 2];
#pragma unroll
        for (int p = 0; p < RV / 2; ++p) {
            const float* at = src + ((r0 + kRadius) / 2 + p) * T::SRS + 2 * (c + kRadius);
            raw1[p] = *reinterpret_cast<const float4*>(at);
            raw2[p] = *reinterpret_cast<const float4*>(at + T::IMG);
        }
        const int out_x = t.x0 + c;
#pragma unroll
        for (int j = 0; j < RV; ++j) {
            const float2 mu1 = V[0][j], mu2 = V[1][j];
            const float2 dm = __fadd2_rn(mu1, Neg(mu2));
            const float2 num_m = __ffma2_rn(Neg(dm), dm, Pack(1.0f));
            const float2 num_s =
                __ffma2_rn(Pack(2.0f), __ffma2_rn(Neg(mu1), mu2, V[4][j]), Pack(0.0009f));
            const float2 denom = __fadd2_rn(
                __fadd2_rn(__ffma2_rn(Neg(mu1), mu1, V[2][j]), __ffma2_rn(Neg(mu2), mu2, V[3][j])),
                Pack(0.0009f));
            const float2 numer = __ffma2_rn(Neg(num_m), num_s, denom);
            const float2 q = Div2(numer, denom);
            float2 d = make_float2(fmaxf(q.x, 0.0f), fmaxf(q.y, 0.0f));
            const float4 r1 = raw1[j >> 1], r2v = raw2[j >> 1];
            const float2 img1 = (j & 1) ? make_float2(r1.y, r1.w) : make_float2(r1.x, r1.z);
            const float2 img2 = (j & 1) ? make_float2(r2v.y, r2v.w) : make_float2(r2v.x, r2v.z);
            float2 e2 = __fadd2_rn(img2, Neg(mu2));
            float2 e1 = __fadd2_rn(img1, Neg(mu1));
            e2 = make_float2(fabsf(e2.x), fabsf(e2.y));
            e1 = make_float2(fabsf(e1.x), fabsf(e1.y));
            const float2 dist = __fadd2_rn(Pack(1.0f), e2);
            const float2 orig = __fadd2_rn(Pack(1.0f), e1);
            const float2 diff = __fadd2_rn(dist, Neg(orig));
            const float2 d1 = Div2(diff, orig);
            float2 ring = make_float2(fmaxf(d1.x, 0.0f), fmaxf(d1.y, 0.0f));
            float2 blur = make_float2(fmaxf(-d1.x, 0.0f), fmaxf(-d1.y, 0.0f));
            if (kEdge) {
                const bool vy = t.y0 + r0 + j < t.h;
                const bool v0 = vy && out_x < t.w, v1 = vy && out_x + 1 < t.w;
                d = make_float2(v0 ? d.x : 0.0f, v1 ? d.y : 0.0f);
                ring = make_float2(v0 ? ring.x : 0.0f, v1 ? ring.y : 0.0f);
                blur = make_float2(v0 ? blur.x : 0.0f, v1 ? blur.y : 0.0f);
            }
            const float2 dd = __fmul2_rn(d, d);
            const float2 rr = __fmul2_rn(ring, ring), bb = __fmul2_rn(blur, blur);
            sum[0] = __fadd2_rn(sum[0], d);
            sum[1] = __fadd2_rn(sum[1], __fmul2_rn(dd, dd));
            sum[2] = __fadd2_rn(sum[2], ring);
            sum[3] = __fadd2_rn(sum[3], __fmul2_rn(rr, rr));
            sum[4] = __fadd2_rn(sum[4], blur);
            sum[5] = __fadd2_rn(sum[5], __fmul2_rn(bb, bb));
        }
    }
}

// Scratch of the reduction: 12 arrays of NT floats, here back to back
// (the source window once every thread is past its last read of it).
template <int NT>
struct LinearScratch {
    float* base;
    __device__ __forceinline__ float* operator()(int a) const { return base + a * NT; }
};

// The CTA's six sums as one compensated partial each (scale.comp:395-436,
// with two-sum compensation in place of the plain ladder): every thread
// folds its two lanes, 16 lanes per sum add the block's values, and a
// 16-lane butterfly finishes. `red(a)` is scratch array a (a < 12) of NT
// floats. Ends with a barrier.
template <int NT, class Scratch>
__device__ __forceinline__ void ReducePartials(const float2 (&sum)[6], Scratch red, double* out) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float s = sum[k].x, c = 0.0f;
        TwoSumAdd(s, c, sum[k].y, 0.0f);
        red(2 * k)[tid] = s;
        red(2 * k + 1)[tid] = c;
    }
    __syncthreads();
    if (tid < 96) {  // warps 0-2, whole
        const int k = tid >> 4, i = tid & 15;
        const float* rs = red(2 * k);
        const float* rc = red(2 * k + 1);
        float s = rs[i], c = rc[i];
#pragma unroll
        for (int j = i + 16; j < NT; j += 16) TwoSumAdd(s, c, rs[j], rc[j]);
#pragma unroll
        for (int off = 8; off > 0; off >>= 1) {
            const float s2 = __shfl_xor_sync(0xffffffffu, s, off);
            const float c2 = __shfl_xor_sync(0xffffffffu, c, off);
            TwoSumAdd(s, c, s2, c2);
        }
        if (i == 0) out[k] = static_cast<double>(s) + static_cast<double>(c);
    }
    __syncthreads();
}

// score.cc:118-163 in FP64 on the device, from the weighted sum of the
// norms' magnitudes (`error`, the sum of w * |norm| over the 108 features).
__device__ __noinline__ double ScoreFromError(double error) {
    if (!isfinite(error)) return nan("");
    const double scaled = error * 0.9562382616834844;
    const double mapped = 2.326765642916932 * scaled -
                          0.020884521182843837 * scaled * scaled +
                          6.248496625763138e-05 * scaled * scaled * scaled;
    if (!isfinite(mapped)) return nan("");
    if (mapped > 0.0) return 100.0 - 10.0 * pow(mapped, 0.6276336467831387);
    return 100.0;
}

// The pair's 108 norms from its segments' FP64 sums (vulkan.cc:545-583:
// mean = sum / (W_l H_l), 4-norm = sqrt(sqrt(sum4 / (W_l H_l)))), written
// straight into its result block (zeros for pruned channels and levels past
// its scales), then its score and scale count. Every thread of the CTA that
// completes the pair takes one of the 108 slots, each written once (the
// result block can be host memory the device writes across the bus): the
// norm of a kept (level, channel), a division and two square roots in FP64
// (one thread doing all of them in turn was most of a small launch's time),
// and its weighted magnitude; the weighted sum is a fixed butterfly in each
// warp and the warps in turn (score.cc's sum in another order: equal to
// ~1e-15, and the same on every run), and thread 0 maps it to the score.
// `red` is shared scratch for NT / 32 doubles. Out of line, as it runs once
// per pair and should cost the blur loops no registers.
template <int NT>
__device__ __noinline__ void WritePairResult(const DevBatch& batch, const DevPair& P,
                                             double* red) {
    // score.cc's weight slot of each norm f (SSIM' mean and 4-norm, ringing
    // mean and 4-norm, blurring mean and 4-norm).
    constexpr uint32_t kWeightSlot = 0x524130u;  // 4 bits per f: 0, 3, 1, 4, 2, 5
    const uint32_t tid = threadIdx.x;
    double* out = P.result;
    double term = 0.0;
    for (uint32_t i = tid; i < 108; i += NT) {
        // Slot i: level l, then Ssimulacra2Scale's order (avg_ssim[c * 2 +
        // n], then avg_edgediff[c * 4 + n]).
        const uint32_t l = i / 18, at = i - 18 * l;
        const uint32_t c = at < 6 ? at / 2 : (at - 6) / 4;
        const uint32_t f = at < 6 ? at % 2 : 2 + (at - 6) % 4;  // the segment's sum
        double norm = 0.0;
        if (l < P.levels && ((P.mask[l] >> c) & 1u)) {
            // Segments run level by level over the kept channels.
            uint32_t k = __popc(P.mask[l] & ((1u << c) - 1u));
            for (uint32_t m = 0; m < l; ++m) k += __popc(P.mask[m] & 7u);
            const size_t sk = static_cast<size_t>(P.seg_first) + k;
            const double inv =
                1.0 / (static_cast<double>(P.w[l]) * static_cast<double>(P.h[l]));
            const double v = inv * __ldcg(batch.seg_sums + sk * 6 + f);
            norm = (f & 1u) ? sqrt(sqrt(v)) : v;
            term += c_weights[c * P.levels + l][(kWeightSlot >> (4 * f)) & 15u] * fabs(norm);
        }
        out[i] = norm;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) term += __shfl_xor_sync(0xffffffffu, term, off);
    if (tid % 32 == 0) red[tid / 32] = term;
    __syncthreads();
    if (tid == 0) {
        double error = 0.0;
        for (int w = 0; w < NT / 32; ++w) error += red[w];
        out[kResultScore] = ScoreFromError(error);
        out[kResultScales] = static_cast<double>(P.levels);
        out[kResultStatus] = 0.0;
    }
}

// Called by every thread of a blur CTA once its partial of segment `si` is
// written (after a barrier). The CTA whose partial completes the segment
// adds the segment's partials in FP64 in a fixed order (thread t takes
// partials t, t + NT, ..., then a butterfly and the warps in turn), so a
// result repeats bit for bit; the CTA whose segment completes the pair
// writes the pair's result. Each counter is reset by the CTA that finds it
// complete, so the next launch starts from zero. `scratch` is shared memory
// for 7 * NT / 32 + 2 doubles that no thread still reads.
// The CTA that completed segment `si`: its FP64 sum, then the pair's result
// if the segment completes the pair.
template <int NT>
__device__ __forceinline__ void SumSegment(const DevBatch& batch, uint32_t si, double* scratch) {
    const uint32_t tid = threadIdx.x;
    volatile uint32_t* flag = reinterpret_cast<volatile uint32_t*>(scratch + 6 * (NT / 32));
    const DevSegment seg = batch.seg[si];
    __threadfence();
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (uint32_t t = tid; t < seg.partials; t += NT) {
        const double* p = batch.partials + (static_cast<size_t>(seg.partial_first) + t) * 6;
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] += __ldcg(p + k);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
    if (tid % 32 == 0)
#pragma unroll
        for (int k = 0; k < 6; ++k) scratch[(tid / 32) * 6 + k] = acc[k];
    __syncthreads();
    if (tid < 6) {
        double sum = 0.0;
        for (int w = 0; w < NT / 32; ++w) sum += scratch[w * 6 + tid];
        batch.seg_sums[static_cast<size_t>(si) * 6 + tid] = sum;
        __threadfence();
    }
    __syncthreads();
    const DevPair& P = batch.pair[seg.pair];
    if (tid == 0) {
        batch.seg_done[si] = 0u;
        flag[1] = atomicAdd(&batch.pair_done[seg.pair], 1u) + 1u == P.seg_count;
    }
    __syncthreads();
    if (!flag[1]) return;
    __threadfence();
    WritePairResult<NT>(batch, P, scratch + 6 * (NT / 32) + 2);
    if (tid == 0) batch.pair_done[seg.pair] = 0u;
}

template <int NT>
__device__ __forceinline__ void FinishSegment(const DevBatch& batch, uint32_t si,
                                              double* scratch) {
    volatile uint32_t* flag = reinterpret_cast<volatile uint32_t*>(scratch + 6 * (NT / 32));
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's partial, before the count that publishes it
        flag[0] = atomicAdd(&batch.seg_done[si], 1u) + 1u == __ldg(&batch.seg[si].partials);
    }
    __syncthreads();
    if (flag[0]) SumSegment<NT>(batch, si, scratch);
}

template <int TW, int TH, int NT>
__device__ __forceinline__ void ComputeTile(float* src, float* hq, const TileRef& t,
                                            const DevBatch& batch) {
    HorizontalPass<TW, TH, NT>(batch.taps2, src, hq);
    __syncthreads();
    float2 sum[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sum[k] = make_float2(0.0f, 0.0f);
    if (t.x0 + TW <= t.w && t.y0 + TH <= t.h)
        VerticalMaps<TW, TH, NT, false>(batch.taps2, src, hq, t, sum);
    else
        VerticalMaps<TW, TH, NT, true>(batch.taps2, src, hq, t, sum);
    __syncthreads();  // the reduction overwrites the source window
    ReducePartials<NT>(sum, LinearScratch<NT>{src},
                       batch.partials + static_cast<size_t>(t.partial) * 6);
    FinishSegment<NT>(batch, t.segment, reinterpret_cast<double*>(src));
}

// One output tile per CTA; MB CTAs per SM is the occupancy the shared
// memory allows, which bounds the registers per thread.
template <int TW, int TH, int NT, int MB, bool kHalf = false>
__global__ void __launch_bounds__(NT, MB) Ss2BlurKernel(DevBatch batch) {
    using T = Tile<TW, TH, NT>;
    extern __shared__ __align__(16) unsigned char smem[];
    float* src = reinterpret_cast<float*>(smem);
    float* hq = reinterpret_cast<float*>(smem + T::kSrcBytes);
    const TileRef t = LocateTile<TW, TH, kHalf>(batch, blockIdx.x);
    if (kHalf) IssueTileLoadsHalf<TW, TH, NT>(smem + T::kSrcBytes, t);
    else IssueTileLoads<TW, TH, NT>(src, t);
    CpAsyncCommit();
    CpAsyncWait<0>();
    __syncthreads();
    if (kHalf) {
        ConvertHalfTile<TW, TH, NT>(smem + T::kSrcBytes, src);
        __syncthreads();
    }
    ComputeTile<TW, TH, NT>(src, hq, t, batch);
}

// Persistent: each CTA walks tiles blockIdx.x, + gridDim.x, ... and copies
// tile i+1's window into its second buffer while it computes tile i.
template <int TW, int TH, int NT, int MB>
__global__ void __launch_bounds__(NT, MB) Ss2BlurPersistentKernel(DevBatch batch) {
    using T = Tile<TW, TH, NT>;
    extern __shared__ __align__(16) unsigned char smem[];
    float* const buf0 = reinterpret_cast<float*>(smem);
    constexpr int kBufFloats = static_cast<int>(T::kSrcBytes / sizeof(float));
    float* hq = reinterpret_cast<float*>(smem + 2 * T::kSrcBytes);
    const uint32_t total = batch.blur_blocks;
    uint32_t tile = blockIdx.x;
    if (tile >= total) return;
    TileRef cur = LocateTile<TW, TH>(batch, tile);
    IssueTileLoads<TW, TH, NT>(buf0, cur);
    CpAsyncCommit();
    int b = 0;
    for (; tile < total; tile += gridDim.x) {
        const uint32_t next = tile + gridDim.x;
        float* const now = buf0 + b * kBufFloats;
        TileRef nxt = cur;
        if (next < total) {
            nxt = LocateTile<TW, TH>(batch, next);
            IssueTileLoads<TW, TH, NT>(buf0 + (b ^ 1) * kBufFloats, nxt);
        }
        CpAsyncCommit();   // possibly empty, so the group count stays uniform
        CpAsyncWait<1>();  // everything but the newest group: this tile's
        __syncthreads();
        ComputeTile<TW, TH, NT>(now, hq, cur, batch);
        // The segment and pair epilogues use this buffer as scratch; the
        // next iteration copies a window into it.
        __syncthreads();
        cur = nxt;
        b ^= 1;
    }
    CpAsyncWait<0>();
}

// Strips: a CTA computes up to S vertically consecutive tiles of one column.
// Tile k + 1's window starts TH rows below tile k's, so the horizontal
// results of its first 12 rows are tile k's last 12, already in `hq`: they
// are moved up instead of being computed again, and only the window's rows
// 6.. are copied in (6..11 for the maps' raw values, 12.. for the horizontal
// pass). Every blurred value and map value is computed by the same
// instructions as in the one-tile kernel, so they are bit-identical to it.
// Each thread keeps its six FP32 sums across the strip's tiles (at most
// 4 S map values per lane) and the CTA reduces them once, with two-sum
// compensation, into one partial for the strip: the compensated reduction,
// its barriers and its scalar adds run once per strip instead of once per
// tile. The partial's grouping differs from one tile per CTA, so results
// agree with that kernel to rounding (~1e-7 relative), not bit for bit.
//
// The reduction's scratch is rows 12..TH-1 of the horizontal planes, free
// once the last tile's vertical pass is done.
template <int TW, int TH, int NT>
struct HqScratch {
    using T = Tile<TW, TH, NT>;
    static constexpr int kPerPlane = (TH - 2 * kRadius) * TW / NT;  // arrays per plane
    static_assert(5 * kPerPlane >= 12, "the reduction fits the free horizontal rows");
    float* hq;
    __device__ __forceinline__ float* operator()(int a) const {
        return hq + (a / kPerPlane) * T::SH * TW + 2 * kRadius * TW + (a % kPerPlane) * NT;
    }
};

// Horizontal rows TH..TH+11 of every quantity to rows 0..11. TH is a
// multiple of 4, so a row and its destination share the store swizzle.
// A thread moves float4 j of every quantity's halo (j < 96 for 32-wide
// tiles: one pass for 128 threads), at constant offsets from one address.
template <int TW, int TH, int NT>
__device__ __forceinline__ void MoveHalo(float* hq) {
    using T = Tile<TW, TH, NT>;
    constexpr int kRowVec = TW / 4;                   // float4 per row
    constexpr int kPlaneVec = 2 * kRadius * kRowVec;  // float4 per plane's halo
    static_assert(TH % 4 == 0, "swizzle parity");
    for (int j = threadIdx.x; j < kPlaneVec; j += NT) {
        float4* at = reinterpret_cast<float4*>(hq) + j;
#pragma unroll
        for (int q = 0; q < 5; ++q) at[q * (T::SH * TW / 4)] = at[q * (T::SH * TW / 4) + TH * kRowVec];
    }
}

// Strip `block` of the launch (blur_start counts strips).
template <int TW, int TH, int NT, int S>
__device__ __forceinline__ void RunStrip(const DevBatch& batch, uint32_t block, float* src,
                                         float* hq) {
    const uint32_t si = FindSlot(batch.blur_start, batch.segments, block);
    const DevSegment seg = batch.seg[si];
    const uint32_t strip = block - __ldg(&batch.blur_start[si]);
    const uint32_t sy = strip / seg.tiles_x;
    const uint32_t tiles_y = seg.tiles / seg.tiles_x;
    const uint32_t ty0 = sy * S;
    const int count = static_cast<int>(min(static_cast<uint32_t>(S), tiles_y - ty0));
    TileRef t = SegmentTile<TW, TH>(batch, seg, si, strip - sy * seg.tiles_x, ty0);
    IssueTileLoads<TW, TH, NT>(src, t);
    CpAsyncCommit();
    float2 sum[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) sum[i] = make_float2(0.0f, 0.0f);
    for (int k = 0; k < count; ++k) {
        CpAsyncWait<0>();
        __syncthreads();
        HorizontalPass<TW, TH, NT>(batch.taps2, src, hq, k == 0 ? 0 : kRadius);
        __syncthreads();
        if (t.x0 + TW <= t.w && t.y0 + TH <= t.h)
            VerticalMaps<TW, TH, NT, false>(batch.taps2, src, hq, t, sum);
        else
            VerticalMaps<TW, TH, NT, true>(batch.taps2, src, hq, t, sum);
        __syncthreads();  // every read of the window and of `hq` is done
        if (k + 1 < count) {
            t.y0 += TH;
            IssueTileLoads<TW, TH, NT>(src, t, kRadius / 2);
            CpAsyncCommit();
            MoveHalo<TW, TH, NT>(hq);
        }
    }
    ReducePartials<NT>(sum, HqScratch<TW, TH, NT>{hq},
                       batch.partials + (static_cast<size_t>(seg.partial_first) + strip) * 6);
    FinishSegment<NT>(batch, si, reinterpret_cast<double*>(src));
}

template <int TW, int TH, int NT, int MB, int S>
__global__ void __launch_bounds__(NT, MB) Ss2BlurStripKernel(DevBatch batch) {
    using T = Tile<TW, TH, NT>;
    extern __shared__ __align__(16) unsigned char smem[];
    RunStrip<TW, TH, NT, S>(batch, blockIdx.x, reinterpret_cast<float*>(smem),
                            reinterpret_cast<float*>(smem + T::kSrcBytes));
}

// A tile queue: as many CTAs as the device holds at once, each taking the
// next strip from a device counter (batch.blur_queue[0]) until none is left.
// The strips are the launch's work items in segment order (pair, level,
// channel); a CTA never waits for another. The last CTA to leave resets the
// counter and the exit count (blur_queue[1]) for the next launch.
template <int TW, int TH, int NT, int MB, int S>
__global__ void __launch_bounds__(NT, MB) Ss2BlurQueueKernel(DevBatch batch) {
    using T = Tile<TW, TH, NT>;
    extern __shared__ __align__(16) unsigned char smem[];
    float* src = reinterpret_cast<float*>(smem);
    float* hq = reinterpret_cast<float*>(smem + T::kSrcBytes);
    __shared__ uint32_t next;
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(&batch.blur_queue[0], 1u);
        __syncthreads();
        const uint32_t block = next;
        __syncthreads();  // every thread has read `next` before it changes
        if (block >= batch.blur_blocks) break;
        RunStrip<TW, TH, NT, S>(batch, block, src, hq);
    }
    if (threadIdx.x == 0 && atomicAdd(&batch.blur_queue[1], 1u) + 1u == gridDim.x) {
        batch.blur_queue[0] = 0u;
        batch.blur_queue[1] = 0u;
    }
}

// The variants compiled in: {tile width, tile height, threads, persistent
// (1: grid-stride with a second copy buffer, 2: strips from a tile queue),
// CTAs per SM, tiles per CTA (a strip of that many; 1 = one tile)}.
struct BlurVariant {
    int w, h, threads, persistent, per_sm, strip;
};
constexpr BlurVariant kBlurVariants[] = {
    {32, 32, 128, 0, 5, 1}, {32, 28, 128, 0, 5, 1}, {64, 32, 256, 0, 2, 1},
    {64, 20, 256, 0, 3, 1}, {32, 32, 128, 1, 3, 1}, {32, 20, 128, 1, 5, 1},
    {64, 32, 256, 1, 1, 1}, {32, 32, 128, 0, 5, 2}, {32, 32, 128, 0, 5, 4},
    {32, 32, 128, 0, 5, 8}, {32, 28, 128, 0, 5, 4}, {32, 32, 128, 0, 5, 16},
    {32, 32, 128, 2, 5, 8},
};
constexpr int kBlurVariantCount = sizeof(kBlurVariants) / sizeof(kBlurVariants[0]);

struct LaunchCache {
    std::mutex mu;
    uint64_t ready = 0;  // dynamic shared memory limit raised, per device
    int grid[64] = {};   // persistent grid size per device
};

template <class Kernel>
cudaError_t Prepare(Kernel kernel, size_t smem, LaunchCache& cache, int threads, bool persistent,
                    int* grid) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(cache.mu);
    if (!(cache.ready & (1ull << device))) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        // All of the unified L1/shared storage as shared memory: the tiles
        // are staged explicitly and nothing here relies on L1 hits.
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 static_cast<int>(cudaSharedmemCarveoutMaxShared));
        if (e != cudaSuccess) return e;
        if (persistent) {
            int per_sm = 0, sms = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
            if (e != cudaSuccess) return e;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            if (e != cudaSuccess) return e;
            cache.grid[device] = (per_sm > 0 ? per_sm : 1) * sms;
        }
        cache.ready |= 1ull << device;
    }
    if (grid) *grid = cache.grid[device];
    return cudaSuccess;
}

// Each launcher prepares its kernel (which also loads it) and, when
// `launch`, launches it.
template <int TW, int TH, int NT, int MB, bool kHalf>
cudaError_t LaunchTilesAs(const DevBatch& b, cudaStream_t stream, bool launch) {
    using T = Tile<TW, TH, NT>;
    static LaunchCache cache;
    constexpr size_t smem = T::kSrcBytes + T::kHqBytes;
    const cudaError_t e =
        Prepare(Ss2BlurKernel<TW, TH, NT, MB, kHalf>, smem, cache, NT, false, nullptr);
    if (e != cudaSuccess || !launch) return e;
    Ss2BlurKernel<TW, TH, NT, MB, kHalf><<<b.blur_blocks, NT, smem, stream>>>(b);
    return cudaGetLastError();
}
template <int TW, int TH, int NT, int MB>
cudaError_t LaunchTiles(const DevBatch& b, cudaStream_t stream, bool launch) {
    return b.half ? LaunchTilesAs<TW, TH, NT, MB, true>(b, stream, launch)
                  : LaunchTilesAs<TW, TH, NT, MB, false>(b, stream, launch);
}

template <int TW, int TH, int NT, int MB>
cudaError_t LaunchPersistent(const DevBatch& b, cudaStream_t stream, bool launch) {
    using T = Tile<TW, TH, NT>;
    static LaunchCache cache;
    constexpr size_t smem = 2 * T::kSrcBytes + T::kHqBytes;
    int grid = 0;
    const cudaError_t e =
        Prepare(Ss2BlurPersistentKernel<TW, TH, NT, MB>, smem, cache, NT, true, &grid);
    if (e != cudaSuccess || !launch) return e;
    const uint32_t blocks = b.blur_blocks < static_cast<uint32_t>(grid) ? b.blur_blocks
                                                                        : static_cast<uint32_t>(grid);
    Ss2BlurPersistentKernel<TW, TH, NT, MB><<<blocks, NT, smem, stream>>>(b);
    return cudaGetLastError();
}

template <int TW, int TH, int NT, int MB, int S>
cudaError_t LaunchQueue(const DevBatch& b, cudaStream_t stream, bool launch) {
    using T = Tile<TW, TH, NT>;
    static LaunchCache cache;
    constexpr size_t smem = T::kSrcBytes + T::kHqBytes;
    int grid = 0;
    const cudaError_t e =
        Prepare(Ss2BlurQueueKernel<TW, TH, NT, MB, S>, smem, cache, NT, true, &grid);
    if (e != cudaSuccess || !launch) return e;
    const uint32_t blocks = b.blur_blocks < static_cast<uint32_t>(grid) ? b.blur_blocks
                                                                        : static_cast<uint32_t>(grid);
    Ss2BlurQueueKernel<TW, TH, NT, MB, S><<<blocks, NT, smem, stream>>>(b);
    return cudaGetLastError();
}

template <int TW, int TH, int NT, int MB, int S>
cudaError_t LaunchStrips(const DevBatch& b, cudaStream_t stream, bool launch) {
    using T = Tile<TW, TH, NT>;
    static LaunchCache cache;
    constexpr size_t smem = T::kSrcBytes + T::kHqBytes;
    const cudaError_t e =
        Prepare(Ss2BlurStripKernel<TW, TH, NT, MB, S>, smem, cache, NT, false, nullptr);
    if (e != cudaSuccess || !launch) return e;
    Ss2BlurStripKernel<TW, TH, NT, MB, S><<<b.blur_blocks, NT, smem, stream>>>(b);
    return cudaGetLastError();
}

cudaError_t Dispatch(const DevBatch& b, int variant, cudaStream_t stream, bool launch) {
    switch (variant) {
        case 0: return LaunchTiles<32, 32, 128, 5>(b, stream, launch);
        case 1: return LaunchTiles<32, 28, 128, 5>(b, stream, launch);
        case 2: return LaunchTiles<64, 32, 256, 2>(b, stream, launch);
        case 3: return LaunchTiles<64, 20, 256, 3>(b, stream, launch);
        case 4: return LaunchPersistent<32, 32, 128, 3>(b, stream, launch);
        case 5: return LaunchPersistent<32, 20, 128, 5>(b, stream, launch);
        case 6: return LaunchPersistent<64, 32, 256, 1>(b, stream, launch);
        case 7: return LaunchStrips<32, 32, 128, 5, 2>(b, stream, launch);
        case 8: return LaunchStrips<32, 32, 128, 5, 4>(b, stream, launch);
        case 9: return LaunchStrips<32, 32, 128, 5, 8>(b, stream, launch);
        case 10: return LaunchStrips<32, 28, 128, 5, 4>(b, stream, launch);
        case 11: return LaunchStrips<32, 32, 128, 5, 16>(b, stream, launch);
        case 12: return LaunchQueue<32, 32, 128, 5, 8>(b, stream, launch);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

namespace {
// Quotient values the division check tries with every divisor: spread over
// (-1, 1] and beyond, where the maps' quotients lie (the SSIM' map divides
// its numerator by a denominator at least as large; the edge map's relative
// difference is at least -1).
__constant__ float c_check_quotients[16] = {
    0.0f,       1.0e-7f,   3.3e-5f,   0.00173f, 0.0137f,  0.1f,      0.25f,     0.3333f,
    0.5f,       0.7731f,   0.9999f,   1.0f,     1.7321f,  -0.2718f,  -0.6667f,  -0.99999f};

// For every divisor whose bit pattern is first + i (i < count) and every
// quotient value t of the table: the dividend a = b t rounded, then Div2's
// quotient against ss2dm::divf's (the two lanes hold two divisors); counts
// the differing divisions and keeps the smallest divisor pattern involved.
__global__ void CheckDivisionKernel(uint32_t first, uint32_t count,
                                   unsigned long long* mismatches, uint32_t* first_bad) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t pairs = count / 2 + count % 2;
    unsigned long long bad = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += stride) {
        const uint32_t b0 = first + 2 * i;
        const bool two = 2 * i + 1 < count;
        const uint32_t b1 = two ? b0 + 1 : b0;
        const float2 b = make_float2(__uint_as_float(b0), __uint_as_float(b1));
        for (int k = 0; k < 16; ++k) {
            const float t = c_check_quotients[k];
            const float2 a = make_float2(__fmul_rn(b.x, t), __fmul_rn(b.y, t));
            const float2 q = Div2(a, b);
            const bool d0 = __float_as_uint(q.x) != __float_as_uint(ss2dm::divf(a.x, b.x));
            const bool d1 =
                two && __float_as_uint(q.y) != __float_as_uint(ss2dm::divf(a.y, b.y));
            bad += static_cast<unsigned long long>(d0) + static_cast<unsigned long long>(d1);
            if (d0 || d1) atomicMin(first_bad, d0 ? b0 : b1);
        }
    }
    if (bad) atomicAdd(mismatches, bad);
}
}  // namespace

cudaError_t CheckDivision(uint32_t first_bits, uint32_t last_bits, uint64_t* mismatches,
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
        CheckDivisionKernel<<<148 * 8, 256>>>(first_bits, last_bits - first_bits + 1, d_count,
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

cudaError_t SetConstants(const double* weights108) {
    return cudaMemcpyToSymbol(c_weights, weights108, sizeof(double) * 108);
}

cudaError_t LaunchBlur(const DevBatch& b, int variant, cudaStream_t stream) {
    if (b.blur_blocks == 0) return cudaSuccess;
    // Half planes run the one-tile-per-CTA kernel of the same tile shape.
    if (b.half) variant = HalfPlaneVariant(variant);
    if (variant < 0) return cudaErrorInvalidValue;
    return Dispatch(b, variant, stream, true);
}

cudaError_t PreloadBlur() {
    for (int v = 0; v < kBlurVariantCount; ++v)
        for (int half = 0; half < 2; ++half) {
            DevBatch b{};
            b.half = static_cast<uint32_t>(half);
            const int run = half ? HalfPlaneVariant(v) : v;
            if (run < 0) continue;
            const cudaError_t e = Dispatch(b, run, nullptr, false);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

int HalfPlaneVariant(int variant) {
    if (variant < 0 || variant >= kBlurVariantCount) return -1;
    const auto one_tile = [](const BlurVariant& v) { return !v.persistent && v.strip == 1; };
    if (one_tile(kBlurVariants[variant])) return variant;
    for (int i = 0; i < kBlurVariantCount; ++i)
        if (one_tile(kBlurVariants[i]) && kBlurVariants[i].w == kBlurVariants[variant].w &&
            kBlurVariants[i].h == kBlurVariants[variant].h)
            return i;
    return -1;
}

int BlurTileCount() { return kBlurVariantCount; }
int BlurTileThreads(int index) { return kBlurVariants[index].threads; }
int BlurTileStrip(int index) { return kBlurVariants[index].strip; }
bool BlurTilePersistent(int index) { return kBlurVariants[index].persistent != 0; }
namespace {

// Estimated duration, in tile times, of one launch of strips of S tiles over
// segments with these tile grids (columns, rows) on `slots` CTA slots. A CTA
// costs its tiles plus kStripCost (its first tile's extra rows, the strip's
// reduction and epilogue), fitted to measured one-pair blur times (720p,
// 1080p, 1440p and 4K, strips of 1 to 16). The device hands CTAs in launch
// order to the slot that frees first; up to kSimulatedWaves waves that is
// simulated, beyond it the estimate is the work per slot plus the last
// wave's idle share of an average CTA.
constexpr double kStripCost = 0.7;
constexpr uint64_t kSimulatedWaves = 4;

double StripLaunchCost(const std::vector<std::pair<uint32_t, uint32_t>>& grids, uint32_t S,
                       uint64_t slots) {
    uint64_t ctas = 0, tiles = 0;
    for (const auto& g : grids) {
        ctas += static_cast<uint64_t>(g.first) * ((g.second + S - 1) / S);
        tiles += static_cast<uint64_t>(g.first) * g.second;
    }
    if (ctas == 0) return 0.0;
    const double work = static_cast<double>(tiles) + kStripCost * static_cast<double>(ctas);
    if (ctas > kSimulatedWaves * slots) {
        const double waves = static_cast<double>(ctas) / static_cast<double>(slots);
        return work / static_cast<double>(slots) +
               (std::ceil(waves) - waves) * work / static_cast<double>(ctas);
    }
    // Launch order: segment by segment, strip rows of all columns in turn.
    std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
    for (uint64_t k = 0; k < std::min<uint64_t>(slots, ctas); ++k) free_at.push(0.0);
    double end = 0.0;
    for (const auto& g : grids)
        for (uint32_t y0 = 0; y0 < g.second; y0 += S) {
            const double d = static_cast<double>(std::min(S, g.second - y0)) + kStripCost;
            for (uint32_t x = 0; x < g.first; ++x) {
                const double t = free_at.top() + d;
                free_at.pop();
                free_at.push(t);
                end = std::max(end, t);
            }
        }
    return end;
}

}  // namespace

int AutoBlurVariant(const std::vector<std::pair<uint32_t, uint32_t>>& grids, int sms) {
    // The strip length of the default tile with the least estimated time
    // (StripLaunchCost; on ties the longer strip, with fewer partials).
    // Large batches take the longest strip, 16; one pair 720p 1 to 4 (equal
    // times), 1080p 2, 1440p 4 and 4K 4 (4K: 122.9 -> 118.8 us against the
    // earlier rule, the longest strip leaving every CTA slot 2 CTAs, which
    // took 8). Memoised per set of grids (sorted, so a batch of the same
    // sizes in another order is the same entry): a batch of the same sizes,
    // or a pipeline, pays for the estimate once.
    const BlurVariant& base = kBlurVariants[kDefaultBlurVariant];
    const uint64_t slots = static_cast<uint64_t>(sms > 0 ? sms : 1) * base.per_sm;
    std::vector<std::pair<uint32_t, uint32_t>> sorted(grids);
    std::sort(sorted.begin(), sorted.end());
    uint64_t key = 1469598103934665603ull ^ static_cast<uint64_t>(sms);
    for (const auto& g : sorted) {
        key = (key ^ g.first) * 1099511628211ull;
        key = (key ^ g.second) * 1099511628211ull;
    }
    static std::mutex mu;
    static std::unordered_map<uint64_t, int> memo;
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto it = memo.find(key);
        if (it != memo.end()) return it->second;
    }
    int best = kDefaultBlurVariant;
    double best_cost = StripLaunchCost(sorted, 1, slots);
    int best_strip = 1;
    for (int i = 0; i < kBlurVariantCount; ++i) {
        const BlurVariant& v = kBlurVariants[i];
        if (v.persistent || v.w != base.w || v.h != base.h || v.threads != base.threads ||
            v.strip <= 1)
            continue;
        const double c = StripLaunchCost(sorted, static_cast<uint32_t>(v.strip), slots);
        if (c < best_cost * (1.0 - 1e-9) || (c <= best_cost * (1.0 + 1e-9) && v.strip > best_strip)) {
            best = i;
            best_cost = c;
            best_strip = v.strip;
        }
    }
    std::lock_guard<std::mutex> lock(mu);
    if (memo.size() >= 4096) memo.clear();
    memo.emplace(key, best);
    return best;
}

uint32_t BlurBlocks(int index, uint32_t tiles_x, uint32_t tiles_y) {
    const uint32_t s = static_cast<uint32_t>(kBlurVariants[index].strip);
    return tiles_x * ((tiles_y + s - 1) / s);
}
void BlurTileShape(int index, int* w, int* h) {
    *w = kBlurVariants[index].w;
    *h = kBlurVariants[index].h;
}

}  // namespace vqm_b200
