// Blur and finalize stages for sm_100a: the five 13-tap blurs, the maps and
// compensated norm partials of every (pair, level, kept channel) tile, then
// the FP64 reduction to norms and score. See ss2_device.cuh for the batch
// layout.
//
// Rounding contract: the library is compiled with -fmad=false; every fused
// multiply-add is an explicit __fmaf_rn placed where VQM's shaders accumulate
// (src/metrics/ssimulacra2/shaders/scale.comp:149-333), so the blurred
// quantities and map values are bit-identical to the CPU oracle's FP32 path
// for bit-identical pyramid planes.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "ss2_device.cuh"
#include "ss2_kernels.h"

namespace vqm_b200 {

__constant__ float c_taps[kTaps];
// score.cc:38-87, flat rows channel * scales + scale.
__constant__ double c_weights[18][6];

// ---------------------------------------------------------------------------
// Work lookup: the last prefix entry <= index.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t FindSlot(const uint32_t* __restrict__ start,
                                             uint32_t count, uint32_t index) {
    uint32_t lo = 0, hi = count;  // start[lo] <= index < start[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&start[mid]) <= index) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Blur: one CTA per TW x TH output tile of one (pair, level, kept channel).
// Both images' zero-padded source tiles go to shared memory; the horizontal
// pass writes all five quantities' row blurs (four output columns per task,
// 16 shared reads for 52 taps); the vertical pass produces four rows per
// thread (16 reads for 52 taps), then the maps and six sums.
// ---------------------------------------------------------------------------

template <int TW, int TH>
struct BlurTile {
    static constexpr int SW = TW + 2 * kRadius;
    static constexpr int SH = TH + 2 * kRadius;
    static constexpr int SP = (SW + 3) / 4 * 4;  // row pitch, float4 aligned
    static constexpr int kThreads = TW * TH / 4;
    static constexpr int kQuads = TW / 4;
    static_assert(TW % 4 == 0, "four-column horizontal windows");
    static_assert(TH % 4 == 0, "four rows per thread");
};

// Compensated (two-sum) addition of (s2, c2) into (s, c).
__device__ __forceinline__ void TwoSumAdd(float& s, float& c, float s2, float c2) {
    const float t = __fadd_rn(s, s2);
    const float bp = __fsub_rn(t, s);
    const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(s2, bp));
    s = t;
    c = __fadd_rn(__fadd_rn(c, c2), e);
}

template <int TW, int TH>
__global__ void __launch_bounds__(BlurTile<TW, TH>::kThreads)
    Ss2BlurKernel(DevBatch batch) {
    using T = BlurTile<TW, TH>;
    constexpr int SW = T::SW, SH = T::SH, SP = T::SP, NT = T::kThreads;
    __shared__ __align__(16) float src[2][SH][SP];
    __shared__ __align__(16) float hq[5][SH][TW];
    __shared__ float red[NT / 32][12];

    const uint32_t tid = threadIdx.x;
    const uint32_t blk = blockIdx.x;
    const uint32_t si = FindSlot(batch.blur_start, batch.segments, blk);
    const DevSegment seg = batch.seg[si];
    const uint32_t tile = blk - __ldg(&batch.blur_start[si]);
    const DevPair& P = batch.pair[seg.pair];
    const uint32_t level = seg.level, channel = seg.channel;
    const uint32_t w = P.w[level], h = P.h[level], pitch = P.pitch[level];
    const float* __restrict__ pa = P.pyramid + P.plane_off[level][channel];
    const float* __restrict__ pb = pa + P.image_stride;
    const int x0 = static_cast<int>((tile % seg.tiles_x) * TW);
    const int y0 = static_cast<int>((tile / seg.tiles_x) * TH);

    // Zero-padded source tiles (scale.comp:107-124).
    for (int i = tid; i < SH * SW; i += NT) {
        const int r = i / SW, c = i % SW;
        const int gx = x0 - kRadius + c, gy = y0 - kRadius + r;
        float va = 0.0f, vb = 0.0f;
        if (gx >= 0 && gx < static_cast<int>(w) && gy >= 0 && gy < static_cast<int>(h)) {
            const size_t at = static_cast<size_t>(gy) * pitch + gx;
            va = __ldg(pa + at);
            vb = __ldg(pb + at);
        }
        src[0][r][c] = va;
        src[1][r][c] = vb;
    }
    __syncthreads();

    // Horizontal pass (scale.comp:149-207), all five quantities.
    for (int task = tid; task < SH * T::kQuads; task += NT) {
        const int r = task / T::kQuads;
        const int c0 = (task % T::kQuads) * 4;
        float a[16], b[16];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float4 va = *reinterpret_cast<const float4*>(&src[0][r][c0 + 4 * k]);
            const float4 vb = *reinterpret_cast<const float4*>(&src[1][r][c0 + 4 * k]);
            a[4 * k + 0] = va.x; a[4 * k + 1] = va.y; a[4 * k + 2] = va.z; a[4 * k + 3] = va.w;
            b[4 * k + 0] = vb.x; b[4 * k + 1] = vb.y; b[4 * k + 2] = vb.z; b[4 * k + 3] = vb.w;
        }
        float acc[5][4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            acc[0][j] = __fmul_rn(c_taps[0], a[j]);
            acc[1][j] = __fmul_rn(c_taps[0], b[j]);
            acc[2][j] = __fmul_rn(c_taps[0], __fmul_rn(a[j], a[j]));
            acc[3][j] = __fmul_rn(c_taps[0], __fmul_rn(b[j], b[j]));
            acc[4][j] = __fmul_rn(c_taps[0], __fmul_rn(a[j], b[j]));
        }
#pragma unroll
        for (int t = 1; t < kTaps; ++t) {
            const float wt = c_taps[t];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float av = a[j + t], bv = b[j + t];
                acc[0][j] = __fmaf_rn(wt, av, acc[0][j]);
                acc[1][j] = __fmaf_rn(wt, bv, acc[1][j]);
                acc[2][j] = __fmaf_rn(wt, __fmul_rn(av, av), acc[2][j]);
                acc[3][j] = __fmaf_rn(wt, __fmul_rn(bv, bv), acc[3][j]);
                acc[4][j] = __fmaf_rn(wt, __fmul_rn(av, bv), acc[4][j]);
            }
        }
#pragma unroll
        for (int q = 0; q < 5; ++q)
            *reinterpret_cast<float4*>(&hq[q][r][c0]) =
                make_float4(acc[q][0], acc[q][1], acc[q][2], acc[q][3]);
    }
    __syncthreads();

    // Vertical pass (scale.comp:211-301): four rows of one column.
    const int ox = tid % TW;
    const int row = (tid / TW) * 4;
    float bq[5][4];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        float m[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) m[k] = hq[q][row + k][ox];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float s = __fmul_rn(c_taps[0], m[j]);
#pragma unroll
            for (int t = 1; t < kTaps; ++t) s = __fmaf_rn(c_taps[t], m[j + t], s);
            bq[q][j] = s;
        }
    }

    // Maps (scale.comp:305-333) and this thread's six sums.
    float sum[6] = {0, 0, 0, 0, 0, 0};
    const int out_x = x0 + ox;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int out_y = y0 + row + j;
        if (out_x >= static_cast<int>(w) || out_y >= static_cast<int>(h)) continue;
        const float mu1 = bq[0][j], mu2 = bq[1][j];
        const float s11 = bq[2][j], s22 = bq[3][j], s12 = bq[4][j];
        const float dm = __fsub_rn(mu1, mu2);
        const float num_m = __fmaf_rn(-dm, dm, 1.0f);
        const float num_s = __fmaf_rn(2.0f, __fmaf_rn(-mu1, mu2, s12), 0.0009f);
        const float denom =
            __fadd_rn(__fadd_rn(__fmaf_rn(-mu1, mu1, s11), __fmaf_rn(-mu2, mu2, s22)), 0.0009f);
        const float d = fmaxf(__fdiv_rn(__fmaf_rn(-num_m, num_s, denom), denom), 0.0f);
        const float dd = __fmul_rn(d, d);
        sum[0] = __fadd_rn(sum[0], d);
        sum[1] = __fadd_rn(sum[1], __fmul_rn(dd, dd));
        const float img1 = src[0][row + j + kRadius][ox + kRadius];
        const float img2 = src[1][row + j + kRadius][ox + kRadius];
        const float dist = __fadd_rn(1.0f, fabsf(__fsub_rn(img2, mu2)));
        const float orig = __fadd_rn(1.0f, fabsf(__fsub_rn(img1, mu1)));
        const float d1 = __fdiv_rn(__fsub_rn(dist, orig), orig);
        const float ring = fmaxf(d1, 0.0f);
        const float blur = fmaxf(-d1, 0.0f);
        const float r2 = __fmul_rn(ring, ring), b2 = __fmul_rn(blur, blur);
        sum[2] = __fadd_rn(sum[2], ring);
        sum[3] = __fadd_rn(sum[3], __fmul_rn(r2, r2));
        sum[4] = __fadd_rn(sum[4], blur);
        sum[5] = __fadd_rn(sum[5], __fmul_rn(b2, b2));
    }

    // Compensated block reduction: warp tree, then across warps.
    float comp[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float s2 = __shfl_xor_sync(0xffffffffu, sum[k], off);
            const float c2 = __shfl_xor_sync(0xffffffffu, comp[k], off);
            TwoSumAdd(sum[k], comp[k], s2, c2);
        }
    const int warp = tid / 32, lane = tid % 32;
    if (lane == 0)
        for (int k = 0; k < 6; ++k) {
            red[warp][k] = sum[k];
            red[warp][6 + k] = comp[k];
        }
    __syncthreads();
    if (tid < 6) {
        float s = red[0][tid], c = red[0][6 + tid];
        for (int wi = 1; wi < NT / 32; ++wi) TwoSumAdd(s, c, red[wi][tid], red[wi][6 + tid]);
        batch.partials[(static_cast<size_t>(seg.partial_first) + tile) * 6 + tid] =
            static_cast<double>(s) + static_cast<double>(c);
    }
}

// ---------------------------------------------------------------------------
// Blur with packed FP32 (Blackwell FFMA2: two fused multiply-adds per
// instruction). Same arithmetic per output as above -- every output is still
// w0*s0 followed by fused ascending taps -- but two outputs share each
// instruction:
//   * the source tile is stored as row pairs, element (r, c) at
//     src[image][r / 2][c].{x: r even, y: r odd}, so one 64-bit shared load
//     gives the same column of two rows and the horizontal pass accumulates
//     rows (2p, 2p+1) together, four output columns per task;
//   * the horizontal results go to row-major planes, so the vertical pass
//     reads columns (c, c+1) as one 64-bit load and accumulates that column
//     pair over four output rows per task;
//   * the maps run on the column pair, packed wherever the arithmetic is a
//     multiply, add or fused multiply-add.
// ---------------------------------------------------------------------------

template <int TW, int TH, int NT>
struct Blur2Tile {
    static constexpr int SW = TW + 2 * kRadius;  // source columns
    static constexpr int SH = TH + 2 * kRadius;  // source rows
    static constexpr int RP = SH / 2;            // source row pairs
    static constexpr int KH = 4;                 // output columns per horizontal task
    static constexpr int HT = RP * (TW / KH);    // horizontal tasks
    static constexpr int RV = 4;                 // output rows per vertical task
    static constexpr int VT = (TW / 2) * (TH / RV);
    static constexpr int kWarps = NT / 32;
    // Dynamic shared memory: the row-pair source tiles of both images, then
    // the five horizontal-pass planes.
    static constexpr size_t kSrcBytes = sizeof(float2) * 2 * RP * SW;
    static constexpr size_t kSmemBytes = kSrcBytes + sizeof(float) * 5 * SH * TW;
    static_assert(TW % KH == 0 && TH % RV == 0 && SH % 2 == 0, "tile shape");
    static_assert(NT % 32 == 0, "whole warps");
    static_assert(kSrcBytes % 16 == 0, "plane alignment");
};

__device__ __forceinline__ float2 Pack(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 Neg(float2 v) { return make_float2(-v.x, -v.y); }

template <int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) Ss2Blur2Kernel(DevBatch batch) {
    using T = Blur2Tile<TW, TH, NT>;
    constexpr int SW = T::SW, SH = T::SH, RP = T::RP;
    extern __shared__ __align__(16) unsigned char smem[];
    auto src = reinterpret_cast<float2 (*)[RP][SW]>(smem);
    auto hq = reinterpret_cast<float (*)[SH][TW]>(smem + T::kSrcBytes);
    __shared__ float red[T::kWarps][12];

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const uint32_t blk = blockIdx.x;
    const uint32_t si = FindSlot(batch.blur_start, batch.segments, blk);
    const DevSegment seg = batch.seg[si];
    const uint32_t tile = blk - __ldg(&batch.blur_start[si]);
    const DevPair& P = batch.pair[seg.pair];
    const int w = static_cast<int>(P.w[seg.level]), h = static_cast<int>(P.h[seg.level]);
    const size_t pitch = P.pitch[seg.level];
    const float* __restrict__ pa = P.pyramid + P.plane_off[seg.level][seg.channel];
    const float* __restrict__ pb = pa + P.image_stride;
    const int x0 = static_cast<int>((tile % seg.tiles_x) * TW);
    const int y0 = static_cast<int>((tile / seg.tiles_x) * TH);

    // Zero-padded source tiles (scale.comp:107-124), as row pairs.
    for (int rp = warp; rp < RP; rp += T::kWarps) {
        const int gy0 = y0 - kRadius + 2 * rp, gy1 = gy0 + 1;
        const bool in0 = gy0 >= 0 && gy0 < h, in1 = gy1 >= 0 && gy1 < h;
        for (int c = lane; c < SW; c += 32) {
            const int gx = x0 - kRadius + c;
            const bool inx = gx >= 0 && gx < w;
            float a0 = 0.0f, a1 = 0.0f, b0 = 0.0f, b1 = 0.0f;
            if (inx && in0) {
                a0 = __ldg(pa + static_cast<size_t>(gy0) * pitch + gx);
                b0 = __ldg(pb + static_cast<size_t>(gy0) * pitch + gx);
            }
            if (inx && in1) {
                a1 = __ldg(pa + static_cast<size_t>(gy1) * pitch + gx);
                b1 = __ldg(pb + static_cast<size_t>(gy1) * pitch + gx);
            }
            src[0][rp][c] = make_float2(a0, a1);
            src[1][rp][c] = make_float2(b0, b1);
        }
    }
    __syncthreads();

    // Horizontal pass (scale.comp:149-207): row pair rp, columns c0..c0+3.
    for (int task = tid; task < T::HT; task += NT) {
        const int rp = task / (TW / T::KH);
        const int c0 = (task % (TW / T::KH)) * T::KH;
        float2 A[T::KH + 12], B[T::KH + 12];
#pragma unroll
        for (int j = 0; j < T::KH + 12; j += 2) {
            const float4 va = *reinterpret_cast<const float4*>(&src[0][rp][c0 + j]);
            const float4 vb = *reinterpret_cast<const float4*>(&src[1][rp][c0 + j]);
            A[j] = make_float2(va.x, va.y);
            A[j + 1] = make_float2(va.z, va.w);
            B[j] = make_float2(vb.x, vb.y);
            B[j + 1] = make_float2(vb.z, vb.w);
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            float2 S[T::KH + 12];
#pragma unroll
            for (int j = 0; j < T::KH + 12; ++j)
                S[j] = q == 0 ? A[j]
                     : q == 1 ? B[j]
                     : q == 2 ? __fmul2_rn(A[j], A[j])
                     : q == 3 ? __fmul2_rn(B[j], B[j])
                              : __fmul2_rn(A[j], B[j]);
            float2 acc[T::KH];
#pragma unroll
            for (int k = 0; k < T::KH; ++k) acc[k] = __fmul2_rn(Pack(c_taps[0]), S[k]);
#pragma unroll
            for (int t = 1; t < kTaps; ++t) {
                const float2 wt = Pack(c_taps[t]);
#pragma unroll
                for (int k = 0; k < T::KH; ++k) acc[k] = __ffma2_rn(wt, S[k + t], acc[k]);
            }
            *reinterpret_cast<float4*>(&hq[q][2 * rp][c0]) =
                make_float4(acc[0].x, acc[1].x, acc[2].x, acc[3].x);
            *reinterpret_cast<float4*>(&hq[q][2 * rp + 1][c0]) =
                make_float4(acc[0].y, acc[1].y, acc[2].y, acc[3].y);
        }
    }
    __syncthreads();

    float2 sum[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sum[k] = make_float2(0.0f, 0.0f);

    // Vertical pass (scale.comp:211-301) on column pair (c, c+1), rows
    // r0..r0+3, then the maps (scale.comp:305-333) of those eight pixels.
    for (int task = tid; task < T::VT; task += NT) {
        const int c = (task % (TW / 2)) * 2;
        const int r0 = (task / (TW / 2)) * T::RV;
        float2 V[5][T::RV];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            float2 M[T::RV + 12];
#pragma unroll
            for (int i = 0; i < T::RV + 12; ++i)
                M[i] = *reinterpret_cast<const float2*>(&hq[q][r0 + i][c]);
#pragma unroll
            for (int j = 0; j < T::RV; ++j) {
                float2 acc = __fmul2_rn(Pack(c_taps[0]), M[j]);
#pragma unroll
                for (int t = 1; t < kTaps; ++t) acc = __ffma2_rn(Pack(c_taps[t]), M[j + t], acc);
                V[q][j] = acc;
            }
        }
        const int out_x = x0 + c;
#pragma unroll
        for (int j = 0; j < T::RV; ++j) {
            const int out_y = y0 + r0 + j;
            if (out_y >= h || out_x >= w) continue;
            const bool second = out_x + 1 < w;
            const float2 mu1 = V[0][j], mu2 = V[1][j];
            const float2 dm = __fadd2_rn(mu1, Neg(mu2));
            const float2 num_m = __ffma2_rn(Neg(dm), dm, Pack(1.0f));
            const float2 num_s =
                __ffma2_rn(Pack(2.0f), __ffma2_rn(Neg(mu1), mu2, V[4][j]), Pack(0.0009f));
            const float2 denom = __fadd2_rn(
                __fadd2_rn(__ffma2_rn(Neg(mu1), mu1, V[2][j]), __ffma2_rn(Neg(mu2), mu2, V[3][j])),
                Pack(0.0009f));
            const float2 numer = __ffma2_rn(Neg(num_m), num_s, denom);
            float2 d;
            d.x = fmaxf(__fdiv_rn(numer.x, denom.x), 0.0f);
            d.y = second ? fmaxf(__fdiv_rn(numer.y, denom.y), 0.0f) : 0.0f;
            const float2 dd = __fmul2_rn(d, d);
            // The raw XYB value is the centre of the source tile.
            const int rr = r0 + j + kRadius;
            const float2 s1a = src[0][rr >> 1][c + kRadius], s1b = src[0][rr >> 1][c + kRadius + 1];
            const float2 s2a = src[1][rr >> 1][c + kRadius], s2b = src[1][rr >> 1][c + kRadius + 1];
            const float2 img1 = (rr & 1) ? make_float2(s1a.y, s1b.y) : make_float2(s1a.x, s1b.x);
            const float2 img2 = (rr & 1) ? make_float2(s2a.y, s2b.y) : make_float2(s2a.x, s2b.x);
            float2 e2 = __fadd2_rn(img2, Neg(mu2));
            float2 e1 = __fadd2_rn(img1, Neg(mu1));
            e2 = make_float2(fabsf(e2.x), fabsf(e2.y));
            e1 = make_float2(fabsf(e1.x), fabsf(e1.y));
            const float2 dist = __fadd2_rn(Pack(1.0f), e2);
            const float2 orig = __fadd2_rn(Pack(1.0f), e1);
            const float2 diff = __fadd2_rn(dist, Neg(orig));
            float2 d1;
            d1.x = __fdiv_rn(diff.x, orig.x);
            d1.y = second ? __fdiv_rn(diff.y, orig.y) : 0.0f;
            const float2 ring = make_float2(fmaxf(d1.x, 0.0f), fmaxf(d1.y, 0.0f));
            const float2 blur = make_float2(fmaxf(-d1.x, 0.0f), fmaxf(-d1.y, 0.0f));
            const float2 r2 = __fmul2_rn(ring, ring), b2 = __fmul2_rn(blur, blur);
            sum[0] = __fadd2_rn(sum[0], d);
            sum[1] = __fadd2_rn(sum[1], __fmul2_rn(dd, dd));
            sum[2] = __fadd2_rn(sum[2], ring);
            sum[3] = __fadd2_rn(sum[3], __fmul2_rn(r2, r2));
            sum[4] = __fadd2_rn(sum[4], blur);
            sum[5] = __fadd2_rn(sum[5], __fmul2_rn(b2, b2));
        }
    }

    // Compensated block reduction: the column pair's two sums, warp tree,
    // then across warps.
    float s[6], comp[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        s[k] = sum[k].x;
        comp[k] = 0.0f;
        TwoSumAdd(s[k], comp[k], sum[k].y, 0.0f);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float s2 = __shfl_xor_sync(0xffffffffu, s[k], off);
            const float c2 = __shfl_xor_sync(0xffffffffu, comp[k], off);
            TwoSumAdd(s[k], comp[k], s2, c2);
        }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            red[warp][k] = s[k];
            red[warp][6 + k] = comp[k];
        }
    __syncthreads();
    if (tid < 6) {
        float a = red[0][tid], cc = red[0][6 + tid];
        for (int wi = 1; wi < T::kWarps; ++wi) TwoSumAdd(a, cc, red[wi][tid], red[wi][6 + tid]);
        batch.partials[(static_cast<size_t>(seg.partial_first) + tile) * 6 + tid] =
            static_cast<double>(a) + static_cast<double>(cc);
    }
}

// ---------------------------------------------------------------------------
// Finalize: one CTA per segment sums its tile partials in FP64 (fixed order,
// so results repeat bit for bit); the last segment of a pair to finish writes
// the pair's 108 norms (vulkan.cc:545-583) and score (score.cc:118-163).
// ---------------------------------------------------------------------------

constexpr int kFinThreads = 256;

__device__ double ScoreFromNorms(const double* norms, int scales) {
    double error = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int s = 0; s < scales; ++s) {
            const double* wt = c_weights[c * scales + s];
            const double* ssim = norms + s * 18;
            const double* edge = norms + s * 18 + 6;
            error += wt[0] * fabs(ssim[c * 2 + 0]);
            error += wt[1] * fabs(edge[c * 4 + 0]);
            error += wt[2] * fabs(edge[c * 4 + 2]);
            error += wt[3] * fabs(ssim[c * 2 + 1]);
            error += wt[4] * fabs(edge[c * 4 + 1]);
            error += wt[5] * fabs(edge[c * 4 + 3]);
        }
    if (!isfinite(error)) return nan("");
    const double scaled = error * 0.9562382616834844;
    const double mapped = 2.326765642916932 * scaled -
                          0.020884521182843837 * scaled * scaled +
                          6.248496625763138e-05 * scaled * scaled * scaled;
    if (!isfinite(mapped)) return nan("");
    if (mapped > 0.0) return 100.0 - 10.0 * pow(mapped, 0.6276336467831387);
    return 100.0;
}

__global__ void __launch_bounds__(kFinThreads) Ss2FinalizeKernel(DevBatch batch) {
    __shared__ double part[kFinThreads / 32][6];
    __shared__ bool is_last;
    const uint32_t si = blockIdx.x;
    const DevSegment seg = batch.seg[si];
    const uint32_t tid = threadIdx.x;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t t = tid; t < seg.tiles; t += kFinThreads) {
        const double* p = batch.partials + (static_cast<size_t>(seg.partial_first) + t) * 6;
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] += __ldcg(p + k);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
    if (tid % 32 == 0)
        for (int k = 0; k < 6; ++k) part[tid / 32][k] = acc[k];
    __syncthreads();
    if (tid < 6) {
        double s = 0.0;
        for (int wi = 0; wi < kFinThreads / 32; ++wi) s += part[wi][tid];
        batch.seg_sums[static_cast<size_t>(si) * 6 + tid] = s;
    }
    __syncthreads();
    const DevPair& P = batch.pair[seg.pair];
    if (tid == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&batch.pair_done[seg.pair], 1u);
        is_last = prev + 1 == P.seg_count;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    if (tid == 0) {
        double norms[108];
        for (int i = 0; i < 108; ++i) norms[i] = 0.0;
        for (uint32_t k = 0; k < P.seg_count; ++k) {
            const uint32_t sk = P.seg_first + k;
            const DevSegment g = batch.seg[sk];
            const double inv = 1.0 / (static_cast<double>(P.w[g.level]) *
                                      static_cast<double>(P.h[g.level]));
            double v[6];
            for (int n = 0; n < 6; ++n) v[n] = __ldcg(batch.seg_sums + static_cast<size_t>(sk) * 6 + n);
            double* out = norms + g.level * 18;
            const int c = static_cast<int>(g.channel);
            out[c * 2 + 0] = inv * v[0];
            out[c * 2 + 1] = sqrt(sqrt(inv * v[1]));
            out[6 + c * 4 + 0] = inv * v[2];
            out[6 + c * 4 + 1] = sqrt(sqrt(inv * v[3]));
            out[6 + c * 4 + 2] = inv * v[4];
            out[6 + c * 4 + 3] = sqrt(sqrt(inv * v[5]));
        }
        for (int i = 0; i < 108; ++i) P.result[i] = norms[i];
        P.result[kResultScore] = ScoreFromNorms(norms, static_cast<int>(P.levels));
        P.result[kResultScales] = static_cast<double>(P.levels);
        P.result[kResultStatus] = 0.0;
        batch.pair_done[seg.pair] = 0u;  // ready for the next launch
    }
}

// ---------------------------------------------------------------------------
// Host-side launchers.
// ---------------------------------------------------------------------------

cudaError_t SetConstants(const float* taps13, const double* weights108) {
    cudaError_t e = cudaMemcpyToSymbol(c_taps, taps13, sizeof(float) * kTaps);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_weights, weights108, sizeof(double) * 108);
}

// The blur variants compiled in: {tile width, tile height, threads, packed}.
// Variant 0 is the scalar kernel; the rest use packed FP32.
struct BlurVariant {
    int w, h, threads, packed;
};
constexpr BlurVariant kBlurVariants[] = {
    {32, 32, 256, 0}, {32, 32, 128, 1}, {64, 32, 256, 1}, {32, 52, 128, 1}, {64, 20, 256, 1},
};
constexpr int kBlurVariantCount = sizeof(kBlurVariants) / sizeof(kBlurVariants[0]);

// Launches one packed variant, raising its dynamic shared-memory limit the
// first time on each device.
template <int TW, int TH, int NT>
cudaError_t LaunchPacked(const DevBatch& b, cudaStream_t stream) {
    using T = Blur2Tile<TW, TH, NT>;
    static std::mutex mu;
    static uint64_t ready = 0;  // bit per device ordinal
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (device >= 64) return cudaErrorInvalidDevice;
        if (!(ready & (1ull << device))) {
            e = cudaFuncSetAttribute(Ss2Blur2Kernel<TW, TH, NT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(T::kSmemBytes));
            if (e != cudaSuccess) return e;
            ready |= 1ull << device;
        }
    }
    Ss2Blur2Kernel<TW, TH, NT><<<b.blur_blocks, NT, T::kSmemBytes, stream>>>(b);
    return cudaGetLastError();
}

cudaError_t LaunchBlur(const DevBatch& b, int variant, cudaStream_t stream) {
    if (b.blur_blocks == 0) return cudaSuccess;
    switch (variant) {
        case 0:
            Ss2BlurKernel<32, 32><<<b.blur_blocks, 256, 0, stream>>>(b);
            return cudaGetLastError();
        case 1: return LaunchPacked<32, 32, 128>(b, stream);
        case 2: return LaunchPacked<64, 32, 256>(b, stream);
        case 3: return LaunchPacked<32, 52, 128>(b, stream);
        case 4: return LaunchPacked<64, 20, 256>(b, stream);
    }
    return cudaErrorInvalidValue;
}

int BlurTileCount() { return kBlurVariantCount; }
int BlurTileThreads(int index) { return kBlurVariants[index].threads; }
void BlurTileShape(int index, int* w, int* h) {
    *w = kBlurVariants[index].w;
    *h = kBlurVariants[index].h;
}

cudaError_t LaunchFinalize(const DevBatch& b, cudaStream_t stream) {
    if (b.segments == 0) return cudaSuccess;
    Ss2FinalizeKernel<<<b.segments, kFinThreads, 0, stream>>>(b);
    return cudaGetLastError();
}

}  // namespace vqm_b200
