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

cudaError_t LaunchBlur(const DevBatch& b, int tile_w, int tile_h, cudaStream_t stream) {
    if (b.blur_blocks == 0) return cudaSuccess;
    if (tile_w == 32 && tile_h == 32) {
        Ss2BlurKernel<32, 32><<<b.blur_blocks, BlurTile<32, 32>::kThreads, 0, stream>>>(b);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int BlurTileCount() { return 1; }
void BlurTileShape(int index, int* w, int* h) {
    (void)index;
    *w = 32;
    *h = 32;
}

cudaError_t LaunchFinalize(const DevBatch& b, cudaStream_t stream) {
    if (b.segments == 0) return cudaSuccess;
    Ss2FinalizeKernel<<<b.segments, kFinThreads, 0, stream>>>(b);
    return cudaGetLastError();
}

}  // namespace vqm_b200
