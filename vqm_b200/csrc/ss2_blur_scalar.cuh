// The scalar blur kernel (one FP32 lane per output): both images'
// zero-padded source tiles in shared memory, a horizontal pass writing all
// five quantities' row blurs (four output columns per task, 16 shared reads
// for 52 taps), a vertical pass producing four rows per thread, then the
// maps and the six sums. Included by ss2_blur.cu, which defines c_taps,
// FindSlot and TwoSumAdd.
#pragma once


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
