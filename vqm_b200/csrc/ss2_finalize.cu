// Finalize stage for sm_100a: one CTA per (pair, level, kept channel)
// segment sums the segment's blur partials (one per blur CTA: a tile or a
// strip of tiles) in FP64, in a fixed order so
// results repeat bit for bit; the last segment of a pair to finish turns the
// pair's sums into its 108 norms (reference: vulkan.cc:545-583 ReadResult)
// and FP64 score (score.cc:118-163).

#include <cuda_runtime.h>

#include <cstdint>

#include "ss2_device.cuh"
#include "ss2_kernels.h"

namespace vqm_b200 {
namespace {

// score.cc:38-87, flat rows channel * scales + scale.
__constant__ double c_weights[18][6];

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
    for (uint32_t t = tid; t < seg.partials; t += kFinThreads) {
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

}  // namespace

cudaError_t SetScoreWeights(const double* weights108) {
    return cudaMemcpyToSymbol(c_weights, weights108, sizeof(double) * 108);
}

cudaError_t PreloadFinalize() {
    cudaFuncAttributes a;
    return cudaFuncGetAttributes(&a, Ss2FinalizeKernel);
}

cudaError_t LaunchFinalize(const DevBatch& b, cudaStream_t stream) {
    if (b.segments == 0) return cudaSuccess;
    Ss2FinalizeKernel<<<b.segments, kFinThreads, 0, stream>>>(b);
    return cudaGetLastError();
}

}  // namespace vqm_b200
