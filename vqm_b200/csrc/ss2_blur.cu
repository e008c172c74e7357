// Blur stage for sm_100a: the five 13-tap blurs, the SSIM' and edge maps and
// the compensated norm partials of every (pair, level, kept channel) output
// tile (reference: src/metrics/ssimulacra2/shaders/scale.comp).
//
// Rounding contract: the library is compiled with -fmad=false; every fused
// multiply-add is explicit and placed where VQM's shaders accumulate
// (scale.comp:149-333): each blurred value is w0*s0 followed by fused
// ascending taps, horizontal pass first. So the blurred quantities and map
// values are bit-identical to the CPU checker's FP32 path for bit-identical
// pyramid planes, whichever kernel variant below computes them.
//
// Variants (kBlurVariants): the scalar kernel (ss2_blur_scalar.cuh), packed
// kernels that issue Blackwell's two-lane FP32 instructions (FFMA2) with one
// output tile per CTA, and persistent packed kernels that keep each CTA
// resident and prefetch its next tile with cp.async while computing the
// current one.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "ss2_device.cuh"
#include "ss2_kernels.h"

namespace vqm_b200 {
namespace {

__constant__ float c_taps[kTaps];

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

#include "ss2_blur_scalar.cuh"

// ---------------------------------------------------------------------------
// Packed tiles.
//
//   * The source tile is stored as row pairs: element (r, c) of image i at
//     src[i][r / 2][c].{x: r even, y: r odd}. One 64-bit shared load gives
//     one column of two rows, so the horizontal pass accumulates rows
//     (2p, 2p+1) together, four output columns per task.
//   * The horizontal results go to row-major planes, so the vertical pass
//     reads columns (c, c+1) as one 64-bit load and accumulates that column
//     pair over four output rows per task.
//   * The maps run on the column pair, packed wherever the arithmetic is a
//     multiply, add or fused multiply-add.
// ---------------------------------------------------------------------------

template <int TW, int TH, int NT>
struct PackedTile {
    static constexpr int SW = TW + 2 * kRadius;  // source columns
    static constexpr int SH = TH + 2 * kRadius;  // source rows
    static constexpr int RP = SH / 2;            // source row pairs
    static constexpr int KH = 4;                 // output columns per horizontal task
    static constexpr int HT = RP * (TW / KH);    // horizontal tasks
    static constexpr int RV = 4;                 // output rows per vertical task
    static constexpr int VT = (TW / 2) * (TH / RV);
    static constexpr int kWarps = NT / 32;
    // One source buffer (both images) and the five horizontal-pass planes.
    static constexpr size_t kSrcBytes = sizeof(float2) * 2 * RP * SW;
    static constexpr size_t kHqBytes = sizeof(float) * 5 * SH * TW;
    static_assert(TW % KH == 0 && TH % RV == 0 && SH % 2 == 0, "tile shape");
    static_assert(NT % 32 == 0, "whole warps");
    static_assert(kSrcBytes % 16 == 0, "plane alignment");
};

// Where one output tile's planes, geometry and partial slot are.
struct TileRef {
    const float* pa;
    const float* pb;
    size_t pitch;
    size_t partial;
    int w, h, x0, y0;
};

template <int TW, int TH>
__device__ __forceinline__ TileRef LocateTile(const DevBatch& batch, uint32_t blk) {
    const uint32_t si = FindSlot(batch.blur_start, batch.segments, blk);
    const DevSegment seg = batch.seg[si];
    const uint32_t tile = blk - __ldg(&batch.blur_start[si]);
    const DevPair& P = batch.pair[seg.pair];
    TileRef t;
    t.pa = P.pyramid + P.plane_off[seg.level][seg.channel];
    t.pb = t.pa + P.image_stride;
    t.pitch = P.pitch[seg.level];
    t.w = static_cast<int>(P.w[seg.level]);
    t.h = static_cast<int>(P.h[seg.level]);
    t.x0 = static_cast<int>((tile % seg.tiles_x) * TW);
    t.y0 = static_cast<int>((tile / seg.tiles_x) * TH);
    t.partial = (static_cast<size_t>(seg.partial_first) + tile) * 6;
    return t;
}

// Asynchronous 4-byte global-to-shared copy; a source size of 0 writes zero
// and reads nothing (the zero padding of scale.comp:107-124).
__device__ __forceinline__ void CpAsync4(float* dst, const float* src, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    const int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(src), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void CpAsyncCommit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void CpAsyncWait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issues the copies of one tile's two source tiles into `buf` (row pairs).
template <int TW, int TH, int NT>
__device__ __forceinline__ void IssueTileLoads(float* buf, const TileRef& t) {
    using T = PackedTile<TW, TH, NT>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* bufb = buf + 2 * T::RP * T::SW;
    for (int r = warp; r < T::SH; r += T::kWarps) {
        const int gy = t.y0 - kRadius + r;
        const bool iny = gy >= 0 && gy < t.h;
        const size_t row = iny ? static_cast<size_t>(gy) * t.pitch : 0;
        const int e0 = (r >> 1) * T::SW * 2 + (r & 1);
        for (int c = lane; c < T::SW; c += 32) {
            const int gx = t.x0 - kRadius + c;
            const bool in = iny && gx >= 0 && gx < t.w;
            const size_t off = in ? row + static_cast<size_t>(gx) : 0;
            CpAsync4(buf + e0 + 2 * c, t.pa + off, in);
            CpAsync4(bufb + e0 + 2 * c, t.pb + off, in);
        }
    }
}

__device__ __forceinline__ float2 Pack(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 Neg(float2 v) { return make_float2(-v.x, -v.y); }

// Horizontal pass (scale.comp:149-207): row pair rp, columns c0..c0+3, all
// five quantities.
template <int TW, int TH, int NT>
__device__ __forceinline__ void HorizontalPass(const float2* src, float* hq) {
    using T = PackedTile<TW, TH, NT>;
    constexpr int SW = T::SW, KH = T::KH;
    const float2* srca = src;
    const float2* srcb = src + T::RP * SW;
    for (int task = threadIdx.x; task < T::HT; task += NT) {
        const int rp = task / (TW / KH);
        const int c0 = (task % (TW / KH)) * KH;
        float2 A[KH + 12], B[KH + 12];
#pragma unroll
        for (int j = 0; j < KH + 12; j += 2) {
            const float4 va = *reinterpret_cast<const float4*>(&srca[rp * SW + c0 + j]);
            const float4 vb = *reinterpret_cast<const float4*>(&srcb[rp * SW + c0 + j]);
            A[j] = make_float2(va.x, va.y);
            A[j + 1] = make_float2(va.z, va.w);
            B[j] = make_float2(vb.x, vb.y);
            B[j + 1] = make_float2(vb.z, vb.w);
        }
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
            for (int k = 0; k < KH; ++k) acc[k] = __fmul2_rn(Pack(c_taps[0]), S[k]);
#pragma unroll
            for (int t = 1; t < kTaps; ++t) {
                const float2 wt = Pack(c_taps[t]);
#pragma unroll
                for (int k = 0; k < KH; ++k) acc[k] = __ffma2_rn(wt, S[k + t], acc[k]);
            }
            float* plane = hq + q * T::SH * TW;
            *reinterpret_cast<float4*>(&plane[(2 * rp) * TW + c0]) =
                make_float4(acc[0].x, acc[1].x, acc[2].x, acc[3].x);
            *reinterpret_cast<float4*>(&plane[(2 * rp + 1) * TW + c0]) =
                make_float4(acc[0].y, acc[1].y, acc[2].y, acc[3].y);
        }
    }
}

// Vertical pass (scale.comp:211-301) on column pairs, the maps
// (scale.comp:305-333) of each task's eight pixels, and the block's
// compensated reduction to six partials (scale.comp:395-436, with two-sum
// compensation in place of the plain ladder). Ends with the partial written
// and a barrier, so src and hq may be reused afterwards.
template <int TW, int TH, int NT>
__device__ __forceinline__ void VerticalMapsReduce(const float2* src, const float* hq,
                                                   const TileRef& t, double* partials,
                                                   float (*red)[12]) {
    using T = PackedTile<TW, TH, NT>;
    constexpr int SW = T::SW, RV = T::RV;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float2* srca = src;
    const float2* srcb = src + T::RP * SW;
    float2 sum[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sum[k] = make_float2(0.0f, 0.0f);

    for (int task = tid; task < T::VT; task += NT) {
        const int c = (task % (TW / 2)) * 2;
        const int r0 = (task / (TW / 2)) * RV;
        float2 V[5][RV];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const float* plane = hq + q * T::SH * TW;
            float2 M[RV + 12];
#pragma unroll
            for (int i = 0; i < RV + 12; ++i)
                M[i] = *reinterpret_cast<const float2*>(&plane[(r0 + i) * TW + c]);
#pragma unroll
            for (int j = 0; j < RV; ++j) {
                float2 acc = __fmul2_rn(Pack(c_taps[0]), M[j]);
#pragma unroll
                for (int k = 1; k < kTaps; ++k) acc = __ffma2_rn(Pack(c_taps[k]), M[j + k], acc);
                V[q][j] = acc;
            }
        }
        const int out_x = t.x0 + c;
#pragma unroll
        for (int j = 0; j < RV; ++j) {
            const int out_y = t.y0 + r0 + j;
            if (out_y >= t.h || out_x >= t.w) continue;
            const bool second = out_x + 1 < t.w;
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
            // The raw XYB values are the centre of the source tile.
            const int rr = r0 + j + kRadius;
            const float2 s1a = srca[(rr >> 1) * SW + c + kRadius];
            const float2 s1b = srca[(rr >> 1) * SW + c + kRadius + 1];
            const float2 s2a = srcb[(rr >> 1) * SW + c + kRadius];
            const float2 s2b = srcb[(rr >> 1) * SW + c + kRadius + 1];
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
        partials[t.partial + tid] = static_cast<double>(a) + static_cast<double>(cc);
    }
    __syncthreads();
}

// One output tile per CTA.
template <int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) Ss2Blur2Kernel(DevBatch batch) {
    using T = PackedTile<TW, TH, NT>;
    extern __shared__ __align__(16) unsigned char smem[];
    float* src = reinterpret_cast<float*>(smem);
    float* hq = reinterpret_cast<float*>(smem + T::kSrcBytes);
    __shared__ float red[T::kWarps][12];
    const TileRef t = LocateTile<TW, TH>(batch, blockIdx.x);
    IssueTileLoads<TW, TH, NT>(src, t);
    CpAsyncCommit();
    CpAsyncWait<0>();
    __syncthreads();
    HorizontalPass<TW, TH, NT>(reinterpret_cast<const float2*>(src), hq);
    __syncthreads();
    VerticalMapsReduce<TW, TH, NT>(reinterpret_cast<const float2*>(src), hq, t, batch.partials, red);
}

// Persistent: each CTA walks tiles blockIdx.x, + gridDim.x, ... and copies
// tile i+1's sources into its second buffer while it computes tile i.
template <int TW, int TH, int NT>
__global__ void __launch_bounds__(NT) Ss2Blur3Kernel(DevBatch batch) {
    using T = PackedTile<TW, TH, NT>;
    extern __shared__ __align__(16) unsigned char smem[];
    float* const buf0 = reinterpret_cast<float*>(smem);
    constexpr int kBufFloats = static_cast<int>(T::kSrcBytes / sizeof(float));
    float* hq = reinterpret_cast<float*>(smem + 2 * T::kSrcBytes);
    __shared__ float red[T::kWarps][12];
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
        CpAsyncCommit();    // possibly empty, so the group count stays uniform
        CpAsyncWait<1>();   // everything but the newest group: this tile's
        __syncthreads();
        HorizontalPass<TW, TH, NT>(reinterpret_cast<const float2*>(now), hq);
        __syncthreads();
        VerticalMapsReduce<TW, TH, NT>(reinterpret_cast<const float2*>(now), hq, cur,
                                       batch.partials, red);
        cur = nxt;
        b ^= 1;
    }
    CpAsyncWait<0>();
}

// The variants compiled in: {tile width, tile height, threads, kind};
// kind 0 scalar, 1 packed, 2 persistent packed.
struct BlurVariant {
    int w, h, threads, kind;
};
constexpr BlurVariant kBlurVariants[] = {
    {32, 32, 256, 0}, {32, 32, 128, 1}, {64, 32, 256, 1}, {32, 52, 128, 1},
    {64, 20, 256, 1}, {32, 32, 128, 2}, {64, 32, 256, 2}, {32, 20, 128, 2},
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

template <int TW, int TH, int NT>
cudaError_t LaunchPacked(const DevBatch& b, cudaStream_t stream) {
    using T = PackedTile<TW, TH, NT>;
    static LaunchCache cache;
    constexpr size_t smem = T::kSrcBytes + T::kHqBytes;
    const cudaError_t e = Prepare(Ss2Blur2Kernel<TW, TH, NT>, smem, cache, NT, false, nullptr);
    if (e != cudaSuccess) return e;
    Ss2Blur2Kernel<TW, TH, NT><<<b.blur_blocks, NT, smem, stream>>>(b);
    return cudaGetLastError();
}

template <int TW, int TH, int NT>
cudaError_t LaunchPersistent(const DevBatch& b, cudaStream_t stream) {
    using T = PackedTile<TW, TH, NT>;
    static LaunchCache cache;
    constexpr size_t smem = 2 * T::kSrcBytes + T::kHqBytes;
    int grid = 0;
    const cudaError_t e = Prepare(Ss2Blur3Kernel<TW, TH, NT>, smem, cache, NT, true, &grid);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = b.blur_blocks < static_cast<uint32_t>(grid) ? b.blur_blocks
                                                                        : static_cast<uint32_t>(grid);
    Ss2Blur3Kernel<TW, TH, NT><<<blocks, NT, smem, stream>>>(b);
    return cudaGetLastError();
}

}  // namespace

cudaError_t SetConstants(const float* taps13, const double* weights108) {
    cudaError_t e = cudaMemcpyToSymbol(c_taps, taps13, sizeof(float) * kTaps);
    if (e != cudaSuccess) return e;
    return SetScoreWeights(weights108);
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
        case 5: return LaunchPersistent<32, 32, 128>(b, stream);
        case 6: return LaunchPersistent<64, 32, 256>(b, stream);
        case 7: return LaunchPersistent<32, 20, 128>(b, stream);
    }
    return cudaErrorInvalidValue;
}

int BlurTileCount() { return kBlurVariantCount; }
int BlurTileThreads(int index) { return kBlurVariants[index].threads; }
void BlurTileShape(int index, int* w, int* h) {
    *w = kBlurVariants[index].w;
    *h = kBlurVariants[index].h;
}

}  // namespace vqm_b200
