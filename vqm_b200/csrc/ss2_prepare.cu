// Prepare stage for sm_100a: decode -> linear Rec.709 -> XYB -> the whole
// 2x2-box pyramid of one image's 32x32 base tile, per CTA
// (reference: src/metrics/ssimulacra2/shaders/prepare.comp).
//
// A CTA is 256 threads; thread (tx, ty) owns the base 2x2 block
// (gx*16 + tx, gy*16 + ty). Levels 0 and 1 come from the thread's own four
// samples; levels 2.. pass the previous level's tile through a shared-memory
// ladder, two buffers alternating so each level costs one barrier. Because
// the 2x2 box nests exactly, no CTA ever needs a neighbour's samples.
//
// Two specialisations: 8-bit grey/RGB without alpha decode through the
// image's 256-entry table in shared memory; every other format runs the
// generic decode of ss2_decode.cuh. The cube root of the XYB transform is the
// shared deterministic one (ss2_detmath.h), so the planes this kernel writes
// are bit-identical to the CPU checker's.

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "ss2_decode.cuh"
#include "ss2_detmath.h"
#include "ss2_device.cuh"
#include "ss2_kernels.h"

namespace vqm_b200 {
namespace {

constexpr int kThreads = 256;

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

// prepare.comp:81-98. Only the channels in `mask` are produced; B's cube
// root is skipped when B is not stored.
__device__ __forceinline__ void Xyb(float r, float g, float b, uint32_t mask, float out[3]) {
    float m0 = __fmaf_rn(kM00, r, __fmaf_rn(kM01, g, __fmaf_rn(kM02, b, kBias)));
    float m1 = __fmaf_rn(kM10, r, __fmaf_rn(kM11, g, __fmaf_rn(kM12, b, kBias)));
    m0 = fmaxf(m0, 0.0f);
    m1 = fmaxf(m1, 0.0f);
    const float c0 = __fsub_rn(ss2dm::cbrt(m0), kCbrtBias);
    const float c1 = __fsub_rn(ss2dm::cbrt(m1), kCbrtBias);
    const float sum = __fadd_rn(c0, c1);
    out[0] = __fmaf_rn(__fmul_rn(0.5f, __fsub_rn(c0, c1)), 14.0f, 0.42f);
    out[1] = __fmaf_rn(0.5f, sum, 0.01f);
    out[2] = 0.0f;
    if (mask & 4u) {
        float m2 = __fmaf_rn(kM20, r, __fmaf_rn(kM21, g, __fmaf_rn(kM22, b, kBias)));
        m2 = fmaxf(m2, 0.0f);
        const float c2 = __fsub_rn(ss2dm::cbrt(m2), kCbrtBias);
        out[2] = __fadd_rn(__fmaf_rn(-0.5f, sum, c2), 0.55f);
    }
}

// prepare.comp:103-111: ((((0 + a) + b) + c) + d) * 0.25.
__device__ __forceinline__ float BoxAverage(float a, float b, float c, float d) {
    return __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(a, b), c), d), 0.25f);
}

// Per-level addressing of this image's planes, staged in shared memory.
struct LevelInfo {
    float* plane[kMaxLevels][3];  // nullptr when pruned
    uint32_t w[kMaxLevels], h[kMaxLevels], pitch[kMaxLevels], mask[kMaxLevels];
    uint32_t levels;
};

// Two adjacent samples of one 8-bit row: one 16-bit load when the address
// allows it, the clamped pair otherwise.
__device__ __forceinline__ void LoadByte2(const uint8_t* row, uint32_t x0, uint32_t x1,
                                         uint32_t& a, uint32_t& b) {
    const uint8_t* p = row + x0;
    if (x1 == x0 + 1 && (reinterpret_cast<uintptr_t>(p) & 1u) == 0) {
        const uint32_t v = __ldg(reinterpret_cast<const uint16_t*>(p));
        a = v & 0xffu;
        b = v >> 8;
    } else {
        a = __ldg(p);
        b = __ldg(row + x1);
    }
}

template <bool kTable>
__global__ void __launch_bounds__(kThreads) PrepareKernel(DevBatch batch) {
    __shared__ float ladder[2][256 * 3];
    __shared__ float lut[256];
    __shared__ DevSource src_s;
    __shared__ LevelInfo lv;

    const uint32_t tid = threadIdx.x;
    const int group = kTable ? 0 : 1;
    const uint32_t n_items = batch.prep_items[group];
    const DevPrepItem* items = batch.prep_item + (kTable ? 0 : batch.prep_items[0]);
    const uint32_t* start = batch.prep_start + (kTable ? 0 : batch.prep_items[0] + 1);
    const uint32_t it = FindSlot(start, n_items, blockIdx.x);
    const DevPrepItem item = items[it];
    const DevPair& P = batch.pair[item.pair];
    const uint32_t t = blockIdx.x - __ldg(&start[it]);
    const uint32_t gx = t % P.prep_tiles_x;
    const uint32_t gy = t / P.prep_tiles_x;
    const int image = static_cast<int>(item.image);

    {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&P.src[image]);
        uint32_t* to = reinterpret_cast<uint32_t*>(&src_s);
        constexpr uint32_t words = offsetof(DevSource, srgb_lut) / 4;
        for (uint32_t i = tid; i < words; i += kThreads) to[i] = from[i];
        if (kTable) lut[tid] = P.src[image].srgb_lut[tid];
        if (tid < kMaxLevels * 3) {
            const uint32_t l = tid / 3, c = tid % 3;
            const bool kept = l < P.levels && (P.mask[l] & (1u << c));
            lv.plane[l][c] = kept ? P.pyramid + static_cast<size_t>(image) * P.image_stride +
                                        P.plane_off[l][c]
                                  : nullptr;
        }
        if (tid < kMaxLevels) {
            lv.w[tid] = P.w[tid];
            lv.h[tid] = P.h[tid];
            lv.pitch[tid] = P.pitch[tid];
            lv.mask[tid] = tid < P.levels ? P.mask[tid] : 0u;
        }
        if (tid == 0) lv.levels = P.levels;
    }
    __syncthreads();
    const DevSource& s = src_s;
    const uint32_t levels = lv.levels;
    const uint32_t width = s.width, height = s.height;
    const uint32_t bx = gx * 16 + (tid & 15);
    const uint32_t by = gy * 16 + (tid >> 4);
    const bool in_block = bx < (width + 1) / 2 && by < (height + 1) / 2;

    // The block's four samples in (0,0), (1,0), (0,1), (1,1) order.
    float lin[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (in_block) {
        const uint32_t x0 = 2 * bx, y0 = 2 * by;
        const uint32_t x1 = min(x0 + 1, width - 1), y1 = min(y0 + 1, height - 1);
        if (kTable) {
            const bool grey = s.family == 0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int pl = grey ? 0 : c;
                const uint8_t* r0 = s.plane[pl] + static_cast<size_t>(y0) * s.row_bytes[pl];
                const uint8_t* r1 = s.plane[pl] + static_cast<size_t>(y1) * s.row_bytes[pl];
                uint32_t a, b, d, e;
                LoadByte2(r0, x0, x1, a, b);
                LoadByte2(r1, x0, x1, d, e);
                lin[0][c] = lut[a];
                lin[1][c] = lut[b];
                lin[2][c] = lut[d];
                lin[3][c] = lut[e];
            }
            if (!s.identity2) {
#pragma unroll
                for (int i = 0; i < 4; ++i) ApplyMatrix(s.m2, lin[i]);
            }
        } else {
            BlockLinearGeneric(s, bx, by, lin);
        }
        // Level 0: rows y0 and (if inside) y0 + 1, each as one float2 when
        // both columns are inside, else the single last column.
        const uint32_t mask0 = lv.mask[0];
        if (mask0) {
            float v[4][3];
#pragma unroll
            for (int i = 0; i < 4; ++i) Xyb(lin[i][0], lin[i][1], lin[i][2], mask0, v[i]);
            const bool two = x0 + 1 < width;
            const bool second_row = y0 + 1 < height;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (!(mask0 & (1u << c))) continue;
                float* row0 = lv.plane[0][c] + static_cast<size_t>(y0) * lv.pitch[0] + x0;
                float* row1 = row0 + lv.pitch[0];
                if (two) {
                    *reinterpret_cast<float2*>(row0) = make_float2(v[0][c], v[1][c]);
                    if (second_row) *reinterpret_cast<float2*>(row1) = make_float2(v[2][c], v[3][c]);
                } else {
                    row0[0] = v[0][c];
                    if (second_row) row1[0] = v[2][c];
                }
            }
        }
    }

    // Levels past the deepest one that stores a channel are not computed:
    // nothing reads them (at six scales level 5 keeps no channel).
    uint32_t last = 0;
    for (uint32_t l = 1; l < levels; ++l)
        if (lv.mask[l]) last = l;

    // Level 1: every thread, from its own four samples.
    if (last >= 1) {
        float v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = BoxAverage(lin[0][c], lin[1][c], lin[2][c], lin[3][c]);
        const uint32_t x = gx * 16 + (tid & 15), y = gy * 16 + (tid >> 4);
        const uint32_t mask = lv.mask[1];
        if (mask && x < lv.w[1] && y < lv.h[1]) {
            float xyb[3];
            Xyb(v[0], v[1], v[2], mask, xyb);
            const size_t at = static_cast<size_t>(y) * lv.pitch[1] + x;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (mask & (1u << c)) lv.plane[1][c][at] = xyb[c];
        }
        if (last >= 2) {
#pragma unroll
            for (int c = 0; c < 3; ++c) ladder[1][tid * 3 + c] = v[c];
        }
    }
    if (last < 2) return;
    __syncthreads();

    // Levels 2..last: the first side^2 threads (64, 16, 4, 1) average the
    // previous level's 2x2 blocks from the ladder (prepare.comp:149-168,
    // clamped to the previous level's last column and row); threads that no
    // longer take part leave, and the rest meet at a barrier of their own.
    for (uint32_t level = 2; level <= last; ++level) {
        const uint32_t side = 32u >> level;  // a power of two: shifts, not divisions
        const uint32_t active = side * side;
        if (tid >= active) return;
        const uint32_t jx = tid & (side - 1);
        const uint32_t jy = tid >> (5 - level);
        const uint32_t slot = (level - 1) & 1u;
        const uint32_t prev_side = side * 2;
        const uint32_t pw = lv.w[level - 1], ph = lv.h[level - 1];
        const uint32_t ox = min(gx * prev_side, pw - 1);
        const uint32_t oy = min(gy * prev_side, ph - 1);
        const uint32_t lx = pw - 1 - ox, ly = ph - 1 - oy;
        const uint32_t cx0 = min(2 * jx, lx), cx1 = min(2 * jx + 1, lx);
        const uint32_t cy0 = min(2 * jy, ly), cy1 = min(2 * jy + 1, ly);
        float v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
            v[c] = BoxAverage(ladder[slot][(cy0 * prev_side + cx0) * 3 + c],
                              ladder[slot][(cy0 * prev_side + cx1) * 3 + c],
                              ladder[slot][(cy1 * prev_side + cx0) * 3 + c],
                              ladder[slot][(cy1 * prev_side + cx1) * 3 + c]);
        const uint32_t x = gx * side + jx;
        const uint32_t y = gy * side + jy;
        const uint32_t mask = lv.mask[level];
        if (mask && x < lv.w[level] && y < lv.h[level]) {
            float xyb[3];
            Xyb(v[0], v[1], v[2], mask, xyb);
            const size_t at = static_cast<size_t>(y) * lv.pitch[level] + x;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (mask & (1u << c)) lv.plane[level][c][at] = xyb[c];
        }
        if (level < last) {
#pragma unroll
            for (int c = 0; c < 3; ++c) ladder[level & 1u][tid * 3 + c] = v[c];
            if (active > 32) {
                // Level 2's 64 threads are warps 0 and 1, whole.
                asm volatile("bar.sync 1, %0;" ::"r"(active) : "memory");
            } else {
                __syncwarp((1u << active) - 1u);
            }
        }
    }
}

}  // namespace

cudaError_t LaunchPrepare(const DevBatch& b, cudaStream_t stream) {
    if (b.prep_blocks[0]) PrepareKernel<true><<<b.prep_blocks[0], kThreads, 0, stream>>>(b);
    if (b.prep_blocks[1]) PrepareKernel<false><<<b.prep_blocks[1], kThreads, 0, stream>>>(b);
    return cudaGetLastError();
}

}  // namespace vqm_b200
