// Pyramid plane layout shared by the host runtime and the kernels.
//
// Each kept (level, channel) plane of an image is stored as "row pairs":
// element (x, y) lives at float offset (y >> 1) * pitch + 2 * x + (y & 1), so
// rows 2p and 2p+1 are interleaved column by column and one aligned 16-byte
// access holds the 2x2 block at (2i, 2p). The prepare kernel writes a base
// 2x2 block as one float4; the blur kernel copies its tiles in 16-byte chunks
// and its horizontal pass gets two rows of a column from one 64-bit load.
//
// pitch = 2 * round_up(w, 32) elements, so every row pair starts on a
// 256-byte boundary (128 with half planes). The columns up to PaddedColumns(w)
// and row h (when h is odd) are padding that prepare writes as 0: a copy chunk
// at the right or bottom edge then reads zeros there, which is the blur's zero
// padding (scale.comp:107-124). With half planes the elements are binary16.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define SS2_HD __host__ __device__ __forceinline__
#else
#define SS2_HD inline
#endif

namespace vqm_b200 {

// Side, in base pixels, of the square tile one prepare CTA covers (its whole
// pyramid is built inside the CTA).
constexpr uint32_t kPrepTile = 64;
SS2_HD uint32_t PrepTiles(uint32_t size) { return (size + kPrepTile - 1) / kPrepTile; }

SS2_HD uint32_t RowPairPitch(uint32_t w) { return 2u * ((w + 31u) / 32u * 32u); }
SS2_HD uint32_t RowPairs(uint32_t h) { return (h + 1u) / 2u; }
SS2_HD size_t PlaneFloats(uint32_t w, uint32_t h) {
    return static_cast<size_t>(RowPairPitch(w)) * RowPairs(h);
}
// Columns of a level plane that prepare writes: the level's width rounded up
// to the blur's copy unit, 2 columns (one 16-byte chunk of float row pairs)
// or 4 with half planes (binary16 elements, same element layout); the
// columns past the width are written as 0.
SS2_HD uint32_t PaddedColumns(uint32_t w, bool half) {
    return half ? (w + 3u) & ~3u : (w + 1u) & ~1u;
}
SS2_HD size_t PlaneIndex(uint32_t pitch, uint32_t x, uint32_t y) {
    return static_cast<size_t>(y >> 1) * pitch + 2u * x + (y & 1u);
}

}  // namespace vqm_b200
