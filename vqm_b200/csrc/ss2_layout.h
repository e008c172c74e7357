// Pyramid plane layout shared by the host runtime and the kernels.
//
// Each kept (level, channel) plane of an image is stored as "row pairs":
// element (x, y) lives at float offset (y >> 1) * pitch + 2 * x + (y & 1), so
// rows 2p and 2p+1 are interleaved column by column and one aligned 16-byte
// access holds the 2x2 block at (2i, 2p). The prepare kernel writes a base
// 2x2 block as one float4; the blur kernel copies its tiles in 16-byte chunks
// and its horizontal pass gets two rows of a column from one 64-bit load.
//
// pitch = 2 * round_up(w, 32) floats, so every row pair starts on a 256-byte
// boundary. Column w (when w is odd) and row h (when h is odd) are padding
// that prepare writes as 0: a 2x2 chunk at the right or bottom edge then
// reads zeros there, which is the blur's zero padding (scale.comp:107-124).
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
SS2_HD size_t PlaneIndex(uint32_t pitch, uint32_t x, uint32_t y) {
    return static_cast<size_t>(y >> 1) * pitch + 2u * x + (y & 1u);
}

}  // namespace vqm_b200
