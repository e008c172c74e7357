// Device-side data layout of the SSIMULACRA 2.1 scorer: what the host
// runtime writes into device memory once per batch shape and the kernels read.
//
// A "batch" is any list of image pairs, of any sizes and formats: a plain
// one-pair call is a batch of one. Work is flattened into three launch
// spaces so that every kernel covers every pair of the batch in one grid:
//
//   prepare  one CTA per (pair, image, 64x64 base tile): decode, linear RGB,
//            XYB, and the whole 2x2 box pyramid of that tile
//            (reference: src/metrics/ssimulacra2/shaders/prepare.comp).
//   blur     one CTA per (pair, level, kept channel, output tile): the five
//            13-tap blurs, the SSIM' and edge maps and the six norm partials
//            (reference: shaders/scale.comp).
//   finalize one CTA per (pair, level, kept channel) segment: the FP64 sum of
//            the tile partials; the last segment of a pair to finish turns
//            the 18 x levels sums into the 108 norms and the score
//            (reference: shaders/reduce.comp, vulkan.cc:545-583 ReadResult,
//            score.cc:118-163 Score).
//
// Pyramid planes are FP32 in row pairs (ss2_layout.h): rows 2p and 2p + 1
// interleaved column by column, each row pair on a 256-byte boundary.
#pragma once

#include <cstdint>

#include <vector_types.h>

namespace vqm_b200 {

constexpr int kMaxLevels = 6;
constexpr int kChannels = 3;
constexpr int kTaps = 13;
constexpr int kRadius = 6;
constexpr int kNormsPerChannel = 6;
constexpr int kSumsPerLevel = 18;
// Per pair result block: 108 norms, the score, the scale count, a status.
// The prepare kernels' cube root takes its short route (special-function
// unit estimate, one Newton step) for inputs in [2^-16, 2^24): there it is
// checked, on every float, to equal the shared correctly rounded cube root.
// XYB mixes of linear samples in [0, 1.6e7] lie in that band: they are at
// least the opsin bias 0.0038 and at most the largest sample plus the bias.
constexpr float kCbrtRouteLo = 1.52587890625e-05f;  // 2^-16
constexpr float kCbrtRouteHi = 16777216.0f;        // 2^24
constexpr float kInRangeLinearMax = 1.6e7f;

constexpr int kResultDoubles = 112;
constexpr int kResultScore = 108;
constexpr int kResultScales = 109;
constexpr int kResultStatus = 110;

// One input image as the decode reads it: the per-image constants of VQM's
// SourceDesc (src/vulkan/vulkan_support.h:104-120) with device pointers and
// byte strides in place of arena word offsets, so caller-owned padded device
// buffers are read in place.
// Everything about one image the prepare kernels read per CTA (staged in
// shared memory); DevSource adds the 8-bit byte table, which the table
// kernels stage separately, so the CTAs do not hold its 1 KB twice.
struct DevSourceHead {
    const uint8_t* plane[4];   // device address of each plane's first row
    uint32_t row_bytes[4];     // row stride of each plane, bytes
    uint32_t plane_w[4];       // samples per row of each plane
    uint32_t plane_h[4];       // rows of each plane
    uint32_t width, height;    // the image (plane 0) size
    uint8_t type;              // 0 Byte, 1 Word, 2 Half, 3 Float
    uint8_t family;            // 0 Grey, 1 Rgb, 2 Yuv
    uint8_t alpha;             // 0 None, 1 Straight, 2 Premultiplied
    uint8_t sub_w, sub_h;      // log2 chroma subsampling
    uint8_t transfer;          // transfer id 0..11 (input.cc:664-698)
    uint8_t mode;              // 0 matrix, 1 constant luminance, 2 ICtCp
    uint8_t filter;            // chroma filter 0 bilinear, 1 bicubic, 2 lanczos
    uint8_t identity1, identity2;
    uint8_t chroma_variant;    // subsampled chroma planes present
    uint8_t lut;               // 1: 8-bit RGB, no alpha: decode by table
    uint8_t in_range;          // 1: every linear sample is in [0, 1.6e7] and
                               // there is no primaries matrix, so every XYB
                               // mix of the image and its levels lies in
                               // [kCbrtRouteLo, kCbrtRouteHi) (see below)
    float scale[3], offset[3]; // luma, chroma, alpha
    float m1[9], m2[9];        // encoded->RGB (or ICtCp->LMS), primaries->709
    float kr, kg, kb, to_linear;
    float shift_x, shift_y;
    float cl[4];               // constant-luminance corner values
    float background;          // alpha blend target
    // The YUV fast path (BlockLinearYuv, ss2_decode.cuh): integer YUV without
    // alpha, matrix mode, a pure power-law transfer and chroma subsampled by
    // at most 2 with bilinear upsampling. For a 2x2 luma block at even
    // coordinates the bilinear phase of each output depends only on its
    // parity, so the host fixes the first window slot and the four tap
    // weights per parity. Also requires the YUV matrix to map every sample
    // code below the transfer power's fast-range limit.
    uint8_t yuv_fast;
    uint8_t chroma_pattern;    // 4:2:0 phases known at compile time: 1 + x type
                               // + 2 y type (type 0: siting offset 0, type 1:
                               // offset 1/4); 0: use cslot and cweight
    int8_t cslot[2][2];        // [0 = x, 1 = y][parity]: first window slot
    float gamma;               // the transfer exponent
    float cweight[2][2][4];    // [y parity][x parity]: w00, w10, w01, w11
};
struct DevSource : DevSourceHead {
    float srgb_lut[256];       // transfer(raw * scale + offset) per byte code
};
static_assert(sizeof(DevSourceHead) % 4 == 0, "the head is copied in words");

// One pair of a batch.
struct DevPair {
    DevSource src[2];
    uint32_t levels;
    uint32_t w[kMaxLevels], h[kMaxLevels], pitch[kMaxLevels];
    uint32_t mask[kMaxLevels];          // kept channels per level, bit c
    // Float offset, from `pyramid`, of plane [level][channel] of image 0;
    // image 1's plane follows at + image_stride. Pruned planes are absent.
    uint64_t plane_off[kMaxLevels][kChannels];
    uint64_t image_stride;
    float* pyramid;
    uint32_t prep_tiles_x, prep_tiles_y;  // kPrepTile-square base tiles per image
    uint32_t seg_first, seg_count;        // this pair's blur segments
    double* result;                       // kResultDoubles per pair
};

// One (pair, level, channel) of the blur stage.
struct DevSegment {
    uint32_t pair;
    uint32_t level;
    uint32_t channel;
    uint32_t tiles_x;
    uint32_t tiles;
    uint32_t partial_first;  // index of this segment's first partial
    uint32_t partials;       // partials the blur writes: one per CTA (a tile, or a strip)
};

// One image of one pair for the prepare stage. Images decoded through the
// 8-bit table come first in the list, the rest (generic decode) after them,
// each group with its own prefix offsets, so each group is one launch of its
// own specialised kernel.
struct DevPrepItem {
    uint32_t pair;
    uint32_t image;
};

// The prepare kernels, one per decode: 8-bit images by table (group 0),
// yuv_fast images of even width and height (group 1: every 2x2 block is
// whole, so its kernel carries no generic decode), every other image
// (group 2).
constexpr int kPrepGroups = 3;
inline int PrepGroup(const DevSource& s) {
    if (s.lut) return 0;
    return s.yuv_fast && s.width % 2 == 0 && s.height % 2 == 0 ? 1 : 2;
}
// Whether an image fits the 4:2:0 chroma window of the 128-thread YUV
// prepare kernel (4:2:0 chroma, or none subsampled).
inline bool Yuv420Window(const DevSource& s) {
    return !s.chroma_variant || (s.sub_w == 1 && s.sub_h == 1);
}

struct DevBatch {
    uint32_t pairs;
    uint32_t segments;
    uint32_t prep_items[kPrepGroups];   // images in each prepare group
    uint32_t prep_blocks[kPrepGroups];  // 64x64 base tiles in each group
    uint32_t blur_blocks;     // sum over segments of tiles
    const DevPair* pair;
    const DevSegment* seg;
    const DevPrepItem* prep_item;  // group 0, then group 1, then group 2
    // Prefix tile offsets, each group's prep_items[g] + 1 entries in group
    // order.
    const uint32_t* prep_start;
    const uint32_t* blur_start;  // segments + 1 prefix offsets
    double* partials;            // 6 doubles per blur partial (segment.partials each)
    double* seg_sums;            // 6 doubles per segment
    uint32_t* pair_done;         // per pair: segments summed so far (0 between launches)
    uint32_t* seg_done;          // per segment: partials written so far (0 between launches)
    uint32_t* blur_queue;        // the tile queue's next strip and exit count (0 between launches)
    uint32_t* status;            // nonzero: a kernel found bad input
    uint32_t half;               // 1: pyramid elements are binary16
    uint32_t yuv420;             // 1: every image of the YUV prepare group
                                 // has 4:2:0 chroma or none subsampled
    // The blur's 13 taps (offsets -6..6) as (w, w) pairs: the blur kernels
    // take them from the launch's parameter space, a constant bank like
    // __constant__ memory, so each batch carries its blur mode's filter.
    float2 taps2[kTaps];
};

}  // namespace vqm_b200
