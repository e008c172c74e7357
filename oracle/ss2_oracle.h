/*
 * CPU oracle for the SSIMULACRA 2.1 scorer -- TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, on the CPU, the arithmetic of VQM's SSIMULACRA 2.1
 * path (GreatValueCreamSoda/vqm): the input decode of
 * src/vulkan/shaders/color.glsl, the XYB pyramid of
 * src/metrics/ssimulacra2/shaders/prepare.comp, the blurs, maps and norm
 * partials of shaders/scale.comp, the partial reduction of shaders/reduce.comp,
 * the FP64 read-back of src/metrics/ssimulacra2/vulkan.cc (ReadResult) and the
 * score mapping of src/metrics/ssimulacra2/score.cc.
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * may load it, and only as the checker. The CUDA scorer never calls it.
 *
 * Pinning: the FP32 variant is checked against the reference test suite's own
 * golden scores (tests/metrics/ssimulacra2/pipeline_test.cc:146-174, 32x32
 * gradient pairs 93.17505696 / 92.12553218 within 5e-3), its identity rule
 * (:120-144, exactly 100) and its scale counts (:760-783); the score mapping,
 * pruning predicate and decode constants are checked bit for bit against the
 * reference's own score.cc / input.cc compiled from source into oracle/_ref.
 *
 * Norm layout of every `norms` array: scale-major, 18 doubles per scale in the
 * order of Ssimulacra2Scale (include/ssimulacra2.h:18-25): avg_ssim[c*2+n]
 * (6 values), then avg_edgediff[c*4+n] (12 values; n 0,1 ringing, 2,3
 * blurring).
 */
#ifndef VQM_SS2_ORACLE_H_
#define VQM_SS2_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* vqm::ImageFormat (include/vqm_image.h:325-337), zimg numeric values. */
typedef struct ss2o_format {
    uint8_t type;            /* 0 Byte, 1 Word, 2 Half, 3 Float */
    uint8_t family;          /* 0 Grey, 1 Rgb, 2 Yuv */
    uint8_t alpha;           /* 0 None, 1 Straight, 2 Premultiplied */
    uint8_t range;           /* 0 Limited, 1 Full */
    uint8_t matrix;          /* MatrixCoefficients */
    uint8_t transfer;        /* TransferCharacteristics */
    uint8_t primaries;       /* ColorPrimaries */
    uint8_t chroma_location; /* ChromaLocation */
    uint8_t subsample_w;     /* log2 */
    uint8_t subsample_h;     /* log2 */
    uint8_t depth;           /* 0 = full depth of the type */
    uint8_t reserved;
} ss2o_format;

/* A packed image in vqm::Image's layout (include/vqm_image.h:339-358). */
typedef struct ss2o_image {
    uint32_t width;
    uint32_t height;
    ss2o_format format;
    const uint8_t* data;
    size_t bytes;
} ss2o_image;

/* Status codes. */
#define SS2O_OK 0
#define SS2O_INVALID 1

/* Scores one pair. precision: 32 = the FP32 restatement (VQM proxy), 64 =
 * the same algorithm in FP64, 16 = the FP32 restatement of VQM's half-plane
 * build (pyramid planes and level averages rounded to binary16), 33 = the
 * FP32 restatement with s11 + s22 blurred as one quantity (the CUDA blur's
 * four-quantity mode; not VQM's rounding). blur: 0 = VQM's sampled
 * Gaussian, 1 = the opt-in recursive Gaussian (FP32: its impulse response
 * as 13 float taps, the CUDA kernels' evaluation; FP64: the recursion
 * itself). Writes 18*scales doubles into norms[108], the scale count into
 * *scales and the score into *score. */
int ss2o_compute(const ss2o_image* original, const ss2o_image* distorted,
                 float background, int chroma_filter, int precision, int blur,
                 double* norms, uint32_t* scales, double* score);

/* Scores n pairs on `threads` host threads (one pair per thread at a time). */
int ss2o_compute_many(uint32_t n, const ss2o_image* originals,
                      const ss2o_image* distorteds, float background,
                      int chroma_filter, int precision, int blur, uint32_t threads,
                      double* norms, uint32_t* scales, double* scores);

/* Pieces, exposed so the tests can pin them one by one. */
int ss2o_plan_scales(uint32_t width, uint32_t height, uint32_t* sizes12);
void ss2o_gaussian(float* taps13);
/* The recursive Gaussian (sigma 1.5): window half-width, the three
 * frequencies and coefficients, and its impulse response in double as 13
 * taps (offsets -6..6). */
void ss2o_recursive_gaussian(int* radius, double* freqs3, double* beta3, double* taps13);
/* One plane blurred, zero padded: precision 64 in double (the recursive
 * mode by its recursion), 32 in float by the 13-tap passes. */
int ss2o_blur_plane(int blur, int precision, const double* in, uint32_t width,
                    uint32_t height, double* out);
int ss2o_channel_pruned(uint32_t channel, uint32_t scale, uint32_t scales);
int ss2o_score(const double* norms, uint32_t scales, double* score);
int ss2o_required_bytes(const ss2o_format* format, uint32_t width,
                        uint32_t height, size_t* bytes);
/* The FP32 decode constants of one format: 44 words in VQM's SourceDesc
 * order (src/vulkan/vulkan_support.h:104-120) with plane offsets zero. */
int ss2o_source_desc(const ss2o_format* format, int chroma_filter,
                     uint32_t* words44);
/* The FP32 pyramid of one image: for each level, 3 planes of W_l*H_l floats
 * (channel X, Y, B) with pruned channels left at NaN, concatenated level by
 * level. Returns the float count through *count. */
int ss2o_pyramid(const ss2o_image* image, float background, int chroma_filter,
                 float* out, size_t capacity, size_t* count);
/* Raw per-level norm sums (18 floats per level) of the FP32 path. */
int ss2o_level_sums(const ss2o_image* original, const ss2o_image* distorted,
                    float background, int chroma_filter, float* sums,
                    uint32_t* scales);
/* The shared deterministic functions, for their accuracy tests: fn 0 cube
 * root, 1 pow(x, y), 2 exp, 3 sin(pi x), 4 rounding to binary16 (the
 * half-plane build's plane rounding), 5 the power-law transfers' power,
 * 6 the maps' division x / y. */
int ss2o_detmath(int fn, const float* x, float y, float* out, size_t n);
const char* ss2o_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* VQM_SS2_ORACLE_H_ */
