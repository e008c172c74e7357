/*
 * vqm_cu_ss2.h -- C ABI of the B200 SSIMULACRA 2.1 scorer.
 *
 * Drop-in boundary for VQM's SSIMULACRA 2 path (GreatValueCreamSoda/vqm):
 * every entry point below replaces one member of the reference's C++ API
 * (include/ssimulacra2.h, include/vqm_image.h, include/vqm_pool.h), cited
 * per function. Plain pointers, sizes and POD structs only; CUDA device
 * pointers take the place of VQM's Vulkan buffers, a cudaStream_t (passed as
 * void*) the place of its queue. include/vqm_cuda.hpp restores the
 * reference's C++ classes and exception types on top of this ABI.
 *
 * Errors: every function returns a status code (VQM_CU_OK = 0). The code
 * names the exception the reference throws in the same situation
 * (std::invalid_argument, std::logic_error, std::runtime_error,
 * std::overflow_error); vqm_cu_last_error() returns that call's message on
 * the calling thread. No function throws.
 *
 * Threading (include/ssimulacra2.h:66-70, 135-144): a pipeline is not
 * thread-safe and holds at most one submission in flight; a batch scorer
 * holds at most one batch in flight. Separate objects may be used from
 * separate threads.
 */
#ifndef VQM_CU_SS2_H_
#define VQM_CU_SS2_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VQM_CU_OK 0
#define VQM_CU_INVALID_ARGUMENT 1 /* std::invalid_argument */
#define VQM_CU_LOGIC_ERROR 2      /* std::logic_error */
#define VQM_CU_RUNTIME_ERROR 3    /* std::runtime_error (device, CUDA) */
#define VQM_CU_OVERFLOW_ERROR 4   /* std::overflow_error */

#define VQM_CU_MEMORY_HOST 0   /* planes are host addresses */
#define VQM_CU_MEMORY_DEVICE 1 /* planes are CUDA device addresses */

/* Norms per scale and the largest result: Ssimulacra2Scale
 * (include/ssimulacra2.h:18-25) flattened, avg_ssim[6] then avg_edgediff[12],
 * scale-major, up to six scales. */
#define VQM_CU_SS2_NORMS_PER_SCALE 18
#define VQM_CU_SS2_MAX_NORMS 108

/* vqm::ImageFormat (include/vqm_image.h:325-337), zimg numeric enum values. */
typedef struct vqm_cu_format {
    uint8_t type;            /* PixelType: 0 Byte, 1 Word, 2 Half, 3 Float */
    uint8_t family;          /* ColorFamily: 0 Grey, 1 Rgb, 2 Yuv */
    uint8_t alpha;           /* AlphaType: 0 None, 1 Straight, 2 Premultiplied */
    uint8_t range;           /* PixelRange: 0 Limited, 1 Full */
    uint8_t matrix;          /* MatrixCoefficients */
    uint8_t transfer;        /* TransferCharacteristics */
    uint8_t primaries;       /* ColorPrimaries */
    uint8_t chroma_location; /* ChromaLocation */
    uint8_t subsample_w;     /* log2, 0..2 */
    uint8_t subsample_h;     /* log2, 0..2 */
    uint8_t depth;           /* 0 = the pixel type's full depth */
    uint8_t reserved;        /* must be 0 */
} vqm_cu_format;

/* One image: vqm::Image (packed, include/vqm_image.h:339-358), vqm::ImageView
 * (strided host planes, include/vqm_views.h:18-24) or a caller-owned device
 * buffer (the CUDA counterpart of VulkanBufferView, include/vqm_vulkan.h).
 * planes[i] points at the first row of plane i (Y/R, U/G, V/B, alpha);
 * strides[i] is its row stride in bytes, 0 meaning tightly packed. Absent
 * planes are ignored. Device planes must stay unmodified until the
 * submission that reads them is finished. */
typedef struct vqm_cu_image {
    uint32_t width;
    uint32_t height;
    vqm_cu_format format;
    int32_t memory; /* VQM_CU_MEMORY_HOST or VQM_CU_MEMORY_DEVICE */
    const void* planes[4];
    size_t strides[4];
} vqm_cu_image;

/* Ssimulacra2Config (include/ssimulacra2.h:35-64). */
typedef struct vqm_cu_ss2_config {
    uint32_t width;
    uint32_t height;
    uint32_t gpu_resident_images; /* slots for upload(); default 2 */
    uint32_t half_planes;         /* 1: binary16 pyramid planes: FP32 arithmetic,
                                     the planes and the level averages rounded
                                     to binary16 (ssimu2_common.glsl:45-91) */
    uint32_t chroma_filter;       /* 0 bilinear, 1 bicubic, 2 lanczos */
    uint32_t streaming_inputs;    /* 1: host-image submit overloads allowed */
    uint64_t input_bytes;         /* pool for allocate_image(); 0 = none */
    int32_t device;               /* CUDA ordinal; -1 = the current device */
    uint32_t blur;                /* VQM_CU_SS2_BLUR_*; 0 = VQM's */
    uint32_t memory_policy;       /* VQM_CU_MEMORY_POLICY_* (MemoryPolicy,
                                     vqm_memory_types.h:12-14) */
} vqm_cu_ss2_config;

/* Where the kernels read the allocate_image() pool from. DIRECT (and
 * AUTOMATIC, which picks it): the pinned host pool in place, over the bus.
 * STAGED: a device copy of the two spans made on the stream at submit, so
 * the prepare kernels read HBM; the pool keeps a device mirror. */
#define VQM_CU_MEMORY_POLICY_AUTOMATIC 0
#define VQM_CU_MEMORY_POLICY_DIRECT 1
#define VQM_CU_MEMORY_POLICY_STAGED 2

/* Blur modes. SAMPLED is VQM's 13-tap sampled Gaussian, sigma 1.5
 * (pipeline.cc:274-291), the only mode that reproduces VQM's scores.
 * RECURSIVE (opt-in, no counterpart in VQM) is the third-order recursive
 * Gaussian, sigma 1.5, that Cloudinary's ssimulacra2 uses and VQM replaced
 * on purpose (docs/divergence.md:22): 9 nonzero taps of radius 4, zero
 * padded; everything else is unchanged. Its scores follow that filter's
 * FP64 evaluation, not VQM. */
#define VQM_CU_SS2_BLUR_SAMPLED 0
#define VQM_CU_SS2_BLUR_RECURSIVE 1

/* PipelineMemoryUsage (include/vqm_memory_types.h:24-33), device bytes. */
typedef struct vqm_cu_memory_usage {
    uint64_t pyramid_bytes;  /* XYB planes */
    uint64_t resident_bytes; /* upload() slots */
    uint64_t input_bytes;    /* allocate_image() pool (pinned host memory)
                                + streaming inputs (device) */
    uint64_t scratch_bytes;  /* partials, tables, counters */
    uint64_t total_bytes;
    uint64_t host_bytes;     /* of total_bytes, pinned host memory (the
                                allocate_image() pool); the rest is device
                                memory */
    uint32_t uses_staging;   /* 1: the STAGED memory policy is in force */
    uint32_t reserved;
} vqm_cu_memory_usage;

typedef struct vqm_cu_ss2_pipeline vqm_cu_ss2_pipeline;
typedef struct vqm_cu_ss2_batch vqm_cu_ss2_batch;

/* ---- library -------------------------------------------------------- */

/* Message of the last failing call on this thread ("" after success). */
const char* vqm_cu_last_error(void);
/* ABI version: (major << 16) | minor. */
uint32_t vqm_cu_version(void);

/* ---- devices (include/vqm_device.h) --------------------------------- */

/* ListDevices: the CUDA devices in ordinal order. vqm_cu_device_info fills
 * device `index`'s name (NUL-terminated, cut to name_bytes), its 16-byte
 * UUID and its kind as VQM's DeviceType (1 integrated, 2 discrete GPU). */
int vqm_cu_device_count(uint32_t* count);
int vqm_cu_device_info(uint32_t index, char* name, size_t name_bytes,
                       uint8_t* uuid16, uint32_t* type);
/* SetDefaultDevice: from now on, process-wide, a config whose device is -1
 * uses the device with this UUID (before any call, -1 is the calling
 * thread's current device). VQM_CU_INVALID_ARGUMENT for an unknown UUID. */
int vqm_cu_set_default_device(const uint8_t* uuid16);

/* ---- formats (src/input.cc) ----------------------------------------- */

/* RequiredBytes (include/vqm_image.h:360-363; src/input.cc:244-255). */
int vqm_cu_required_bytes(const vqm_cu_format* format, uint32_t width,
                          uint32_t height, size_t* bytes);
/* ValidateImage (src/input.cc:152-222): VQM_CU_INVALID_ARGUMENT with
 * "<name>: <reason>" when the format/size pair is not decodable. */
int vqm_cu_validate_format(const vqm_cu_format* format, uint32_t width,
                           uint32_t height, const char* name);
/* PlanSsimulacra2Scales (src/metrics/ssimulacra2/pipeline.cc:28-48): writes
 * up to 6 (width, height) pairs into sizes12, the count into *scales. */
int vqm_cu_ss2_plan_scales(uint32_t width, uint32_t height, uint32_t* sizes12,
                           uint32_t* scales);
/* Ssimulacra2ChannelPruned (src/metrics/ssimulacra2/score.cc:103-114): *pruned
 * = 1 when all six weights of (channel, scale) in a `scales`-level plan are
 * at most 0.01, so its norms are never computed and publish as 0. Channels
 * 0-2 are X, Y, B; scale < scales <= 6, else VQM_CU_INVALID_ARGUMENT. */
int vqm_cu_ss2_channel_pruned(uint32_t channel, uint32_t scale, uint32_t scales,
                              int* pruned);
/* The 13 blur taps (offsets -6..6) a blur mode applies along each axis, as
 * the kernels hold them: MakeGaussian's (pipeline.cc:274-291) for
 * VQM_CU_SS2_BLUR_SAMPLED, the recursive Gaussian's impulse response for
 * VQM_CU_SS2_BLUR_RECURSIVE. VQM_CU_INVALID_ARGUMENT for another mode. */
int vqm_cu_ss2_blur_taps(uint32_t blur, float* taps13);
/* Ssimulacra2Result::Score (src/metrics/ssimulacra2/score.cc:118-163), FP64,
 * norms in the layout above. VQM_CU_INVALID_ARGUMENT for more than six
 * scales or nonfinite norms, as the reference throws. */
int vqm_cu_ss2_score(const double* norms, uint32_t scales, double* score);

/* The decode constants this library derives for one format, as the 44
 * words of VQM's per-image SourceDesc (src/vulkan/vulkan_support.h:104-120,
 * built by src/vulkan/vulkan_source.cc:77-182) with plane offsets and row
 * strides left 0. For inspection and tests. */
int vqm_cu_ss2_source_constants(const vqm_cu_format* format,
                                uint32_t chroma_filter, uint32_t* words44);

/* ---- pipeline: one geometry, one pair in flight ---------------------- */
/*      (class Ssimulacra2Pipeline, include/ssimulacra2.h:83-215)          */

/* Ssimulacra2Pipeline(Ssimulacra2Config) (ssimulacra2.h:85-89): allocates
 * all device memory for the geometry. INVALID_ARGUMENT below 8x8. */
int vqm_cu_ss2_create(const vqm_cu_ss2_config* config,
                      vqm_cu_ss2_pipeline** pipeline);
/* ~Ssimulacra2Pipeline: waits for pending work, frees everything. */
int vqm_cu_ss2_destroy(vqm_cu_ss2_pipeline* pipeline);
/* The stream all of the pipeline's work is ordered on (cudaStream_t). The
 * default is a stream the pipeline owns; a caller's stream replaces it. */
int vqm_cu_ss2_set_stream(vqm_cu_ss2_pipeline* pipeline, void* stream);
int vqm_cu_ss2_get_stream(vqm_cu_ss2_pipeline* pipeline, void** stream);

/* Submit(Image/ImageView, Image/ImageView) (ssimulacra2.h:145-151) and the
 * caller-owned device buffer form of Submit(VulkanBufferView, ...)
 * (:192-195): host planes are copied to the device before this returns;
 * device planes are read in place. LOGIC_ERROR while a submission is in
 * flight. */
int vqm_cu_ss2_submit(vqm_cu_ss2_pipeline* pipeline,
                      const vqm_cu_image* original,
                      const vqm_cu_image* distorted, float background,
                      uint64_t* token);
/* Submit(UploadedImage, UploadedImage) (ssimulacra2.h:152-155). */
int vqm_cu_ss2_submit_resident(vqm_cu_ss2_pipeline* pipeline,
                               uint64_t original, uint64_t distorted,
                               float background, uint64_t* token);
/* Submit(UploadedImage, Image) (ssimulacra2.h:156-159). */
int vqm_cu_ss2_submit_resident_image(vqm_cu_ss2_pipeline* pipeline,
                                     uint64_t original,
                                     const vqm_cu_image* distorted,
                                     float background, uint64_t* token);
/* Submit(ImageBuffer, ImageBuffer) (ssimulacra2.h:181-184). */
int vqm_cu_ss2_submit_buffers(vqm_cu_ss2_pipeline* pipeline,
                              uint64_t original, uint64_t distorted,
                              float background, uint64_t* token);
/* Submit(..., VulkanSubmitSync) (ssimulacra2.h:198-201): the pipeline's
 * stream first waits for every event in wait_events; after the pair's work
 * it records every event in signal_events (cudaEvent_t, passed as void*). */
int vqm_cu_ss2_submit_sync(vqm_cu_ss2_pipeline* pipeline,
                           const vqm_cu_image* original,
                           const vqm_cu_image* distorted,
                           void* const* wait_events, uint32_t wait_count,
                           void* const* signal_events, uint32_t signal_count,
                           float background, uint64_t* token);
/* Finish(token) (ssimulacra2.h:203): waits for the pair and writes its
 * norms (18 per scale) and scale count. INVALID_ARGUMENT for an unknown or
 * already finished token. */
int vqm_cu_ss2_finish(vqm_cu_ss2_pipeline* pipeline, uint64_t token,
                      double* norms108, uint32_t* scales);
/* Compute (ssimulacra2.h:102-104) = submit + finish, plus the score. */
int vqm_cu_ss2_compute(vqm_cu_ss2_pipeline* pipeline,
                       const vqm_cu_image* original,
                       const vqm_cu_image* distorted, float background,
                       double* norms108, uint32_t* scales, double* score);

/* Upload(Image) (ssimulacra2.h:115-118): copies into a resident slot and
 * returns its handle (never 0). INVALID_ARGUMENT when every slot is used. */
int vqm_cu_ss2_upload(vqm_cu_ss2_pipeline* pipeline, const vqm_cu_image* image,
                      uint64_t* handle);
/* Release(UploadedImage) (ssimulacra2.h:119-121): unknown or released
 * handles are ignored. */
int vqm_cu_ss2_release(vqm_cu_ss2_pipeline* pipeline, uint64_t handle);
/* AllocateImage / MapImage / Release(ImageBuffer) (ssimulacra2.h:161-176):
 * spans of a pinned host pool of config.input_bytes, RequiredBytes(format)
 * long, 64-byte aligned, in vqm::Image's packed layout. *host_ptr is a host
 * address the caller writes (memcpy, as into VQM's mapped arena, or
 * cudaMemcpy with cudaMemcpyDefault); the prepare kernels read the span in
 * place over the bus (unified addressing), so nothing is copied at submit. */
int vqm_cu_ss2_allocate_image(vqm_cu_ss2_pipeline* pipeline,
                              const vqm_cu_format* format, uint64_t* handle,
                              size_t* bytes);
int vqm_cu_ss2_map_image(vqm_cu_ss2_pipeline* pipeline, uint64_t handle,
                         void** host_ptr);
int vqm_cu_ss2_release_image(vqm_cu_ss2_pipeline* pipeline, uint64_t handle);
/* GetMemoryUsage (ssimulacra2.h:204-205). */
int vqm_cu_ss2_memory_usage(vqm_cu_ss2_pipeline* pipeline,
                            vqm_cu_memory_usage* usage);
/* Diagnostic: copies the XYB plane (level, channel) of image 0 (original) or
 * 1 (distorted) written by the last finished pair into out (width_l *
 * height_l floats, row-major). INVALID_ARGUMENT for a pruned channel. */
int vqm_cu_ss2_debug_plane(vqm_cu_ss2_pipeline* pipeline, uint32_t image,
                           uint32_t level, uint32_t channel, float* out);
/* CUDA-graph replay of the pair's kernels (prepare, blur, finalize): on by
 * default; 0 launches them one by one. */
int vqm_cu_ss2_set_graphs(vqm_cu_ss2_pipeline* pipeline, int enabled);
/* The reference-pyramid reuse of VQM's pipeline (src/metrics/ssimulacra2/
 * vulkan.cc:238-243, 714-736): a submission whose original is the same
 * resident slot handle, with the same background, as the previous
 * submission's skips the original's decode and pyramid. *count receives how
 * many submissions have done so. */
int vqm_cu_ss2_reference_reuses(vqm_cu_ss2_pipeline* pipeline, uint64_t* count);
/* VulkanRuntime::pending() (src/vulkan/vulkan_runtime.h:275-285): *in_flight
 * receives 1 from a successful submit until finish takes its token, else 0.
 * VQM reports a call made while a submission is in flight before it looks at
 * the call's images; the facades check image sizes on the host, so they ask
 * this before reporting such an error. */
int vqm_cu_ss2_in_flight(const vqm_cu_ss2_pipeline* pipeline, uint32_t* in_flight);

/* ---- scoring without allocation --------------------------------------- */

/* No counterpart in the reference. For callers that cannot let a library
 * allocate device memory (their own allocator owns all of it, or a
 * cudaMalloc/cudaFree would stall their real-time streams): scores one pair
 * of device images (memory == VQM_CU_MEMORY_DEVICE) on `stream` without any
 * allocation, with all scratch in one fixed 32 MiB device array that the
 * library reserves on every GPU that loads it, held until exit. Pairs whose
 * scratch exceeds it return INVALID_ARGUMENT with the bytes they need; the
 * need grows with the padded row width, not the area alone (1920x1080,
 * 1080x1920 and 2048x1200 fit; 1200x2048 and 2560x1440 do not). Planes and
 * the result must be device or managed memory of the current device, else
 * INVALID_ARGUMENT before any kernel runs.
 * Returns once the work is queued; result_device (caller-owned device
 * memory, VQM_CU_SS2_RESULT_DOUBLES doubles) then receives 108 norms (18 per
 * scale, zero past the pair's scales), the FP64 score, the scale count and
 * a status word 0. All calls share the array and it keeps the last call's
 * contents, so calls whose work overlaps on the GPU race: serialize them.
 * The first call on a device sets up that device (symbol address lookup,
 * constant upload) and should come before any stream capture. */
#define VQM_CU_SS2_RESULT_DOUBLES 112
int vqm_cu_ss2_compute_noalloc(const vqm_cu_image* original,
                               const vqm_cu_image* distorted,
                               float background, uint32_t chroma_filter,
                               void* stream, double* result_device);

/* ---- batch: many pairs of any sizes and formats, one launch per stage --- */
/*      (Ssimulacra2Pool::ComputeMany / ScoreMany, include/vqm_pool.h:51-87) */

typedef struct vqm_cu_ss2_batch_config {
    uint64_t max_pixels;   /* largest sum of W*H over one batch's pairs */
    uint32_t max_pairs;    /* largest pair count of one batch */
    uint32_t chroma_filter;
    int32_t device;        /* CUDA ordinal; -1 = the current device */
    uint32_t tile_w, tile_h; /* blur tile (its one-tile-per-CTA kernel);
                                0 = chosen per submit */
    uint32_t variant;      /* blur kernel: 0 = by tile, or chosen per submit
                              from the tile count (a strip length of the
                              default tile; strips regroup the compensated
                              partial sums, so results agree to rounding,
                              ~1e-7 relative), k = compiled variant k - 1 */
    uint32_t half_planes;  /* 1: binary16 pyramid planes, as
                              vqm_cu_ss2_config.half_planes */
    uint32_t blur;         /* VQM_CU_SS2_BLUR_*; 0 = VQM's */
} vqm_cu_ss2_batch_config;

/* The blur kernels compiled into the library, for tuning: *count variants,
 * and for each (if `shapes` is not null) VQM_CU_SS2_VARIANT_WORDS words: its
 * tile width, tile height, threads per CTA, tiles per CTA down a column (1:
 * one tile per CTA) and 1 if its CTAs stay resident over many tiles. */
#define VQM_CU_SS2_VARIANT_WORDS 5
int vqm_cu_ss2_blur_variants(uint32_t* count, uint32_t* shapes);
/* A host-only diagnostic with no counterpart in the reference: the blur
 * variant a batch created without one takes for `n` pairs of the sizes in
 * `sizes` (width, height interleaved) on a device of `sms` SMs (the strip
 * length with the least estimated time). */
int vqm_cu_ss2_auto_blur_variant(const uint32_t* sizes, uint32_t n, uint32_t sms,
                                 uint32_t* variant);

/* A self-check with no counterpart in the reference: the prepare kernels
 * compute the XYB cube roots by a shorter route than the shared
 * correctly-rounded cube root the CPU oracle uses (an estimate from the
 * special-function unit instead of a bit-level one, so one Newton step
 * instead of three); both must give the same float. This runs both on the
 * current device for every float whose bit pattern lies in [first_bits,
 * last_bits] and reports how many differ (*mismatches) and the smallest
 * such pattern (*first_bad, 0xffffffff when none). Synchronous; allocates a
 * few bytes of device memory. */
int vqm_cu_ss2_check_cbrt(uint32_t first_bits, uint32_t last_bits,
                          uint64_t* mismatches, uint32_t* first_bad);
/* The same self-check for the blur maps' division, which takes the divisor's
 * reciprocal from the special-function unit and one Newton step where the
 * shared division takes three from a bit seed (both then correct the
 * quotient with its exact residual): for every divisor whose bit pattern
 * lies in [first_bits, last_bits] and sixteen quotient values in [-1, 1.8],
 * compares the two quotients; *mismatches counts the differing divisions,
 * *first_bad is the smallest divisor pattern among them. */
int vqm_cu_ss2_check_division(uint32_t first_bits, uint32_t last_bits,
                              uint64_t* mismatches, uint32_t* first_bad);
/* Which device decode an image of format `format` takes (a diagnostic; no
 * device is touched): VQM_CU_DECODE_GENERIC, _TABLE (8-bit grey/RGB through a
 * per-image table), _TABLE_IN_RANGE (the same, with every linear sample
 * non-negative so the cube roots need no range check) or _YUV (integer YUV
 * with a power-law transfer and at most 2x chroma subsampling, phases fixed
 * per pixel parity; an image of such a format with an odd width or height
 * runs the generic decode). The results are the same whichever path runs. */
#define VQM_CU_DECODE_GENERIC 0
#define VQM_CU_DECODE_TABLE 1
#define VQM_CU_DECODE_TABLE_IN_RANGE 2
#define VQM_CU_DECODE_YUV 3
int vqm_cu_ss2_decode_path(const vqm_cu_format* format, uint32_t chroma_filter,
                           uint32_t* path);

int vqm_cu_ss2_batch_create(const vqm_cu_ss2_batch_config* config,
                            vqm_cu_ss2_batch** batch);
int vqm_cu_ss2_batch_destroy(vqm_cu_ss2_batch* batch);
int vqm_cu_ss2_batch_set_stream(vqm_cu_ss2_batch* batch, void* stream);
/* Submits n pairs (host or device images; sizes may differ per pair, the
 * two images of a pair must match). Host planes are copied before return. */
int vqm_cu_ss2_batch_submit(vqm_cu_ss2_batch* batch, uint32_t n,
                            const vqm_cu_image* originals,
                            const vqm_cu_image* distorteds, float background,
                            uint64_t* token);
/* As vqm_cu_ss2_batch_submit, but host planes are copied asynchronously and
 * stay borrowed until vqm_cu_ss2_batch_finish returns (no reference
 * counterpart: VQM copies host pixels before Submit returns). A caller that
 * keeps its images alive anyway, such as a pool scoring a list, lets the
 * next submission's copies queue behind these ones. */
int vqm_cu_ss2_batch_submit_borrowed(vqm_cu_ss2_batch* batch, uint32_t n,
                                     const vqm_cu_image* originals,
                                     const vqm_cu_image* distorteds,
                                     float background, uint64_t* token);
/* Waits and writes norms (n x 108, zero beyond each pair's scales), scale
 * counts and scores (FP64, computed on the device). */
int vqm_cu_ss2_batch_finish(vqm_cu_ss2_batch* batch, uint64_t token,
                            double* norms, uint32_t* scales, double* scores);
/* Opt-in stage timing, the CUDA counterpart of VQM's VQM_STAGE_TIMING
 * (src/timing.h:18-112): CUDA events recorded on the batch's stream around
 * the prepare, blur and finalize launches. After batch_finish, stage_ms3
 * holds the last batch's device milliseconds of each stage. */
int vqm_cu_ss2_batch_set_timing(vqm_cu_ss2_batch* batch, int enabled);
int vqm_cu_ss2_batch_stage_ms(vqm_cu_ss2_batch* batch, float* stage_ms3);
/* The batch's device memory, after PipelineMemoryUsage::total
 * (include/vqm_memory_types.h:24-33): *held = the bytes it holds now
 * (pyramid, tables, partials, counters, its copy of host inputs), reused from
 * submit to submit and never shrunk by a submit. batch_device_bytes_after
 * validates a submission as batch_submit would and gives what the batch
 * will hold once it is submitted (its buffers grown as the submit grows
 * them), allocating nothing. batch_trim frees the memory of an idle batch
 * (VQM_CU_LOGIC_ERROR while one is in flight); its next submit allocates
 * again. */
int vqm_cu_ss2_batch_device_bytes(vqm_cu_ss2_batch* batch, uint64_t* held);
int vqm_cu_ss2_batch_device_bytes_after(vqm_cu_ss2_batch* batch, uint32_t n,
                                        const vqm_cu_image* originals,
                                        const vqm_cu_image* distorteds,
                                        uint64_t* bytes);
int vqm_cu_ss2_batch_trim(vqm_cu_ss2_batch* batch);
/* ComputeMany / ScoreMany = submit + finish. */
int vqm_cu_ss2_batch_compute(vqm_cu_ss2_batch* batch, uint32_t n,
                             const vqm_cu_image* originals,
                             const vqm_cu_image* distorteds, float background,
                             double* norms, uint32_t* scales, double* scores);

/* ------------------------------------------------------------------------ */
/*      Serving loop (no reference counterpart: VQM scores synchronously    */
/*      per caller; this is continuous batching for request streams)       */
/* ------------------------------------------------------------------------ */

/* A wait that ran out; the request is still pending. */
#define VQM_CU_TIMEOUT 5

typedef struct vqm_cu_ss2_server vqm_cu_ss2_server;

typedef struct vqm_cu_ss2_server_config {
    uint64_t memory_budget;  /* device bytes for admitted work; 0 = 40 GiB */
    uint32_t workers;        /* batch scorers in flight at once; 0 = 2 */
    uint32_t max_batch_pairs;/* pairs per launch at most; 0 = 64 */
    uint32_t chroma_filter;  /* 0 bilinear, 1 bicubic, 2 lanczos */
    int32_t device;          /* CUDA ordinal; -1 = the current device */
    uint32_t variant;        /* blur kernel, as vqm_cu_ss2_batch_config */
    uint32_t blur;           /* VQM_CU_SS2_BLUR_*; 0 = VQM's */
} vqm_cu_ss2_server_config;

typedef struct vqm_cu_ss2_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t batches;          /* batch launches (prepare, blur) */
    uint64_t largest_batch;    /* pairs in the largest batch formed */
    uint64_t bytes_in_flight;  /* device bytes the admitted, not yet
                                  completed requests need */
    uint64_t peak_bytes;       /* largest bytes_in_flight seen */
    uint64_t queued;           /* submitted, not yet in a batch */
    uint64_t budget_bytes;     /* the cap in force (see server_create) */
    uint64_t device_bytes;     /* device memory the workers hold now */
    uint64_t peak_device_bytes;/* largest device_bytes seen */
    uint64_t trims;            /* idle workers' memory freed to admit work */
} vqm_cu_ss2_server_stats;

/* Starts a dispatcher thread, which forms batches from the queued requests
 * in arrival order whenever a worker is free, and a completion thread, which
 * finishes batches in submission order. Each worker is a batch scorer with
 * its own stream and device memory, reused from batch to batch. The budget
 * caps the device memory all workers hold together, counted as allocated
 * (with the buffers' growth): a batch is formed only while the bytes its
 * worker will hold, plus what the other workers hold, stay within it; when
 * the head request does not fit, idle workers' memory is freed first, and
 * otherwise the request waits for running batches to finish. So a request
 * up to the whole budget is admitted once the rest of the server is idle.
 * The cap in force is memory_budget, lowered at creation to the device's
 * free memory less 256 MiB when that is smaller. */
int vqm_cu_ss2_server_create(const vqm_cu_ss2_server_config* config,
                             vqm_cu_ss2_server** server);
/* Finishes every queued and in-flight request, then stops the threads. */
int vqm_cu_ss2_server_destroy(vqm_cu_ss2_server* server);
/* Queues one pair (host or device images, validated here). The images'
 * memory must stay valid and unchanged until the request's wait returns.
 * VQM_CU_INVALID_ARGUMENT if the pair alone needs more than the budget. */
int vqm_cu_ss2_server_submit(vqm_cu_ss2_server* server,
                             const vqm_cu_image* original,
                             const vqm_cu_image* distorted, float background,
                             uint64_t* ticket);
/* Waits up to timeout_ms (negative: no limit) and writes the pair's norms
 * (108, zero beyond its scales), scale count, score and latency from submit
 * to completion in milliseconds (any output may be null); the ticket is
 * then released. VQM_CU_TIMEOUT leaves the request pending. A request whose
 * batch failed returns that failure's status and message. */
int vqm_cu_ss2_server_wait(vqm_cu_ss2_server* server, uint64_t ticket,
                           int32_t timeout_ms, double* norms108,
                           uint32_t* scales, double* score,
                           double* latency_ms);
int vqm_cu_ss2_server_get_stats(vqm_cu_ss2_server* server,
                            vqm_cu_ss2_server_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* VQM_CU_SS2_H_ */
