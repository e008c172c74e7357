// Host-side pieces of the scorer that do not touch the device: image format
// rules and decode constants (restating src/input.cc and
// src/vulkan/vulkan_source.cc), the scale plan and pruning mask
// (src/metrics/ssimulacra2/pipeline.cc, score.cc) and the FP64 score.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/vqm_cu_ss2.h"
#include "ss2_device.cuh"

namespace vqm_b200 {

constexpr uint32_t kMinDimension = 8;

struct PlaneGeometry {
    size_t width = 0, height = 0, sample_bytes = 0, offset = 0;
    bool present() const { return sample_bytes != 0; }
};

// input.cc:114-145: plane sizes and packed offsets, each plane 4-byte aligned.
std::array<PlaneGeometry, 4> PlaneLayout(const vqm_cu_format& f, uint32_t w, uint32_t h);
// input.cc:244-255.
size_t RequiredBytes(const vqm_cu_format& f, uint32_t w, uint32_t h);
// input.cc:152-222: throws std::invalid_argument("<name>: <reason>").
void ValidateFormat(const vqm_cu_format& f, uint32_t w, uint32_t h, const char* name);

// vulkan_source.cc:77-182 plus the per-image table of the 8-bit fast path.
// Plane pointers, strides and plane sizes are filled by the caller.
void BuildSourceConstants(const vqm_cu_format& f, uint32_t chroma_filter, float background,
                          DevSource& out);

struct ScalePlan {
    int count = 0;
    uint32_t w[kMaxLevels] = {}, h[kMaxLevels] = {};
    uint32_t mask[kMaxLevels] = {};  // kept channels per level (bit c)
};
// pipeline.cc:28-48 and the pruning mask of vulkan.cc:380-410 / score.cc:103-114.
ScalePlan PlanScales(uint32_t width, uint32_t height);
bool ChannelPruned(int channel, int scale, int scales);

// pipeline.cc:274-291: 13 taps, sigma 1.5, normalised in double, as float.
std::array<float, kTaps> GaussianTaps();
// The impulse response of the third-order recursive Gaussian (sigma 1.5) of
// Cloudinary's ssimulacra2, centred in 13 taps (the outer four are 0); see
// ss2_host.cc.
std::array<float, kTaps> RecursiveGaussianTaps();
// The taps of a vqm_cu_ss2 blur mode (VQM_CU_SS2_BLUR_*); throws
// std::invalid_argument for an unknown mode.
std::array<float, kTaps> BlurTaps(uint32_t blur);
// score.cc:38-87 as a flat 108-double table.
const double* ScoreWeights();
// score.cc:118-163; throws std::invalid_argument like the reference.
double Score(const double* norms, int scales);

// Sets the calling thread's vqm_cu_last_error() message.
void SetLastErrorMessage(const char* message);
// A config's device ordinal: `requested` when >= 0, else the default device
// vqm_cu_set_default_device chose, else the thread's current device.
int ResolveDeviceOrdinal(int32_t requested);

}  // namespace vqm_b200
