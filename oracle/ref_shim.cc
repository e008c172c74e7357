// C entry points over the reference's own host code, for pinning the oracle
// and the CUDA scorer's host constants -- TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/Makefile (target `ref`) together with the reference's
// src/metrics/ssimulacra2/score.cc and src/input.cc, compiled unmodified from
// the reference checkout into oracle/_ref/libvqm_ref.so. Nothing here is a
// copy of reference code: these functions only call it and flatten its C++
// types into plain arrays so Python tests can read them through ctypes.
//
// What stays out: the shaders (GLSL, no compiler here) and vulkan_source.cc,
// whose header pulls in <vulkan/vulkan.h>; the descriptor assembly it performs
// is recomposed below from the input.cc functions it calls
// (src/vulkan/vulkan_source.cc:77-182).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "input.h"
#include "metrics/ssimulacra2/ssimulacra2_internal.h"
#include "ssimulacra2.h"

namespace {
thread_local std::string g_error;

vqm::ImageFormat ToFormat(const uint8_t* f) {
    vqm::ImageFormat out;
    out.type = static_cast<vqm::PixelType>(f[0]);
    out.family = static_cast<vqm::ColorFamily>(f[1]);
    out.alpha = static_cast<vqm::AlphaType>(f[2]);
    out.range = static_cast<vqm::PixelRange>(f[3]);
    out.matrix = static_cast<vqm::MatrixCoefficients>(f[4]);
    out.transfer = static_cast<vqm::TransferCharacteristics>(f[5]);
    out.primaries = static_cast<vqm::ColorPrimaries>(f[6]);
    out.chroma_location = static_cast<vqm::ChromaLocation>(f[7]);
    out.subsample_w = f[8];
    out.subsample_h = f[9];
    out.depth = f[10];
    return out;
}

void PutF(uint32_t* words, int i, double v) {
    const float f = static_cast<float>(v);
    std::memcpy(&words[i], &f, 4);
}
}  // namespace

extern "C" {

const char* vqmref_last_error(void) { return g_error.c_str(); }

// Ssimulacra2Result::Score (score.cc:118-163). Returns 0 on success, 1 when
// Score() throws std::invalid_argument.
int vqmref_score(const double* norms, uint32_t scales, double* score) {
    vqm::Ssimulacra2Result r;
    r.scales.resize(scales);
    for (uint32_t s = 0; s < scales; ++s) {
        for (int k = 0; k < 6; ++k) r.scales[s].avg_ssim[k] = norms[s * 18 + k];
        for (int k = 0; k < 12; ++k)
            r.scales[s].avg_edgediff[k] = norms[s * 18 + 6 + k];
    }
    try {
        *score = r.Score();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        return 1;
    }
}

int vqmref_channel_pruned(uint32_t c, uint32_t s, uint32_t scales) {
    return vqm::internal::Ssimulacra2ChannelPruned(c, s, scales) ? 1 : 0;
}

// RequiredBytes (input.cc:244-255); 1 on std::invalid_argument.
int vqmref_required_bytes(const uint8_t* f, uint32_t w, uint32_t h, size_t* out) {
    try {
        *out = vqm::RequiredBytes(ToFormat(f), {w, h});
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// ValidateImage (input.cc:152-222); 0 when valid, 1 with the message.
int vqmref_validate(const uint8_t* f, uint32_t w, uint32_t h) {
    try {
        vqm::internal::ValidateImage(ToFormat(f), {w, h}, "image");
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// The 44 descriptor words (plane offsets and row strides left zero) recomposed
// from input.cc exactly as vulkan_source.cc:77-182 combines them.
int vqmref_source_desc(const uint8_t* fbytes, uint32_t chroma_filter,
                       uint32_t* words) {
    using namespace vqm;
    using namespace vqm::internal;
    try {
        const ImageFormat f = ToFormat(fbytes);
        std::memset(words, 0, 44 * 4);
        const OpMode mode = SelectMode(f);
        const TransferDecode transfer = SelectTransfer(f.transfer);
        const bool grey = f.family == ColorFamily::Grey;
        const bool sub = f.family == ColorFamily::Yuv &&
                         (f.subsample_w != 0 || f.subsample_h != 0);
        words[4] = uint32_t(f.type) | (uint32_t(f.family) << 2) |
                   (uint32_t(f.alpha) << 4) | (uint32_t(f.subsample_w) << 6) |
                   (uint32_t(f.subsample_h) << 8) | (uint32_t(transfer.id) << 10) |
                   (chroma_filter << 15) | (uint32_t(mode) << 17);
        const ScaleOffset luma = PlaneScaleOffset(f, false, false);
        const ScaleOffset chroma =
            PlaneScaleOffset(f, f.family == ColorFamily::Yuv, false);
        const ScaleOffset alpha = PlaneScaleOffset(f, false, true);
        PutF(words, 6, luma.scale);
        PutF(words, 7, chroma.scale);
        PutF(words, 8, alpha.scale);
        PutF(words, 9, luma.offset);
        PutF(words, 10, chroma.offset);
        PutF(words, 11, alpha.offset);
        uint32_t flags = 0;
        Matrix3 m1{1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (mode == OpMode::ConstantLuminance) {
            flags |= 1u;
        } else if (mode == OpMode::ICtCp) {
            m1 = IctCpToLmsMatrix(f.transfer);
        } else {
            bool identity = false;
            m1 = NclToRgbMatrix(f, identity);
            if (identity) flags |= 1u;
        }
        Matrix3 m2{1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (grey || f.primaries == ColorPrimaries::Bt709) {
            flags |= 2u;
        } else if (mode == OpMode::ICtCp) {
            m2 = Multiply(GamutMatrix(f.primaries, ColorPrimaries::Bt709),
                          LmsToRgbMatrix());
        } else {
            m2 = GamutMatrix(f.primaries, ColorPrimaries::Bt709);
        }
        for (int i = 0; i < 9; ++i) {
            PutF(words, 12 + i, m1[i]);
            PutF(words, 21 + i, m2[i]);
        }
        double kr = 0, kg = 1, kb = 0;
        LumaCoefficients(f, kr, kg, kb);
        PutF(words, 30, kr);
        PutF(words, 31, kg);
        PutF(words, 32, kb);
        PutF(words, 33, transfer.to_linear_scale);
        words[5] = flags;
        // Chroma siting is the one piece of vulkan_source.cc with no input.cc
        // counterpart; the tests compare it separately against the formula.
        (void)sub;
        if (mode == OpMode::ConstantLuminance) {
            const auto cl = ConstantLuminanceConstants(kr, kb);
            for (int i = 0; i < 4; ++i) std::memcpy(&words[36 + i], &cl[i], 4);
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

}  // extern "C"
