// C entry points over the reference's independent FP64 input-conversion
// reference, tests/input/input_reference.h of the reference checkout --
// TEST INFRASTRUCTURE ONLY.
//
// input_reference.h is the reference's own double-precision model of the
// input surface, written from the standards (transfer curves, YUV matrices,
// primaries and gamut, constant luminance, ICtCp, zimg's chroma resampler)
// rather than from the shader code. The reference's input-format tests
// (tests/input/input_format_test.cc:208-433, input_format_chroma_test.cc:
// 104-430) build one frame of each A/B pair from it. Built by
// oracle/Makefile (target `ref`) into oracle/_ref/libvqm_ref.so beside
// ref_shim.cc; these functions only call the header's inline functions and
// flatten their results into plain arrays for ctypes. Enum arguments are the
// reference's numeric values (include/vqm_image.h).

#include <cstddef>
#include <cstdint>

#include "input_reference.h"

namespace {
namespace r = vqm::test::ref;

void Put(const r::Mat3& m, double* out9) {
    for (int i = 0; i < 9; ++i) out9[i] = m[static_cast<std::size_t>(i)];
}
}  // namespace

extern "C" {

// ref::DecodeTransfer: zimg's display-referred to_linear of one value.
double vqmin_decode_transfer(int transfer, double v) {
    return r::DecodeTransfer(static_cast<vqm::TransferCharacteristics>(transfer), v);
}

// ref::HlgToLinear: per-channel inverse OETF, luminance OOTF, peak factor.
void vqmin_hlg_to_linear(const double* v3, double kr, double kg, double kb, double scale,
                         double* out3) {
    const r::Vec3 o = r::HlgToLinear({v3[0], v3[1], v3[2]}, kr, kg, kb, scale);
    for (int i = 0; i < 3; ++i) out3[i] = o[static_cast<std::size_t>(i)];
}

// ref::NclToRgb: encoded YUV -> encoded RGB for a matrix-coefficients value.
void vqmin_ncl_to_rgb(int matrix, double* out9) {
    Put(r::NclToRgb(static_cast<vqm::MatrixCoefficients>(matrix)), out9);
}

// ref::NclToRgbFromPrimaries: the chromaticity-derived matrix.
void vqmin_ncl_to_rgb_from_primaries(int primaries, double* out9) {
    Put(r::NclToRgbFromPrimaries(static_cast<vqm::ColorPrimaries>(primaries)), out9);
}

// ref::Gamut: linear RGB in `from` primaries -> linear RGB in `to` primaries.
void vqmin_gamut(int from, int to, double* out9) {
    Put(r::Gamut(static_cast<vqm::ColorPrimaries>(from), static_cast<vqm::ColorPrimaries>(to)),
        out9);
}

// ref::YuvConstantsFromPrimaries: Kr, Kb from the chromaticities (H.265 E-22..27).
void vqmin_yuv_constants_from_primaries(int primaries, double* kr, double* kb) {
    r::YuvConstantsFromPrimaries(static_cast<vqm::ColorPrimaries>(primaries), *kr, *kb);
}

// ref::ClToRgb: constant-luminance Y'CbCr -> linear RGB.
void vqmin_cl_to_rgb(double kr, double kb, const double* yuv3, double* out3) {
    const r::Vec3 o = r::ClToRgb(kr, kb, {yuv3[0], yuv3[1], yuv3[2]});
    for (int i = 0; i < 3; ++i) out3[i] = o[static_cast<std::size_t>(i)];
}

// ref::IctCpToLms and ref::LmsToRgb (BT.2100).
void vqmin_ictcp_to_lms(int transfer, double* out9) {
    Put(r::IctCpToLms(static_cast<vqm::TransferCharacteristics>(transfer)), out9);
}
void vqmin_lms_to_rgb(double* out9) { Put(r::LmsToRgb(), out9); }

// ref::AxisTaps: the resampler's (mirrored index, weight) taps of one output
// position; writes at most `capacity` of them and returns how many there are.
int vqmin_axis_taps(int filter, uint32_t out_pos, double scale, double shift, uint32_t dim,
                    uint32_t* index, double* weight, int capacity) {
    const auto taps = r::AxisTaps(static_cast<vqm::ChromaFilter>(filter), out_pos, scale, shift,
                                  dim);
    const int n = static_cast<int>(taps.size());
    for (int i = 0; i < n && i < capacity; ++i) {
        index[i] = static_cast<uint32_t>(taps[static_cast<std::size_t>(i)].first);
        weight[i] = taps[static_cast<std::size_t>(i)].second;
    }
    return n;
}

// ref::ChromaShift: the chroma phase of a siting along one axis.
double vqmin_chroma_shift(int location, int horizontal, uint32_t subsample) {
    return r::ChromaShift(static_cast<vqm::ChromaLocation>(location), horizontal != 0, subsample);
}

}  // extern "C"
