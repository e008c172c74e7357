// CPU oracle for the SSIMULACRA 2.1 scorer -- TEST INFRASTRUCTURE ONLY.
//
// A restatement of VQM's SSIMULACRA 2.1 arithmetic (GreatValueCreamSoda/vqm),
// written for the CPU and templated on the arithmetic type:
//   * float  -- the FP32 restatement, following VQM's operation order where
//               the order decides the rounding: ascending 13-tap sums with the
//               first tap a rounded product and the rest fused multiply-adds,
//               the difference-form SSIM map, zero padding, the box-average
//               association order, pruning, and the per-tile reduction ladder
//               of scale.comp / reduce.comp. It is the proxy for VQM's own
//               scores (VQM itself needs a Vulkan device and cannot run here).
//   * double -- the same algorithm in FP64, used to state each score's error.
//
// Every function cites the reference file:line it follows. Multiply-adds that
// a GPU shader compiler contracts into one rounding are written as std::fma so
// the FP32 path rounds like the device code it stands in for.
//
// The tests, the smoke check and the CPU-baseline leg of the benchmark are the
// only callers; the CUDA scorer never links or calls this library.

#include "ss2_oracle.h"

// pow, cube root, exp and sin(pi x) of the FP32 path: the deterministic
// functions the CUDA kernels evaluate too (pinned to double-precision libm by
// tests/test_detmath.py). The FP64 path uses libm itself.
#include "../vqm_b200/csrc/ss2_detmath.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_error;

// ---------------------------------------------------------------------------
// Constants of the metric.
// ---------------------------------------------------------------------------

constexpr int kChannels = 3;
constexpr int kMaxScales = 6;    // ssimulacra2_internal.h:18-22
constexpr uint32_t kMinDim = 8;  // ssimulacra2_internal.h:20-21
constexpr int kTaps = 13;        // radius ceil(3.5 * 1.5) = 6
constexpr int kRadius = 6;

// score.cc:18-24.
constexpr double kScoreScale = 0.9562382616834844;
constexpr double kScoreLinear = 2.326765642916932;
constexpr double kScoreQuadratic = 0.020884521182843837;
constexpr double kScoreCubic = 6.248496625763138e-05;
constexpr double kScoreExponent = 0.6276336467831387;

// score.cc:38-87: one row per (channel, scale) as the flat run Score() reads;
// columns ssim_1, ring_1, blur_1, ssim_4, ring_4, blur_4.
constexpr double kWeights[18][6] = {
    {0.0, 0.0007376606707406586, 0.0, 0.0, 0.0007793481682867309, 0.0},
    {0.0, 0.0004371155730107379, 0.0, 1.1041726426657346, 0.00066284834129271,
     0.00015231632783718752},
    {0.0, 0.0016406437456599754, 0.0, 1.8422455520539298, 11.441172603757666,
     0.0},
    {0.0007989109436015163, 0.000176816438078653, 0.0, 1.8787594979546387,
     10.94906990605142, 0.0},
    {0.0007289346991508072, 0.9677937080626833, 0.0, 0.00014003424285435884,
     0.9981766977854967, 0.00031949755934435053},
    {0.0004550992113792063, 0.0, 0.0, 0.0013648766163243398, 0.0, 0.0},
    {0.0, 0.0, 0.0, 7.466890328078848, 0.0, 17.445833984131262},
    {0.0006235601634041466, 0.0, 0.0, 6.683678146179332,
     0.00037724407979611296, 1.027889937768264},
    {225.20515300849274, 0.0, 0.0, 19.213238186143016, 0.0011401524586618361,
     0.001237755635509985},
    {176.39317598450694, 0.0, 0.0, 24.43300999870476, 0.28520802612117757,
     0.0004485436923833408},
    {0.0, 0.0, 0.0, 34.77906344483772, 44.835625328877896, 0.0},
    {0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0008680556573291698, 0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0005313191874358747, 0.0, 0.00016533814161379112, 0.0, 0.0},
    {0.0, 0.0, 0.0, 0.0004179171803251336, 0.0017290828234722833, 0.0},
    {0.0020827005846636437, 0.0, 0.0, 8.826982764996862, 23.19243343998926,
     0.0},
    {95.1080498811086, 0.9863978034400682, 0.9834382792465353,
     0.0012286405048278493, 171.2667255897307, 0.9807858872435379},
    {0.0, 0.0, 0.0, 0.0005130064588990679, 0.0, 0.00010854057858411537},
};
constexpr double kWeightPruning = 0.01;  // score.cc:97

struct Size {
    uint32_t w = 0, h = 0;
};

struct Plan {
    int count = 0;
    Size sizes[kMaxScales];
};

// pipeline.cc:28-48: the previous level decides whether the next is emitted;
// the next level is ceil(w/2) x ceil(h/2).
Plan PlanScales(uint32_t width, uint32_t height) {
    if (width < kMinDim || height < kMinDim)
        throw std::invalid_argument("minimum image size is 8x8 pixels");
    Plan plan;
    uint32_t w = width, h = height;
    while (plan.count < kMaxScales && w >= kMinDim && h >= kMinDim) {
        if (plan.count != 0) {
            w = w / 2 + w % 2;
            h = h / 2 + h % 2;
        }
        plan.sizes[plan.count++] = {w, h};
    }
    return plan;
}

// score.cc:103-114: a (channel, scale) pair is pruned when its six weights of
// the flat row channel * scales + scale are all at most 0.01.
bool ChannelPruned(int channel, int scale, int scales) {
    if (channel >= kChannels || scale >= scales || scales > kMaxScales)
        return false;
    const double* w = kWeights[channel * scales + scale];
    double m = w[0];
    for (int i = 1; i < 6; ++i) m = std::max(m, w[i]);
    return m <= kWeightPruning;
}

// pipeline.cc:274-291: sampled Gaussian, normalised in double, cast to float.
std::array<double, kTaps> GaussianDouble() {
    std::array<double, kTaps> w{};
    double sum = 0.0;
    for (int i = 0; i < kTaps; ++i) {
        const double offset = static_cast<double>(i) - kRadius;
        w[i] = std::exp(-0.5 * (offset / 1.5) * (offset / 1.5));
        sum += w[i];
    }
    for (int i = 0; i < kTaps; ++i) w[i] /= sum;
    return w;
}

// score.cc:118-163.
double Score(const double* norms, int scales) {
    if (scales > kMaxScales)
        throw std::invalid_argument("Ssimulacra2Result has too many scales");
    double error = 0.0;
    for (int c = 0; c < kChannels; ++c) {
        for (int s = 0; s < scales; ++s) {
            const double* w = kWeights[c * scales + s];
            const double* ssim = norms + s * 18;
            const double* edge = norms + s * 18 + 6;
            error += w[0] * std::abs(ssim[c * 2 + 0]);
            error += w[1] * std::abs(edge[c * 4 + 0]);
            error += w[2] * std::abs(edge[c * 4 + 2]);
            error += w[3] * std::abs(ssim[c * 2 + 1]);
            error += w[4] * std::abs(edge[c * 4 + 1]);
            error += w[5] * std::abs(edge[c * 4 + 3]);
        }
    }
    if (!std::isfinite(error))
        throw std::invalid_argument(
            "Ssimulacra2Result contains nonfinite or overflowing norms");
    const double scaled = error * kScoreScale;
    const double mapped = kScoreLinear * scaled -
                          kScoreQuadratic * scaled * scaled +
                          kScoreCubic * scaled * scaled * scaled;
    if (!std::isfinite(mapped))
        throw std::invalid_argument("Ssimulacra2Result score mapping overflowed");
    if (mapped > 0.0) return 100.0 - 10.0 * std::pow(mapped, kScoreExponent);
    return 100.0;
}

// ---------------------------------------------------------------------------
// Input formats: layout and decode constants (input.cc, vulkan_source.cc).
// ---------------------------------------------------------------------------

using Matrix3 = std::array<double, 9>;
using Vec3d = std::array<double, 3>;

size_t SampleBytes(uint8_t type) {
    switch (type) {
        case 0: return 1;
        case 1: case 2: return 2;
        case 3: return 4;
    }
    return 0;
}
int TypeDepth(uint8_t type) {
    switch (type) {
        case 0: return 8;
        case 1: case 2: return 16;
        case 3: return 32;
    }
    return 0;
}
int EffectiveDepth(const ss2o_format& f) {
    return f.depth != 0 ? f.depth : TypeDepth(f.type);
}

struct PlaneGeom {
    size_t width = 0, height = 0, sample_bytes = 0, offset = 0;
};

// input.cc:114-145: planes in zimg order, each starting on a 4-byte boundary.
std::array<PlaneGeom, 4> PlaneLayout(const ss2o_format& f, uint32_t w,
                                     uint32_t h) {
    std::array<PlaneGeom, 4> layout{};
    const size_t sb = SampleBytes(f.type);
    if (sb == 0) throw std::invalid_argument("invalid pixel type");
    if (f.subsample_w > 2 || f.subsample_h > 2)
        throw std::invalid_argument("subsampling greater than 4x is not supported");
    size_t cursor = 0;
    for (int p = 0; p < 4; ++p) {
        const bool chroma = p == 1 || p == 2;
        const bool present = p == 0 || (chroma && f.family != 0) ||
                             (p == 3 && f.alpha != 0);
        if (!present) continue;
        layout[p].width = chroma ? (w >> f.subsample_w) : w;
        layout[p].height = chroma ? (h >> f.subsample_h) : h;
        layout[p].sample_bytes = sb;
        layout[p].offset = cursor;
        cursor = (cursor + layout[p].width * layout[p].height * sb + 3) / 4 * 4;
    }
    return layout;
}

// input.cc:244-255.
size_t RequiredBytes(const ss2o_format& f, uint32_t w, uint32_t h) {
    const auto layout = PlaneLayout(f, w, h);
    size_t total = 0;
    for (const auto& p : layout)
        if (p.sample_bytes) total = p.offset + p.width * p.height * p.sample_bytes;
    return (total + 3) / 4 * 4;
}

// zimg's colorimetry as VQM transliterates it (input.cc:262-587). The double
// arithmetic below keeps input.cc's operation order so the constants it
// produces are bit-identical (the tests compare them against input.cc itself).
double Det2(double a00, double a01, double a10, double a11) {
    return a00 * a11 - a01 * a10;
}
Matrix3 Inverse(const Matrix3& m) {
    double det = 0.0;
    det += m[0] * Det2(m[4], m[5], m[7], m[8]);
    det -= m[1] * Det2(m[3], m[5], m[6], m[8]);
    det += m[2] * Det2(m[3], m[4], m[6], m[7]);
    return {Det2(m[4], m[5], m[7], m[8]) / det, Det2(m[2], m[1], m[8], m[7]) / det,
            Det2(m[1], m[2], m[4], m[5]) / det, Det2(m[5], m[3], m[8], m[6]) / det,
            Det2(m[0], m[2], m[6], m[8]) / det, Det2(m[2], m[0], m[5], m[3]) / det,
            Det2(m[3], m[4], m[6], m[7]) / det, Det2(m[1], m[0], m[7], m[6]) / det,
            Det2(m[0], m[1], m[3], m[4]) / det};
}
Matrix3 Multiply(const Matrix3& a, const Matrix3& b) {
    Matrix3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 3; ++k) acc += a[i * 3 + k] * b[k * 3 + j];
            r[i * 3 + j] = acc;
        }
    return r;
}
Vec3d MulV(const Matrix3& m, const Vec3d& v) {
    return {m[0] * v[0] + m[1] * v[1] + m[2] * v[2],
            m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
            m[6] * v[0] + m[7] * v[1] + m[8] * v[2]};
}
double Dot(const Vec3d& a, const Vec3d& b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
Vec3d Cross(const Vec3d& a, const Vec3d& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
            a[0] * b[1] - a[1] * b[0]};
}
Matrix3 Identity() { return {1, 0, 0, 0, 1, 0, 0, 0, 1}; }
Vec3d XyToXyz(double x, double y) { return {x / y, 1.0, (1.0 - x - y) / y}; }

// Chromaticities of the primaries (zimg colorspace_param.h).
bool PrimariesXy(uint8_t p, double xy[3][2]) {
    static const double k470M[3][2] = {{0.670, 0.330}, {0.210, 0.710}, {0.140, 0.080}};
    static const double k470Bg[3][2] = {{0.640, 0.330}, {0.290, 0.600}, {0.150, 0.060}};
    static const double kSmpteC[3][2] = {{0.630, 0.340}, {0.310, 0.595}, {0.155, 0.070}};
    static const double k709[3][2] = {{0.640, 0.330}, {0.300, 0.600}, {0.150, 0.060}};
    static const double kFilm[3][2] = {{0.681, 0.319}, {0.243, 0.692}, {0.145, 0.049}};
    static const double k2020[3][2] = {{0.708, 0.292}, {0.170, 0.797}, {0.131, 0.046}};
    static const double kP3[3][2] = {{0.680, 0.320}, {0.265, 0.690}, {0.150, 0.060}};
    static const double kEbu[3][2] = {{0.630, 0.340}, {0.295, 0.605}, {0.155, 0.077}};
    const double(*src)[2] = nullptr;
    switch (p) {
        case 4: src = k470M; break;
        case 5: src = k470Bg; break;
        case 6: case 7: src = kSmpteC; break;
        case 1: src = k709; break;
        case 8: src = kFilm; break;
        case 9: src = k2020; break;
        case 11: case 12: src = kP3; break;
        case 22: src = kEbu; break;
        default: return false;
    }
    std::memcpy(xy, src, sizeof(double) * 6);
    return true;
}
Vec3d WhitePoint(uint8_t p) {
    switch (p) {
        case 4: case 8: return XyToXyz(0.31, 0.316);          // C
        case 10: return XyToXyz(1.0 / 3.0, 1.0 / 3.0);        // E
        case 11: return XyToXyz(0.314, 0.351);                // DCI
        default: return XyToXyz(0.3127, 0.3290);              // D65
    }
}
Matrix3 PrimariesXyz(uint8_t p) {
    double xy[3][2];
    if (!PrimariesXy(p, xy))
        throw std::invalid_argument("color primaries do not define chromaticities");
    const Vec3d r = XyToXyz(xy[0][0], xy[0][1]);
    const Vec3d g = XyToXyz(xy[1][0], xy[1][1]);
    const Vec3d b = XyToXyz(xy[2][0], xy[2][1]);
    return {r[0], g[0], b[0], r[1], g[1], b[1], r[2], g[2], b[2]};
}
void YuvConstantsFromPrimaries(uint8_t p, double& kr, double& kb) {
    if (p == 1) { kr = 0.2126; kb = 0.0722; return; }
    if (p == 9) { kr = 0.2627; kb = 0.0593; return; }
    double xy[3][2];
    if (!PrimariesXy(p, xy))
        throw std::invalid_argument("color primaries do not define chromaticities");
    const Vec3d r = XyToXyz(xy[0][0], xy[0][1]);
    const Vec3d g = XyToXyz(xy[1][0], xy[1][1]);
    const Vec3d b = XyToXyz(xy[2][0], xy[2][1]);
    const Vec3d white = WhitePoint(p);
    const Vec3d xr = {r[0], g[0], b[0]}, yr = {r[1], g[1], b[1]},
                zr = {r[2], g[2], b[2]};
    const double den = Dot(xr, Cross(yr, zr));
    kr = Dot(white, Cross(g, b)) / den;
    kb = Dot(white, Cross(r, g)) / den;
}
Matrix3 RgbToYuvFromKrKb(double kr, double kb) {
    const double kg = 1.0 - kr - kb;
    const double us = 1.0 / (2.0 - 2.0 * kb);
    const double vs = 1.0 / (2.0 - 2.0 * kr);
    return {kr, kg, kb, -kr * us, -kg * us, (1.0 - kb) * us,
            (1.0 - kr) * vs, -kg * vs, -kb * vs};
}
void YuvConstants(uint8_t m, double& kr, double& kb) {
    switch (m) {
        case 4: kr = 0.3; kb = 0.11; return;
        case 7: kr = 0.212; kb = 0.087; return;
        case 5: case 6: kr = 0.299; kb = 0.114; return;
        case 1: kr = 0.2126; kb = 0.0722; return;
        case 9: case 10: kr = 0.2627; kb = 0.0593; return;
    }
    throw std::invalid_argument("matrix coefficients have no luma weights");
}
Matrix3 RgbToYuvMatrix(uint8_t m) {
    if (m == 8) return {0.25, 0.5, 0.25, -0.25, 0.5, -0.25, 0.5, 0.0, -0.5};
    if (m == 14) throw std::invalid_argument("matrix coefficients are not NCL");
    double kr = 0, kb = 0;
    YuvConstants(m, kr, kb);
    return RgbToYuvFromKrKb(kr, kb);
}
Matrix3 YuvToRgbFromPrimaries(uint8_t p) {
    if (p == 1) return Inverse(RgbToYuvMatrix(1));
    if (p == 9) return Inverse(RgbToYuvMatrix(9));
    double kr = 0, kb = 0;
    YuvConstantsFromPrimaries(p, kr, kb);
    return Inverse(RgbToYuvFromKrKb(kr, kb));
}
Matrix3 LmsToIctCp(uint8_t transfer) {
    if (transfer == 18)
        return {0.5, 0.5, 0.0, 3625.0 / 4096.0, -7465.0 / 4096.0, 3840.0 / 4096.0,
                9500.0 / 4096.0, -9212.0 / 4096.0, -288.0 / 4096.0};
    return {0.5, 0.5, 0.0, 6610.0 / 4096.0, -13613.0 / 4096.0, 7003.0 / 4096.0,
            17933.0 / 4096.0, -17390.0 / 4096.0, -543.0 / 4096.0};
}
Matrix3 RgbToXyz(uint8_t p) {
    if (p == 10) return Identity();
    const Matrix3 m = PrimariesXyz(p);
    const Vec3d s = MulV(Inverse(m), WhitePoint(p));
    Matrix3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i * 3 + j] = m[i * 3 + j] * s[j];
    return r;
}
Matrix3 XyzToRgb(uint8_t p) {
    if (p == 10) return Identity();
    return Inverse(RgbToXyz(p));
}
Matrix3 GamutMatrix(uint8_t from, uint8_t to) {
    return Multiply(XyzToRgb(to), RgbToXyz(from));
}
Matrix3 LmsToRgbMatrix() {
    const Matrix3 m{1688.0 / 4096.0, 2146.0 / 4096.0, 262.0 / 4096.0,
                    683.0 / 4096.0,  2951.0 / 4096.0, 462.0 / 4096.0,
                    99.0 / 4096.0,   309.0 / 4096.0,  3688.0 / 4096.0};
    return Inverse(m);
}
double Rec709Oetf(double x) {
    x = std::max(x, 0.0);
    return x < 0.018053968510807 ? x * 4.5
                                 : 1.09929682680944 * std::pow(x, 0.45) -
                                       (1.09929682680944 - 1.0);
}

// input.cc:700-712.
int SelectMode(const ss2o_format& f) {
    if (f.family == 0) return 0;
    if (f.matrix == 10 || f.matrix == 13) return 1;
    if (f.matrix == 14) return 2;
    return 0;
}

// input.cc:664-698.
void SelectTransfer(uint8_t t, int& id, float& scale) {
    scale = 1.0f;
    switch (t) {
        case 8: id = 0; return;
        case 1: case 6: case 14: case 15: case 7: id = 1; return;
        case 4: id = 2; return;
        case 5: id = 3; return;
        case 13: id = 4; return;
        case 9: id = 5; return;
        case 10: id = 6; return;
        case 11: id = 7; return;
        case 12: id = 8; return;
        case 16: id = 9; scale = 10000.0f / 100.0f; return;
        case 17: id = 10; return;
        case 18: id = 11; scale = 1000.0f / 100.0f; return;
    }
    throw std::invalid_argument("unsupported transfer characteristics");
}

// input.cc:714-757.
void PlaneScaleOffset(const ss2o_format& f, bool chroma, bool alpha,
                      float& scale, float& offset) {
    const bool is_float = f.type == 2 || f.type == 3;
    const int depth = EffectiveDepth(f);
    if (depth < 1 || depth > TypeDepth(f.type))
        throw std::invalid_argument("invalid bit depth for pixel type");
    if (f.range > 1) throw std::invalid_argument("invalid pixel range");
    if (f.range == 0 && depth < 8)
        throw std::invalid_argument("limited range requires a bit depth of at least 8");
    if (is_float) { scale = 1.0f; offset = 0.0f; return; }
    const bool full = alpha || f.range == 1;
    const bool ycgco = f.matrix == 8;
    const double numeric_max = static_cast<double>((1u << depth) - 1u);
    const double range =
        full ? numeric_max
             : static_cast<double>(chroma && !ycgco ? 224u << (depth - 8)
                                                    : 219u << (depth - 8));
    double off = 0.0;
    if (alpha) off = 0.0;
    else if (chroma) off = static_cast<double>(1u << (depth - 1));
    else if (!full) off = static_cast<double>(16u << (depth - 8));
    scale = static_cast<float>(1.0 / range);
    offset = static_cast<float>(-off / range);
}

// input.cc:759-783.
void LumaCoefficients(const ss2o_format& f, double& kr, double& kg, double& kb) {
    kr = 0.0; kg = 1.0; kb = 0.0;
    const int mode = SelectMode(f);
    if (f.family == 0) return;
    if (mode == 1) {
        if (f.matrix == 13) YuvConstantsFromPrimaries(f.primaries, kr, kb);
        else YuvConstants(f.matrix, kr, kb);
    } else if (f.transfer == 18) {
        YuvConstantsFromPrimaries(f.primaries, kr, kb);
    } else {
        return;
    }
    kg = 1.0 - kr - kb;
}

// input.cc:785-800.
Matrix3 NclToRgbMatrix(const ss2o_format& f, bool& identity) {
    identity = true;
    if (f.family == 0) return Identity();
    if (f.matrix == 0 || f.matrix == 2) return Identity();
    identity = false;
    if (f.matrix == 12) return YuvToRgbFromPrimaries(f.primaries);
    return Inverse(RgbToYuvMatrix(f.matrix));
}

// vulkan_source.cc:44-73.
void ChromaSiting(const ss2o_format& f, double& sx, double& sy) {
    const double rw = 1.0 / static_cast<double>(1u << f.subsample_w);
    const double rh = 1.0 / static_cast<double>(1u << f.subsample_h);
    const double left = 0.5 - 0.5 * rw;
    const double top = 0.5 - 0.5 * rh;
    const double bottom = -(0.5 - 0.5 * rh);
    sx = 0.0; sy = 0.0;
    switch (f.chroma_location) {
        case 0: sx = left; break;
        case 1: break;
        case 2: sx = left; sy = top; break;
        case 3: sy = top; break;
        case 4: sx = left; sy = bottom; break;
        case 5: sy = bottom; break;
    }
}

// The decode constants of one image: VQM's SourceDesc
// (src/vulkan/vulkan_support.h:104-120, built by vulkan_source.cc:77-182),
// kept in double and rounded to the working type at use.
struct Desc {
    int type = 0, family = 0, alpha = 0, sub_w = 0, sub_h = 0;
    int transfer = 0, mode = 0, filter = 0;
    bool identity1 = true, identity2 = true, chroma_variant = false;
    double scale[3]{}, offset[3]{};   // luma, chroma, alpha (stored as float)
    double m1[9]{}, m2[9]{};          // stored as float
    double kr = 0, kg = 1, kb = 0, to_linear = 1, shift_x = 0, shift_y = 0;
    double cl[4]{};
    float scale_f[3]{}, offset_f[3]{}, m1_f[9]{}, m2_f[9]{};
    float kr_f = 0, kg_f = 1, kb_f = 0, to_linear_f = 1, shift_x_f = 0,
          shift_y_f = 0, cl_f[4]{};
};

Desc BuildDesc(const ss2o_format& f, int chroma_filter) {
    Desc d;
    d.type = f.type;
    d.family = f.family;
    d.alpha = f.alpha;
    d.sub_w = f.subsample_w;
    d.sub_h = f.subsample_h;
    d.mode = SelectMode(f);
    float tls = 1.0f;
    SelectTransfer(f.transfer, d.transfer, tls);
    d.to_linear = tls;
    d.to_linear_f = tls;
    d.filter = chroma_filter;
    d.chroma_variant = f.subsample_w != 0 || f.subsample_h != 0;
    float s, o;
    PlaneScaleOffset(f, false, false, s, o);
    d.scale_f[0] = s; d.offset_f[0] = o;
    PlaneScaleOffset(f, f.family == 2, false, s, o);
    d.scale_f[1] = s; d.offset_f[1] = o;
    PlaneScaleOffset(f, false, true, s, o);
    d.scale_f[2] = s; d.offset_f[2] = o;
    Matrix3 m1 = Identity();
    if (d.mode == 1) {
        d.identity1 = true;
    } else if (d.mode == 2) {
        m1 = Inverse(LmsToIctCp(f.transfer));
        d.identity1 = false;
    } else {
        bool id = false;
        m1 = NclToRgbMatrix(f, id);
        d.identity1 = id;
    }
    Matrix3 m2 = Identity();
    if (f.family == 0 || f.primaries == 1) {
        d.identity2 = true;
    } else if (d.mode == 2) {
        m2 = Multiply(GamutMatrix(f.primaries, 1), LmsToRgbMatrix());
        d.identity2 = false;
    } else {
        m2 = GamutMatrix(f.primaries, 1);
        d.identity2 = false;
    }
    double kr, kg, kb;
    LumaCoefficients(f, kr, kg, kb);
    double sx = 0.0, sy = 0.0;
    if (f.family == 2 && d.chroma_variant) ChromaSiting(f, sx, sy);
    double cl[4] = {0, 0, 0, 0};
    if (d.mode == 1) {
        cl[0] = Rec709Oetf(1.0 - kb);
        cl[1] = 1.0 - Rec709Oetf(kb);
        cl[2] = Rec709Oetf(1.0 - kr);
        cl[3] = 1.0 - Rec709Oetf(kr);
    }
    for (int i = 0; i < 3; ++i) {
        d.scale[i] = d.scale_f[i];
        d.offset[i] = d.offset_f[i];
    }
    for (int i = 0; i < 9; ++i) {
        d.m1[i] = m1[i];
        d.m2[i] = m2[i];
        d.m1_f[i] = static_cast<float>(m1[i]);
        d.m2_f[i] = static_cast<float>(m2[i]);
    }
    d.kr = kr; d.kg = kg; d.kb = kb;
    d.kr_f = static_cast<float>(kr);
    d.kg_f = static_cast<float>(kg);
    d.kb_f = static_cast<float>(kb);
    d.shift_x = sx; d.shift_y = sy;
    d.shift_x_f = static_cast<float>(sx);
    d.shift_y_f = static_cast<float>(sy);
    for (int i = 0; i < 4; ++i) {
        d.cl[i] = cl[i];
        d.cl_f[i] = static_cast<float>(cl[i]);
    }
    return d;
}

// Per-type view of the constants: the FP32 path reads the float copies VQM
// uploads; the FP64 path reads the double values they were rounded from.
template <class T> struct K;
template <> struct K<float> {
    static float scale(const Desc& d, int i) { return d.scale_f[i]; }
    static float offset(const Desc& d, int i) { return d.offset_f[i]; }
    static float m1(const Desc& d, int i) { return d.m1_f[i]; }
    static float m2(const Desc& d, int i) { return d.m2_f[i]; }
    static float kr(const Desc& d) { return d.kr_f; }
    static float kg(const Desc& d) { return d.kg_f; }
    static float kb(const Desc& d) { return d.kb_f; }
    static float tl(const Desc& d) { return d.to_linear_f; }
    static float sx(const Desc& d) { return d.shift_x_f; }
    static float sy(const Desc& d) { return d.shift_y_f; }
    static float cl(const Desc& d, int i) { return d.cl_f[i]; }
};
template <> struct K<double> {
    static double scale(const Desc& d, int i) { return d.scale[i]; }
    static double offset(const Desc& d, int i) { return d.offset[i]; }
    static double m1(const Desc& d, int i) { return d.m1[i]; }
    static double m2(const Desc& d, int i) { return d.m2[i]; }
    static double kr(const Desc& d) { return d.kr; }
    static double kg(const Desc& d) { return d.kg; }
    static double kb(const Desc& d) { return d.kb; }
    static double tl(const Desc& d) { return d.to_linear; }
    static double sx(const Desc& d) { return d.shift_x; }
    static double sy(const Desc& d) { return d.shift_y; }
    static double cl(const Desc& d, int i) { return d.cl[i]; }
};

float HalfToFloat(uint16_t h) {
    const uint32_t sign = static_cast<uint32_t>(h & 0x8000u) << 16;
    const uint32_t exp = (h >> 10) & 0x1Fu;
    uint32_t man = h & 0x3FFu;
    uint32_t bits;
    if (exp == 0) {
        if (man == 0) {
            bits = sign;
        } else {
            int shift = 0;
            while ((man & 0x400u) == 0) { man <<= 1; ++shift; }
            man &= 0x3FFu;
            bits = sign | (static_cast<uint32_t>(127 - 14 - shift) << 23) | (man << 13);
        }
    } else if (exp == 0x1F) {
        bits = sign | 0x7F800000u | (man << 13);
    } else {
        bits = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    float r;
    std::memcpy(&r, &bits, 4);
    return r;
}

// ---------------------------------------------------------------------------
// Decode to linear Rec.709 (color.glsl).
// ---------------------------------------------------------------------------

template <class T> T Pow(T a, T b);
template <> float Pow<float>(float a, float b) { return ss2dm::pow(a, b); }
template <> double Pow<double>(double a, double b) { return std::pow(a, b); }
// The pure power-law transfers (color.glsl:157-159): the shared
// single-precision power in the FP32 path.
template <class T> T Gamma(T a, T b);
template <> float Gamma<float>(float a, float b) { return ss2dm::powf_gamma(a, b); }
template <> double Gamma<double>(double a, double b) { return std::pow(a, b); }
template <class T> T Exp(T a);
template <> float Exp<float>(float a) { return ss2dm::exp(a); }
template <> double Exp<double>(double a) { return std::exp(a); }
template <class T> T Cbrt(T a);
template <> float Cbrt<float>(float a) { return ss2dm::cbrt(a); }
template <> double Cbrt<double>(double a) { return std::cbrt(a); }
// sin(pi v) / (pi v) with the reference's float pi in the denominator.
template <class T> T Sinc(T v);
template <> float Sinc<float>(float v) {
    const float pi = 3.14159265358979323846f;
    return v == 0.0f ? 1.0f : ss2dm::sinpi(v) / (pi * v);
}
template <> double Sinc<double>(double v) {
    const double pi = 3.14159265358979323846;
    return v == 0.0 ? 1.0 : std::sin(pi * v) / (pi * v);
}

template <class T>
struct Decoder {
    const Desc& d;
    const uint8_t* data;
    uint32_t width, height;
    size_t plane_offset[4];
    uint32_t row_samples[4];
    uint32_t plane_w[4], plane_h[4];

    Decoder(const Desc& desc, const ss2o_image& img) : d(desc), data(img.data) {
        width = img.width;
        height = img.height;
        const auto layout = PlaneLayout(img.format, img.width, img.height);
        for (int p = 0; p < 4; ++p) {
            plane_offset[p] = layout[p].offset;
            row_samples[p] = static_cast<uint32_t>(layout[p].width);
            const bool chroma = p == 1 || p == 2;
            plane_w[p] = chroma ? (width >> d.sub_w) : width;
            plane_h[p] = chroma ? (height >> d.sub_h) : height;
        }
    }

    // color.glsl:94-113: raw sample times scale plus offset of its plane class.
    T Raw(int plane, uint32_t x, uint32_t y) const {
        const size_t index = static_cast<size_t>(y) * row_samples[plane] + x;
        const uint8_t* base = data + plane_offset[plane];
        float v;
        switch (d.type) {
            case 0: v = static_cast<float>(base[index]); break;
            case 1: {
                uint16_t s;
                std::memcpy(&s, base + 2 * index, 2);
                v = static_cast<float>(s);
                break;
            }
            case 2: {
                uint16_t s;
                std::memcpy(&s, base + 2 * index, 2);
                v = HalfToFloat(s);
                break;
            }
            default: std::memcpy(&v, base + 4 * index, 4); break;
        }
        const int cls = plane == 3 ? 2 : (plane != 0 && d.family == 2 ? 1 : 0);
        return std::fma(static_cast<T>(v), K<T>::scale(d, cls),
                        K<T>::offset(d, cls));
    }

    // color.glsl:117-205.
    static T Rec709InvOetf(T x) {
        x = std::max(x, T(0));
        const T alpha = T(1.09929682680944), beta = T(0.018053968510807);
        return x < T(4.5) * beta
                   ? x / T(4.5)
                   : Pow<T>((x + (alpha - T(1))) / alpha, T(1) / T(0.45));
    }
    static T SrgbEotf(T v) {
        return v <= T(0.04045) ? v / T(12.92)
                               : Pow<T>((v + T(0.055)) / T(1.055), T(2.4));
    }
    static T St2084Eotf(T x) {
        if (x <= T(0)) return T(0);
        const T xp = Pow<T>(x, T(1) / T(78.84375));
        const T num = std::max(xp - T(0.8359375), T(0));
        const T den = std::max(T(18.8515625) - T(18.6875) * xp,
                               T(1.17549435e-38));
        return Pow<T>(num / den, T(1) / T(0.1593017578125));
    }
    static T AribInvOetf(T x) {
        x = std::max(x, T(0));
        return x <= T(0.5)
                   ? (x * x) * (T(1) / T(3))
                   : (Exp<T>((x - T(0.55991073)) / T(0.17883277)) +
                      T(0.28466892)) / T(12);
    }
    T Transfer(int id, T v) const {
        switch (id) {
            case 0: return v;
            case 1: return v < T(0) ? T(0) : Gamma<T>(v, T(2.4));
            case 2: return v < T(0) ? T(0) : Gamma<T>(v, T(2.2));
            case 3: return v < T(0) ? T(0) : Gamma<T>(v, T(2.8));
            case 4: return SrgbEotf(v);
            case 5: return v <= T(0) ? T(0.01) : Pow<T>(T(10), T(2) * (v - T(1)));
            case 6: return v <= T(0) ? T(0.00316227766)
                                     : Pow<T>(T(10), T(2.5) * (v - T(1)));
            case 7:
                return v >= T(0) && v <= T(1)
                           ? Pow<T>(v, T(2.4))
                           : (v < T(0) ? -Rec709InvOetf(-v) : Rec709InvOetf(v));
            case 8:
                if (v >= T(0) && v <= T(1)) return Pow<T>(v, T(2.4));
                return v >= T(0) ? Rec709InvOetf(v)
                                 : -Rec709InvOetf(T(-4) * v) / T(4);
            case 9: return K<T>::tl(d) * St2084Eotf(v);
            case 10: return v < T(0) ? T(0) : (T(52.37) / T(48)) * Pow<T>(v, T(2.6));
        }
        return v;
    }
    void TransferRgb(T c[3]) const {
        if (d.transfer == 11) {
            for (int i = 0; i < 3; ++i) c[i] = AribInvOetf(c[i]);
            const T luma = std::max(
                std::fma(K<T>::kb(d), c[2],
                         std::fma(K<T>::kg(d), c[1], K<T>::kr(d) * c[0])),
                T(1.17549435e-38));
            const T f = Pow<T>(luma, T(0.2)) * K<T>::tl(d);
            for (int i = 0; i < 3; ++i) c[i] = c[i] * f;
            return;
        }
        for (int i = 0; i < 3; ++i) c[i] = Transfer(d.transfer, c[i]);
    }
    // color.glsl:209-218.
    static void ApplyMatrix(const Desc& desc, bool second, T v[3]) {
        T r[3];
        for (int row = 0; row < 3; ++row) {
            const T a = second ? K<T>::m2(desc, row * 3 + 0) : K<T>::m1(desc, row * 3 + 0);
            const T b = second ? K<T>::m2(desc, row * 3 + 1) : K<T>::m1(desc, row * 3 + 1);
            const T c = second ? K<T>::m2(desc, row * 3 + 2) : K<T>::m1(desc, row * 3 + 2);
            r[row] = std::fma(c, v[2], std::fma(b, v[1], a * v[0]));
        }
        v[0] = r[0]; v[1] = r[1]; v[2] = r[2];
    }
    // color.glsl:223-236.
    void ClToRgb(T e[3]) const {
        const T u = e[1], v = e[2];
        const T kbv = u < T(0) ? K<T>::cl(d, 0) : K<T>::cl(d, 1);
        const T krv = v < T(0) ? K<T>::cl(d, 2) : K<T>::cl(d, 3);
        const T b = Rec709InvOetf(std::fma(u * T(2), kbv, e[0]));
        const T r = Rec709InvOetf(std::fma(v * T(2), krv, e[0]));
        const T luma = Rec709InvOetf(e[0]);
        const T g = std::fma(-K<T>::kb(d), b, std::fma(-K<T>::kr(d), r, luma)) /
                    K<T>::kg(d);
        e[0] = r; e[1] = g; e[2] = b;
    }

    // color.glsl:271-283.
    static T RoundHalfup(T x) {
        return x < T(0) ? std::floor(x + T(0.5)) : std::floor(x + T(0.49999997));
    }
    static int MirrorIndex(T xpos, uint32_t dim) {
        const T extent = static_cast<T>(dim);
        const T m = xpos < T(0) ? -xpos
                                : (xpos >= extent ? T(2) * extent - xpos : xpos);
        return static_cast<int>(std::min(std::max(m, T(0)), extent - T(1)));
    }
    static T Kernel(int filter, T x) {
        x = std::abs(x);
        if (filter == 0) return std::max(T(1) - x, T(0));
        if (filter == 1) {
            if (x < T(1)) return std::fma(x * x, std::fma(x, T(1.5), T(-2.5)), T(1));
            if (x < T(2))
                return std::fma(x, std::fma(x, std::fma(T(-0.5), x, T(2.5)), T(-4)),
                                T(2));
            return T(0);
        }
        return x < T(3) ? Sinc<T>(x) * Sinc<T>(x / T(3)) : T(0);
    }

    // color.glsl:288-367: bilinear chroma of the four samples of a block.
    void BilinearPhase(uint32_t out_pos, T scale, T shift, int centre, int& s0,
                       int& s1, T& w0, T& w1) const {
        const T pos = (static_cast<T>(out_pos) + T(0.5)) / scale + shift;
        const T base = RoundHalfup(pos - T(1)) + T(0.5);
        const T t = pos - base;
        s0 = static_cast<int>(std::floor(base)) - centre + 1;
        s1 = s0 + 1;
        w0 = T(1) - t;
        w1 = t;
    }
    void ChromaBilinear(int plane, const uint32_t px[4], const uint32_t py[4],
                        T out[4]) const {
        const uint32_t dx = plane_w[plane], dy = plane_h[plane];
        const int cx = static_cast<int>(px[0] >> d.sub_w);
        const int cy = static_cast<int>(py[0] >> d.sub_h);
        T win[9];
        const bool interior = cx > 0 && cx + 1 < static_cast<int>(dx) && cy > 0 &&
                              cy + 1 < static_cast<int>(dy);
        for (int j = -1; j <= 1; ++j)
            for (int i = -1; i <= 1; ++i) {
                uint32_t sx, sy;
                if (interior) {
                    sx = static_cast<uint32_t>(cx + i);
                    sy = static_cast<uint32_t>(cy + j);
                } else {
                    sx = static_cast<uint32_t>(MirrorIndex(static_cast<T>(cx + i) + T(0.5), dx));
                    sy = static_cast<uint32_t>(MirrorIndex(static_cast<T>(cy + j) + T(0.5), dy));
                }
                win[(j + 1) * 3 + (i + 1)] = Raw(plane, sx, sy);
            }
        const T scx = static_cast<T>(1u << d.sub_w), scy = static_cast<T>(1u << d.sub_h);
        const T shx = K<T>::sx(d), shy = K<T>::sy(d);
        int xa0, xa1, xb0, xb1, ya0, ya1, yb0, yb1;
        T xwa0, xwa1, xwb0, xwb1, ywa0, ywa1, ywb0, ywb1;
        BilinearPhase(px[0], scx, shx, cx, xa0, xa1, xwa0, xwa1);
        BilinearPhase(px[1], scx, shx, cx, xb0, xb1, xwb0, xwb1);
        BilinearPhase(py[0], scy, shy, cy, ya0, ya1, ywa0, ywa1);
        BilinearPhase(py[2], scy, shy, cy, yb0, yb1, ywb0, ywb1);
        // Along an axis that is not subsampled the second tap of a phase can
        // fall one slot past the 3x3 window (color.glsl indexes past its
        // array there), always with weight exactly 0: such a slot reads 0.
        auto at = [&](int y, int x) { return y <= 2 && x <= 2 ? win[y * 3 + x] : T(0); };
        auto window = [&](int xa, int xb, int ya, int yb, T xwa, T xwb, T ywa,
                          T ywb) {
            const T w00 = xwa * ywa, w10 = xwb * ywa, w01 = xwa * ywb,
                    w11 = xwb * ywb;
            return std::fma(w11, at(yb, xb),
                            std::fma(w01, at(yb, xa),
                                     std::fma(w10, at(ya, xb), w00 * at(ya, xa))));
        };
        out[0] = window(xa0, xa1, ya0, ya1, xwa0, xwa1, ywa0, ywa1);
        out[1] = window(xb0, xb1, ya0, ya1, xwb0, xwb1, ywa0, ywa1);
        out[2] = window(xa0, xa1, yb0, yb1, xwa0, xwa1, ywb0, ywb1);
        out[3] = window(xb0, xb1, yb0, yb1, xwb0, xwb1, ywb0, ywb1);
    }

    // color.glsl:371-432: bicubic / Lanczos chroma.
    void AxisTaps(uint32_t out_pos, T scale, T shift, uint32_t dim, int taps,
                  T* w, int* idx) const {
        const T pos = (static_cast<T>(out_pos) + T(0.5)) / scale + shift;
        const T base = RoundHalfup(pos - static_cast<T>(taps) / T(2)) + T(0.5);
        T total = T(0);
        for (int j = 0; j < taps; ++j)
            total += Kernel(d.filter, base + static_cast<T>(j) - pos);
        for (int j = 0; j < taps; ++j) {
            w[j] = Kernel(d.filter, base + static_cast<T>(j) - pos) / total;
            idx[j] = MirrorIndex(base + static_cast<T>(j), dim);
        }
    }
    void ChromaTaps(int plane, const uint32_t px[4], const uint32_t py[4],
                    T out[4]) const {
        const int taps = d.filter == 1 ? 4 : 6;
        const T scx = static_cast<T>(1u << d.sub_w), scy = static_cast<T>(1u << d.sub_h);
        T wx0[6], wx1[6], wy0[6], wy1[6];
        int ix0[6], ix1[6], iy0[6], iy1[6];
        AxisTaps(px[0], scx, K<T>::sx(d), plane_w[plane], taps, wx0, ix0);
        AxisTaps(px[1], scx, K<T>::sx(d), plane_w[plane], taps, wx1, ix1);
        AxisTaps(py[0], scy, K<T>::sy(d), plane_h[plane], taps, wy0, iy0);
        AxisTaps(py[2], scy, K<T>::sy(d), plane_h[plane], taps, wy1, iy1);
        auto taps2d = [&](const T* wx, const int* ix, const T* wy, const int* iy) {
            T sum = T(0);
            for (int j = 0; j < taps; ++j) {
                T row = T(0);
                for (int k = 0; k < taps; ++k)
                    row = std::fma(wx[k], Raw(plane, static_cast<uint32_t>(ix[k]),
                                              static_cast<uint32_t>(iy[j])), row);
                sum = std::fma(wy[j], row, sum);
            }
            return sum;
        };
        out[0] = taps2d(wx0, ix0, wy0, iy0);
        out[1] = taps2d(wx1, ix1, wy0, iy0);
        out[2] = taps2d(wx0, ix0, wy1, iy1);
        out[3] = taps2d(wx1, ix1, wy1, iy1);
    }

    // color.glsl:447-541: the four samples of block (bx, by), linear Rec.709,
    // in (0,0), (1,0), (0,1), (1,1) order.
    void Block(uint32_t bx, uint32_t by, T bg, T rgb[4][3]) const {
        const uint32_t lx = width - 1, ly = height - 1;
        const uint32_t px[4] = {std::min(2 * bx, lx), std::min(2 * bx + 1, lx),
                                std::min(2 * bx, lx), std::min(2 * bx + 1, lx)};
        const uint32_t py[4] = {std::min(2 * by, ly), std::min(2 * by, ly),
                                std::min(2 * by + 1, ly), std::min(2 * by + 1, ly)};
        T cu[4] = {0, 0, 0, 0}, cv[4] = {0, 0, 0, 0};
        if (d.chroma_variant && d.family == 2) {
            if (d.filter == 0) {
                ChromaBilinear(1, px, py, cu);
                ChromaBilinear(2, px, py, cv);
            } else {
                ChromaTaps(1, px, py, cu);
                ChromaTaps(2, px, py, cv);
            }
        }
        const bool has_alpha = d.alpha != 0;
        const bool premul = d.alpha == 2;
        for (int i = 0; i < 4; ++i) {
            const T alpha = has_alpha ? Raw(3, px[i], py[i]) : T(1);
            T e[3];
            e[0] = e[1] = e[2] = Raw(0, px[i], py[i]);
            if (d.family != 0) {
                if (d.chroma_variant && d.family == 2) {
                    e[1] = cu[i];
                    e[2] = cv[i];
                } else {
                    e[1] = Raw(1, px[i], py[i]);
                    e[2] = Raw(2, px[i], py[i]);
                }
            }
            if (d.mode == 1) ClToRgb(e);
            else if (!d.identity1) ApplyMatrix(d, false, e);
            if (premul) {
                const T cl = std::min(std::max(alpha, T(0)), T(1));
                if (cl == T(0)) e[0] = e[1] = e[2] = T(0);
                else for (int k = 0; k < 3; ++k) e[k] = e[k] / cl;
            }
            if (has_alpha) {
                const T target = (T(1) - alpha) * bg;
                for (int k = 0; k < 3; ++k) e[k] = std::fma(alpha, e[k], target);
            }
            if (d.mode != 1) TransferRgb(e);
            if (!d.identity2) ApplyMatrix(d, true, e);
            rgb[i][0] = e[0]; rgb[i][1] = e[1]; rgb[i][2] = e[2];
        }
    }
};

// ---------------------------------------------------------------------------
// XYB pyramid (prepare.comp).
// ---------------------------------------------------------------------------

// prepare.comp:40-54, 78-98.
template <class T>
void Xyb(const T lin[3], T out[3]) {
    const T m00 = T(0.30), m02 = T(0.078), m01 = T(1.0 - 0.078 - 0.30);
    const T m10 = T(0.23), m12 = T(0.078), m11 = T(1.0 - 0.078 - 0.23);
    const T m20 = T(0.24342268924547819), m21 = T(0.20476744424496821);
    const T m22 = T(1.0 - 0.24342268924547819 - 0.20476744424496821);
    const T bias = T(0.0037930732552754493);
    const T cbias = T(0.15595419704914093);
    T m0 = std::fma(m00, lin[0], std::fma(m01, lin[1], std::fma(m02, lin[2], bias)));
    T m1 = std::fma(m10, lin[0], std::fma(m11, lin[1], std::fma(m12, lin[2], bias)));
    T m2 = std::fma(m20, lin[0], std::fma(m21, lin[1], std::fma(m22, lin[2], bias)));
    m0 = std::max(m0, T(0));
    m1 = std::max(m1, T(0));
    m2 = std::max(m2, T(0));
    // prepare.comp:78 evaluates pow(v, 1/3); the cube root here is that value
    // in exact arithmetic, rounded to the working type.
    const T c0 = Cbrt<T>(m0) - cbias;
    const T c1 = Cbrt<T>(m1) - cbias;
    const T c2 = Cbrt<T>(m2) - cbias;
    out[0] = std::fma(T(0.5) * (c0 - c1), T(14), T(0.42));
    out[1] = std::fma(T(0.5), c0 + c1, T(0.01));
    out[2] = std::fma(T(-0.5), c0 + c1, c2) + T(0.55);
}

template <class T>
struct Pyramid {
    int levels = 0;
    Size sizes[kMaxScales];
    // planes[level][channel]: W_l*H_l values, empty when pruned.
    std::vector<T> planes[kMaxScales][3];
};

// IEEE binary16 rounding (to nearest, ties to even) of a float, returned as
// float: the plane_round / plane_store of the half-plane build
// (ssimu2_common.glsl:45-56, 86-91). Normal halves keep 11 significant bits;
// below 2^-14 the quantum is 2^-24; beyond 65504 the value becomes infinite.
float RoundHalf(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t a = u & 0x7fffffffu;
    if (a >= 0x7f800000u) return f;  // inf, NaN
    float r;
    if (a >= 0x38800000u) {  // |f| >= 2^-14: drop 13 mantissa bits, ties to even
        const uint32_t lsb = (u >> 13) & 1u;
        const uint32_t v = (u + 0xfffu + lsb) & ~0x1fffu;
        std::memcpy(&r, &v, 4);
        if (std::fabs(r) > 65504.0f) r = std::copysign(INFINITY, f);
    } else {  // subnormal half: a multiple of 2^-24
        r = std::nearbyint(f * 16777216.0f) * 5.9604644775390625e-8f;
        if (r == 0.0f) r = std::copysign(0.0f, f);
    }
    return r;
}

// prepare.comp:103-111: ((((0+a)+b)+c)+d) * 0.25, rounded to half with
// half planes (the average used to pass through the plane region).
template <class T>
T BoxAverage(T a, T b, T c, T d, bool half = false) {
    T s = T(0);
    s += a; s += b; s += c; s += d;
    s = s * T(0.25);
    if constexpr (std::is_same_v<T, float>)
        if (half) s = RoundHalf(s);
    return s;
}

// prepare.comp:170-232: level 0 from the decoded blocks, level l >= 1 the
// edge-clamped 2x2 average of level l-1 in linear RGB, XYB stored per level
// for the channels the pruning mask keeps.
template <class T>
void BuildPyramid(const ss2o_image& img, const Desc& desc, T bg, const Plan& plan,
                  Pyramid<T>& pyr, bool half = false) {
    pyr.levels = plan.count;
    for (int l = 0; l < plan.count; ++l) {
        pyr.sizes[l] = plan.sizes[l];
        for (int c = 0; c < 3; ++c) {
            if (!ChannelPruned(c, l, plan.count))
                pyr.planes[l][c].assign(size_t(plan.sizes[l].w) * plan.sizes[l].h, T(0));
            else
                pyr.planes[l][c].clear();
        }
    }
    const Decoder<T> dec(desc, img);
    const uint32_t W = img.width, H = img.height;
    std::vector<T> lin(size_t(W) * H * 3);
    const uint32_t bw = (W + 1) / 2, bh = (H + 1) / 2;
    for (uint32_t by = 0; by < bh; ++by)
        for (uint32_t bx = 0; bx < bw; ++bx) {
            T rgb[4][3];
            dec.Block(bx, by, bg, rgb);
            for (int i = 0; i < 4; ++i) {
                const uint32_t x = std::min(2 * bx + (i & 1), W - 1);
                const uint32_t y = std::min(2 * by + (i >> 1), H - 1);
                T* dst = &lin[(size_t(y) * W + x) * 3];
                dst[0] = rgb[i][0]; dst[1] = rgb[i][1]; dst[2] = rgb[i][2];
            }
        }
    std::vector<T> next;
    for (int l = 0; l < plan.count; ++l) {
        const uint32_t w = plan.sizes[l].w, h = plan.sizes[l].h;
        for (uint32_t y = 0; y < h; ++y)
            for (uint32_t x = 0; x < w; ++x) {
                T xyb[3];
                Xyb(&lin[(size_t(y) * w + x) * 3], xyb);
                for (int c = 0; c < 3; ++c)
                    if (!pyr.planes[l][c].empty()) {
                        T v = xyb[c];
                        if constexpr (std::is_same_v<T, float>)
                            if (half) v = RoundHalf(v);
                        pyr.planes[l][c][size_t(y) * w + x] = v;
                    }
            }
        if (l + 1 < plan.count) {
            const uint32_t nw = plan.sizes[l + 1].w, nh = plan.sizes[l + 1].h;
            next.assign(size_t(nw) * nh * 3, T(0));
            for (uint32_t y = 0; y < nh; ++y)
                for (uint32_t x = 0; x < nw; ++x) {
                    const uint32_t x0 = std::min(2 * x, w - 1), x1 = std::min(2 * x + 1, w - 1);
                    const uint32_t y0 = std::min(2 * y, h - 1), y1 = std::min(2 * y + 1, h - 1);
                    for (int c = 0; c < 3; ++c)
                        next[(size_t(y) * nw + x) * 3 + c] = BoxAverage(
                            lin[(size_t(y0) * w + x0) * 3 + c], lin[(size_t(y0) * w + x1) * 3 + c],
                            lin[(size_t(y1) * w + x0) * 3 + c], lin[(size_t(y1) * w + x1) * 3 + c],
                            half);
                }
            lin.swap(next);
        }
    }
}

// ---------------------------------------------------------------------------
// The opt-in recursive Gaussian (no counterpart in VQM): the third-order
// truncated-cosine recursion of D. Charalampidis, IEEE Trans. Signal
// Processing 64(14), 2016, sigma 1.5, which Cloudinary's ssimulacra2
// (81feacf6) applies through libjxl's lib/jxl/gauss_blur.cc (e47d2a2b).
// Neither project is present here, so this restatement is pinned by the
// filter's defining properties (unit gain, variance sigma^2, recursion ==
// convolution), not by their outputs.
//
// Derived here from closed forms, independently of the library's numeric
// sums: with N = round(3.2795 sigma + 0.2546) and w_k = (2k+1) pi / (2N),
//   sum_{|m|<=N} cos(w_k m)             = (-1)^k / tan(w_k / 2)          (a_k)
//   sum_{|m|<=N} (N^2 - m^2) cos(w_k m) = (-1)^k / (tan^2(w_k/2) sin w_k) (b_k)
// and beta solves a . beta = 1, b . beta = N^2 - sigma^2 (unit gain,
// variance sigma^2) and v . beta = v . rho with v = a x b, the direction the
// first two leave free, rho_k = exp(-sigma^2 w_k^2 / 2) / N: beta is the
// point nearest rho on the two constraints.
// ---------------------------------------------------------------------------

struct RecursiveGauss {
    int n = 0;
    double w[3] = {}, beta[3] = {};
};

RecursiveGauss MakeRecursiveGauss() {
    constexpr double kPi = 3.14159265358979323846;
    const double sigma = 1.5;
    RecursiveGauss g;
    g.n = static_cast<int>(std::lround(3.2795 * sigma + 0.2546));
    double a[3], b[3], rho[3];
    for (int k = 0; k < 3; ++k) {
        g.w[k] = (2 * k + 1) * kPi / (2.0 * g.n);
        const double sign = (k & 1) ? -1.0 : 1.0;
        const double t = std::tan(0.5 * g.w[k]);
        a[k] = sign / t;
        b[k] = sign / (t * t * std::sin(g.w[k]));
        rho[k] = std::exp(-0.5 * sigma * sigma * g.w[k] * g.w[k]) / g.n;
    }
    const double v[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                         a[0] * b[1] - a[1] * b[0]};
    double m[3][4] = {{a[0], a[1], a[2], 1.0},
                      {b[0], b[1], b[2], double(g.n) * g.n - sigma * sigma},
                      {v[0], v[1], v[2], v[0] * rho[0] + v[1] * rho[1] + v[2] * rho[2]}};
    // Gaussian elimination with partial pivoting on the 3x4 system.
    for (int c = 0; c < 3; ++c) {
        int piv = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::abs(m[r][c]) > std::abs(m[piv][c])) piv = r;
        for (int k = 0; k < 4; ++k) std::swap(m[c][k], m[piv][k]);
        for (int r = 0; r < 3; ++r) {
            if (r == c) continue;
            const double f = m[r][c] / m[c][c];
            for (int k = c; k < 4; ++k) m[r][k] -= f * m[c][k];
        }
    }
    for (int k = 0; k < 3; ++k) g.beta[k] = m[k][3] / m[k][k];
    return g;
}

// The impulse response h(m) = sum_k beta_k cos(w_k m), |m| < N, centred in
// 13 taps (h(+-N) = 0 exactly: cos(w_k N) = 0).
std::array<double, kTaps> RecursiveTapsDouble() {
    const RecursiveGauss g = MakeRecursiveGauss();
    std::array<double, kTaps> h{};
    for (int m = -(g.n - 1); m <= g.n - 1; ++m) {
        double v = 0.0;
        for (int k = 0; k < 3; ++k) v += g.beta[k] * std::cos(g.w[k] * m);
        h[m + kRadius] = v;
    }
    return h;
}

// The recursion itself, in double, along one line of `len` samples at
// stride `step`, zero-padded: S_k[n] = 2 cos(w_k) S_k[n-1] - S_k[n-2]
// + (-1)^k sin(w_k) (x[n+N-1] + x[n-N-1]) from zero state,
// y[n] = sum_k beta_k S_k[n].
void RecursiveLine(const RecursiveGauss& g, const double* x, double* y, int len, size_t step) {
    double c2[3], sn[3], s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        c2[k] = 2.0 * std::cos(g.w[k]);
        sn[k] = ((k & 1) ? -1.0 : 1.0) * std::sin(g.w[k]);
    }
    auto at = [&](int i) { return (i >= 0 && i < len) ? x[size_t(i) * step] : 0.0; };
    for (int n = 1 - g.n; n < len; ++n) {
        const double in = at(n + g.n - 1) + at(n - g.n - 1);
        double out = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double s = c2[k] * s1[k] - s2[k] + sn[k] * in;
            s2[k] = s1[k];
            s1[k] = s;
            out += g.beta[k] * s;
        }
        if (n >= 0) y[size_t(n) * step] = out;
    }
}

// Rows, then columns, as the reference's blur runs them.
void RecursiveBlur(const std::vector<double>& src, std::vector<double>& dst, uint32_t w,
                   uint32_t h) {
    static const RecursiveGauss g = MakeRecursiveGauss();
    std::vector<double> tmp(src.size());
    dst.assign(src.size(), 0.0);
    for (uint32_t y = 0; y < h; ++y)
        RecursiveLine(g, &src[size_t(y) * w], &tmp[size_t(y) * w], static_cast<int>(w), 1);
    for (uint32_t x = 0; x < w; ++x)
        RecursiveLine(g, &tmp[x], &dst[x], static_cast<int>(h), w);
}

// ---------------------------------------------------------------------------
// Blurs, maps and norms (scale.comp) and their reduction (reduce.comp).
// ---------------------------------------------------------------------------

// blur 0: VQM's sampled Gaussian; 1: the recursive Gaussian's impulse
// response. The FP32 path rounds the taps to float as the kernels do.
constexpr int kBlurSampled = 0;
constexpr int kBlurRecursive = 1;

template <class T>
std::array<T, kTaps> Taps(int blur) {
    const auto w = blur == kBlurRecursive ? RecursiveTapsDouble() : GaussianDouble();
    std::array<T, kTaps> t{};
    for (int i = 0; i < kTaps; ++i) t[i] = static_cast<T>(static_cast<float>(w[i]));
    return t;
}
template <>
std::array<double, kTaps> Taps<double>(int blur) {
    return blur == kBlurRecursive ? RecursiveTapsDouble() : GaussianDouble();
}

// scale.comp:149-207: horizontal pass, zero padded, acc = w0*s0 then fused
// ascending taps. The zero halo makes a whole-plane pass identical to the
// tile-by-tile one.
template <class T>
void BlurH(const std::vector<T>& src, std::vector<T>& dst, uint32_t w, uint32_t h,
           const std::array<T, kTaps>& wt) {
    dst.assign(src.size(), T(0));
    std::vector<T> row(w + 2 * kRadius, T(0));
    for (uint32_t y = 0; y < h; ++y) {
        std::copy(src.begin() + size_t(y) * w, src.begin() + size_t(y + 1) * w,
                  row.begin() + kRadius);
        T* out = &dst[size_t(y) * w];
        for (uint32_t x = 0; x < w; ++x) {
            const T* s = &row[x];
            T acc = wt[0] * s[0];
            for (int t = 1; t < kTaps; ++t) acc = std::fma(wt[t], s[t], acc);
            out[x] = acc;
        }
    }
}

// scale.comp:211-301: vertical pass, a = 0, a += w_t * m_t ascending, each a
// fused multiply-add (the first one rounds w0*m0 exactly once).
template <class T>
void BlurV(const std::vector<T>& src, std::vector<T>& dst, uint32_t w, uint32_t h,
           const std::array<T, kTaps>& wt) {
    dst.assign(src.size(), T(0));
    for (uint32_t y = 0; y < h; ++y) {
        T* out = &dst[size_t(y) * w];
        for (int t = 0; t < kTaps; ++t) {
            const int sy = static_cast<int>(y) - kRadius + t;
            if (sy < 0 || sy >= static_cast<int>(h)) {
                // A zero row still takes part in the sum: fma(w, 0, a) == a.
                continue;
            }
            const T* s = &src[size_t(sy) * w];
            for (uint32_t x = 0; x < w; ++x) out[x] = std::fma(wt[t], s[x], out[x]);
        }
    }
}

// The maps' two quotients: in the FP32 path the shared division of
// ss2_detmath.h that the kernels use (its divisors, at least 0.0009 and 1,
// are in its domain), in the FP64 path the IEEE one.
template <class T> T MapDiv(T a, T b);
template <> float MapDiv<float>(float a, float b) { return ss2dm::divf(a, b); }
template <> double MapDiv<double>(double a, double b) { return a / b; }

// scale.comp:305-333: the SSIM' map in difference form and the edge maps.
template <class T>
void Maps(T mu1, T mu2, T s11, T s22, T s12, T img1, T img2, T out[6]) {
    const T C2 = T(0.0009);
    const T dm = mu1 - mu2;
    const T num_m = std::fma(-dm, dm, T(1));
    const T num_s = std::fma(T(2), std::fma(-mu1, mu2, s12), C2);
    const T denom = (std::fma(-mu1, mu1, s11) + std::fma(-mu2, mu2, s22)) + C2;
    const T d = std::max(MapDiv<T>(std::fma(-num_m, num_s, denom), denom), T(0));
    const T dd = d * d;
    out[0] = d;
    out[1] = dd * dd;
    const T dist = T(1) + std::abs(img2 - mu2);
    const T orig = T(1) + std::abs(img1 - mu1);
    const T d1 = MapDiv<T>(dist - orig, orig);
    const T ring = std::max(d1, T(0));
    const T blur = std::max(-d1, T(0));
    out[2] = ring;
    out[3] = (ring * ring) * (ring * ring);
    out[4] = blur;
    out[5] = (blur * blur) * (blur * blur);
}

// The four-quantity form of the maps: sigma11 and sigma22 enter the SSIM'
// denominator only as their sum, so s11 + s22 can be blurred as one quantity
// `ssum` (the blur of a*a + b*b, formed as fma(a, a, b*b)). The denominator
// is 2 * (0.5 * ssum - mu1^2 + 0.5 * (mu1 - mu2) * (mu1 + mu2)) + C2, whose
// correction term is exactly 0 when mu1 == mu2. For identical inputs ssum is
// exactly 2 * s11 (fma(a, a, a*a) == 2 * (a*a) and the taps commute with the
// factor 2) and s12 == s11, so the denominator is bit-identical to num_s and
// the map is exactly 0: identity still scores exactly 100. Not VQM's
// rounding: a mode of the CUDA blur, measured against the five-quantity form.
template <class T>
void Maps4(T mu1, T mu2, T ssum, T s12, T img1, T img2, T out[6]) {
    const T C2 = T(0.0009);
    const T dm = mu1 - mu2;
    const T num_m = std::fma(-dm, dm, T(1));
    const T num_s = std::fma(T(2), std::fma(-mu1, mu2, s12), C2);
    const T h = std::fma(-mu1, mu1, T(0.5) * ssum);
    const T denom = std::fma(T(2), std::fma(T(0.5) * dm, mu1 + mu2, h), C2);
    const T d = std::max(MapDiv<T>(std::fma(-num_m, num_s, denom), denom), T(0));
    const T dd = d * d;
    out[0] = d;
    out[1] = dd * dd;
    const T dist = T(1) + std::abs(img2 - mu2);
    const T orig = T(1) + std::abs(img1 - mu1);
    const T d1 = MapDiv<T>(dist - orig, orig);
    const T ring = std::max(d1, T(0));
    const T blur = std::max(-d1, T(0));
    out[2] = ring;
    out[3] = (ring * ring) * (ring * ring);
    out[4] = blur;
    out[5] = (blur * blur) * (blur * blur);
}

// One (level, channel): the six norm sums in VQM's reduction order
// (scale.comp:370-436, reduce.comp:21-63): per 32x32 tile, each of 256
// invocations sums its column's four rows, a halving ladder adds the 256
// invocation sums, the tile partial is stored, then reduce adds the partials
// 256-way strided and halves again.
// The FP64 recursive mode blurs by the recursion itself; every other mode
// by the 13-tap passes.
template <class T>
void Blur2D(const std::vector<T>& src, std::vector<T>& hq, std::vector<T>& dst, uint32_t w,
            uint32_t h, const std::array<T, kTaps>& wt, bool recursion) {
    if constexpr (std::is_same_v<T, double>) {
        if (recursion) {
            RecursiveBlur(src, dst, w, h);
            return;
        }
    }
    BlurH(src, hq, w, h, wt);
    BlurV(hq, dst, w, h, wt);
}

template <class T>
void ChannelSums(const std::vector<T>& a, const std::vector<T>& b, uint32_t w,
                 uint32_t h, const std::array<T, kTaps>& wt, T sums[6], bool four = false,
                 bool recursion = false) {
    std::vector<T> q[5], hq, bq[5];
    const size_t n = size_t(w) * h;
    for (int i = 0; i < 5; ++i) q[i].resize(n);
    for (size_t i = 0; i < n; ++i) {
        q[0][i] = a[i];
        q[1][i] = b[i];
        q[2][i] = four ? std::fma(a[i], a[i], b[i] * b[i]) : a[i] * a[i];
        q[3][i] = four ? T(0) : b[i] * b[i];
        q[4][i] = a[i] * b[i];
    }
    for (int i = 0; i < 5; ++i) {
        if (four && i == 3) continue;
        Blur2D(q[i], hq, bq[i], w, h, wt, recursion);
    }
    const uint32_t gx = (w + 31) / 32, gy = (h + 31) / 32;
    const uint32_t groups = gx * gy;
    std::vector<T> partials(size_t(groups) * 6);
    std::vector<T> pool(256 * 6);
    for (uint32_t ty = 0; ty < gy; ++ty)
        for (uint32_t tx = 0; tx < gx; ++tx) {
            for (int tid = 0; tid < 256; ++tid) {
                T s[6] = {0, 0, 0, 0, 0, 0};
                const uint32_t ox = tid % 32, row = (tid / 32) * 4;
                for (uint32_t r = 0; r < 4; ++r) {
                    const uint32_t x = tx * 32 + ox, y = ty * 32 + row + r;
                    if (x >= w || y >= h) continue;
                    const size_t i = size_t(y) * w + x;
                    T m[6];
                    if (four)
                        Maps4(bq[0][i], bq[1][i], bq[2][i], bq[4][i], a[i], b[i], m);
                    else
                        Maps(bq[0][i], bq[1][i], bq[2][i], bq[3][i], bq[4][i], a[i], b[i], m);
                    for (int k = 0; k < 6; ++k) s[k] += m[k];
                }
                for (int k = 0; k < 6; ++k) pool[k * 256 + tid] = s[k];
            }
            for (int st = 128; st > 0; st >>= 1)
                for (int tid = 0; tid < st; ++tid)
                    for (int k = 0; k < 6; ++k) pool[k * 256 + tid] += pool[k * 256 + tid + st];
            const uint32_t g = tx + ty * gx;
            for (int k = 0; k < 6; ++k) partials[size_t(k) * groups + g] = pool[k * 256];
        }
    T red[256];
    for (int k = 0; k < 6; ++k) {
        for (uint32_t i = 0; i < 256; ++i) {
            T s = T(0);
            for (uint32_t j = i; j < groups; j += 256) s += partials[size_t(k) * groups + j];
            red[i] = s;
        }
        for (int st = 128; st > 0; st >>= 1)
            for (int i = 0; i < st; ++i) red[i] += red[i + st];
        sums[k] = red[0];
    }
}

template <class T>
struct PairResult {
    int scales = 0;
    T sums[kMaxScales][18];
};

// The whole pair: both pyramids, then every kept (level, channel).
template <class T>
PairResult<T> ComputePair(const ss2o_image& o, const ss2o_image& dsrc, float background,
                          int chroma_filter, bool half = false, bool four = false,
                          int blur = kBlurSampled) {
    if (blur != kBlurSampled && blur != kBlurRecursive)
        throw std::invalid_argument("unknown blur mode");
    if (o.width != dsrc.width || o.height != dsrc.height)
        throw std::invalid_argument("image sizes differ");
    const Plan plan = PlanScales(o.width, o.height);
    const Desc d0 = BuildDesc(o.format, chroma_filter);
    const Desc d1 = BuildDesc(dsrc.format, chroma_filter);
    if (o.bytes < RequiredBytes(o.format, o.width, o.height) ||
        dsrc.bytes < RequiredBytes(dsrc.format, dsrc.width, dsrc.height))
        throw std::invalid_argument("data size does not match the image format");
    Pyramid<T> p0, p1;
    BuildPyramid<T>(o, d0, static_cast<T>(background), plan, p0, half);
    BuildPyramid<T>(dsrc, d1, static_cast<T>(background), plan, p1, half);
    const auto wt = Taps<T>(blur);
    PairResult<T> r;
    r.scales = plan.count;
    for (int l = 0; l < plan.count; ++l) {
        for (int k = 0; k < 18; ++k) r.sums[l][k] = T(0);
        for (int c = 0; c < 3; ++c) {
            if (ChannelPruned(c, l, plan.count)) continue;
            T s[6];
            ChannelSums<T>(p0.planes[l][c], p1.planes[l][c], plan.sizes[l].w,
                           plan.sizes[l].h, wt, s, four, blur == kBlurRecursive);
            r.sums[l][c * 2 + 0] = s[0];
            r.sums[l][c * 2 + 1] = s[1];
            r.sums[l][6 + c * 4 + 0] = s[2];
            r.sums[l][6 + c * 4 + 1] = s[3];
            r.sums[l][6 + c * 4 + 2] = s[4];
            r.sums[l][6 + c * 4 + 3] = s[5];
        }
    }
    return r;
}

// vulkan.cc:545-583: mean and fourth root in double.
template <class T>
void ReadResult(const PairResult<T>& r, const Plan& plan, double* norms) {
    for (int s = 0; s < r.scales; ++s) {
        const double inv = 1.0 / (static_cast<double>(plan.sizes[s].w) *
                                  static_cast<double>(plan.sizes[s].h));
        double* out = norms + s * 18;
        for (int c = 0; c < 3; ++c) {
            out[c * 2 + 0] = inv * static_cast<double>(r.sums[s][c * 2 + 0]);
            out[c * 2 + 1] = std::sqrt(std::sqrt(inv * static_cast<double>(r.sums[s][c * 2 + 1])));
            for (int n = 0; n < 4; ++n) {
                const double v = inv * static_cast<double>(r.sums[s][6 + c * 4 + n]);
                out[6 + c * 4 + n] = (n & 1) ? std::sqrt(std::sqrt(v)) : v;
            }
        }
    }
}

int Fail(const std::exception& e) {
    g_error = e.what();
    return SS2O_INVALID;
}

int ComputeOne(const ss2o_image* o, const ss2o_image* d, float bg, int filter,
               int precision, int blur, double* norms, uint32_t* scales, double* score) {
    const Plan plan = PlanScales(o->width, o->height);
    std::fill(norms, norms + 108, 0.0);
    if (precision == 64) {
        const auto r = ComputePair<double>(*o, *d, bg, filter, false, false, blur);
        ReadResult(r, plan, norms);
    } else {
        const auto r = ComputePair<float>(*o, *d, bg, filter, precision == 16,
                                          precision == 33, blur);
        ReadResult(r, plan, norms);
    }
    if (scales) *scales = static_cast<uint32_t>(plan.count);
    if (score) *score = Score(norms, plan.count);
    return SS2O_OK;
}

}  // namespace

extern "C" {

int ss2o_compute(const ss2o_image* original, const ss2o_image* distorted,
                 float background, int chroma_filter, int precision, int blur,
                 double* norms, uint32_t* scales, double* score) {
    try {
        return ComputeOne(original, distorted, background, chroma_filter,
                          precision, blur, norms, scales, score);
    } catch (const std::exception& e) {
        return Fail(e);
    }
}

int ss2o_compute_many(uint32_t n, const ss2o_image* originals,
                      const ss2o_image* distorteds, float background,
                      int chroma_filter, int precision, int blur, uint32_t threads,
                      double* norms, uint32_t* scales, double* scores) {
    std::atomic<uint32_t> next{0};
    std::atomic<int> status{SS2O_OK};
    std::string first_error;  // written once, by the thread that wins the CAS
    auto worker = [&]() {
        for (;;) {
            const uint32_t i = next.fetch_add(1);
            if (i >= n) return;
            try {
                ComputeOne(&originals[i], &distorteds[i], background, chroma_filter,
                           precision, blur, norms + size_t(i) * 108,
                           scales ? scales + i : nullptr, scores ? scores + i : nullptr);
            } catch (const std::exception& e) {
                int expected = SS2O_OK;
                if (status.compare_exchange_strong(expected, SS2O_INVALID))
                    first_error = e.what();
            }
        }
    };
    const uint32_t t = std::max<uint32_t>(1, std::min(threads, n));
    std::vector<std::thread> pool;
    for (uint32_t i = 1; i < t; ++i) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (status.load() != SS2O_OK) g_error = first_error;
    return status.load();
}

int ss2o_plan_scales(uint32_t width, uint32_t height, uint32_t* sizes12) {
    try {
        const Plan p = PlanScales(width, height);
        for (int i = 0; i < kMaxScales; ++i) {
            sizes12[2 * i] = i < p.count ? p.sizes[i].w : 0;
            sizes12[2 * i + 1] = i < p.count ? p.sizes[i].h : 0;
        }
        return p.count;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

void ss2o_gaussian(float* taps13) {
    const auto w = GaussianDouble();
    for (int i = 0; i < kTaps; ++i) taps13[i] = static_cast<float>(w[i]);
}

void ss2o_recursive_gaussian(int* radius, double* freqs3, double* beta3, double* taps13) {
    const RecursiveGauss g = MakeRecursiveGauss();
    const auto h = RecursiveTapsDouble();
    *radius = g.n;
    for (int k = 0; k < 3; ++k) {
        freqs3[k] = g.w[k];
        beta3[k] = g.beta[k];
    }
    for (int i = 0; i < kTaps; ++i) taps13[i] = h[i];
}

int ss2o_blur_plane(int blur, int precision, const double* in, uint32_t width,
                    uint32_t height, double* out) {
    try {
        if (blur != kBlurSampled && blur != kBlurRecursive)
            throw std::invalid_argument("unknown blur mode");
        const size_t n = size_t(width) * height;
        if (precision == 64) {
            std::vector<double> src(in, in + n), hq, dst;
            Blur2D<double>(src, hq, dst, width, height, Taps<double>(blur),
                           blur == kBlurRecursive);
            std::copy(dst.begin(), dst.end(), out);
        } else {
            std::vector<float> src(n), hq, dst;
            for (size_t i = 0; i < n; ++i) src[i] = static_cast<float>(in[i]);
            Blur2D<float>(src, hq, dst, width, height, Taps<float>(blur), false);
            for (size_t i = 0; i < n; ++i) out[i] = dst[i];
        }
        return SS2O_OK;
    } catch (const std::exception& e) {
        return Fail(e);
    }
}

int ss2o_channel_pruned(uint32_t channel, uint32_t scale, uint32_t scales) {
    return ChannelPruned(static_cast<int>(channel), static_cast<int>(scale),
                         static_cast<int>(scales)) ? 1 : 0;
}

int ss2o_score(const double* norms, uint32_t scales, double* score) {
    try {
        *score = Score(norms, static_cast<int>(scales));
        return SS2O_OK;
    } catch (const std::exception& e) {
        return Fail(e);
    }
}

int ss2o_required_bytes(const ss2o_format* format, uint32_t width,
                        uint32_t height, size_t* bytes) {
    try {
        *bytes = RequiredBytes(*format, width, height);
        return SS2O_OK;
    } catch (const std::exception& e) {
        return Fail(e);
    }
}

int ss2o_source_desc(const ss2o_format* format, int chroma_filter,
                     uint32_t* words) {
    try {
        const Desc d = BuildDesc(*format, chroma_filter);
        std::memset(words, 0, 44 * 4);
        words[4] = (uint32_t(format->type)) | (uint32_t(format->family) << 2) |
                   (uint32_t(format->alpha) << 4) |
                   (uint32_t(format->subsample_w) << 6) |
                   (uint32_t(format->subsample_h) << 8) |
                   (uint32_t(d.transfer) << 10) | (uint32_t(chroma_filter) << 15) |
                   (uint32_t(d.mode) << 17);
        words[5] = (d.identity1 ? 1u : 0u) | (d.identity2 ? 2u : 0u);
        auto put = [&](int i, float v) { std::memcpy(&words[i], &v, 4); };
        for (int i = 0; i < 3; ++i) {
            put(6 + i, d.scale_f[i]);
            put(9 + i, d.offset_f[i]);
        }
        for (int i = 0; i < 9; ++i) {
            put(12 + i, d.m1_f[i]);
            put(21 + i, d.m2_f[i]);
        }
        put(30, d.kr_f); put(31, d.kg_f); put(32, d.kb_f);
        put(33, d.to_linear_f);
        put(34, d.shift_x_f); put(35, d.shift_y_f);
        for (int i = 0; i < 4; ++i) put(36 + i, d.cl_f[i]);
        return SS2O_OK;
    } catch (const std::exception& e) {
        return Fail(e);
    }
}

int ss2o_pyramid(const ss2o_image* image, float background, int chroma_filter,
                 float* out, size_t capacity, size_t* count) {
    try {
        const Plan plan = PlanScales(image->width, image->height);
        const Desc d = BuildDesc(image->format, chroma_filter);
        Pyramid<float> p;
        BuildPyramid<float>(*image, d, background, plan, p);
        size_t total = 0;
        for (int l = 0; l < plan.count; ++l)
            total += size_t(3) * plan.sizes[l].w * plan.sizes[l].h;
        *count = total;
        if (out == nullptr) return SS2O_OK;
        if (capacity < total) throw std::invalid_argument("capacity too small");
        size_t at = 0;
        for (int l = 0; l < plan.count; ++l) {
            const size_t n = size_t(plan.sizes[l].w) * plan.sizes[l].h;
            for (int c = 0; c < 3; ++c) {
                if (p.planes[l][c].empty())
                    std::fill(out + at, out + at + n, std::numeric_limits<float>::quiet_NaN());
                else
                    std::copy(p.planes[l][c].begin(), p.planes[l][c].end(), out + at);
                at += n;
            }
        }
        return SS2O_OK;
    } catch (const std::exception& e) {
        return Fail(e);
    }
}

int ss2o_level_sums(const ss2o_image* original, const ss2o_image* distorted,
                    float background, int chroma_filter, float* sums,
                    uint32_t* scales) {
    try {
        const auto r = ComputePair<float>(*original, *distorted, background, chroma_filter);
        for (int l = 0; l < r.scales; ++l)
            for (int k = 0; k < 18; ++k) sums[l * 18 + k] = r.sums[l][k];
        *scales = static_cast<uint32_t>(r.scales);
        return SS2O_OK;
    } catch (const std::exception& e) {
        return Fail(e);
    }
}

int ss2o_detmath(int fn, const float* x, float y, float* out, size_t n) {
    for (size_t i = 0; i < n; ++i) {
        switch (fn) {
            case 0: out[i] = ss2dm::cbrt(x[i]); break;
            case 1: out[i] = ss2dm::pow(x[i], y); break;
            case 2: out[i] = ss2dm::exp(x[i]); break;
            case 3: out[i] = ss2dm::sinpi(x[i]); break;
            case 4: out[i] = RoundHalf(x[i]); break;
            case 5: out[i] = ss2dm::powf_gamma(x[i], y); break;
            case 6: out[i] = ss2dm::divf(x[i], y); break;
            default: g_error = "unknown function"; return SS2O_INVALID;
        }
    }
    return SS2O_OK;
}

const char* ss2o_last_error(void) { return g_error.c_str(); }

}  // extern "C"
