// Host-side format rules, decode constants, scale plan and score of the
// SSIMULACRA 2.1 scorer. The colour algebra keeps the operation order of the
// reference's src/input.cc (zimg's) so the FP32 constants it produces are
// bit-identical to the reference's; the tests compare them against input.cc
// itself compiled from source.

#include "ss2_host.h"

#include "ss2_detmath.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

namespace vqm_b200 {
namespace {

using Matrix3 = std::array<double, 9>;
using Vec3 = std::array<double, 3>;

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
int EffectiveDepth(const vqm_cu_format& f) { return f.depth != 0 ? f.depth : TypeDepth(f.type); }

bool KnownMatrix(uint8_t m) {
    return m <= 17 && m != 3;
}
bool KnownPrimaries(uint8_t p) {
    return (p >= 1 && p <= 12 && p != 3) || p == 22;
}

const char* TransferError(uint8_t t) {
    switch (t) {
        case 1: case 4: case 5: case 6: case 7: case 8: case 9: case 10: case 11:
        case 12: case 13: case 14: case 15: case 16: case 17: case 18:
            return nullptr;
        case 2:
            return "transfer characteristics are required";
    }
    return "unsupported transfer characteristics";
}

bool IsBt709Curve(uint8_t t) { return t == 1 || t == 6 || t == 14 || t == 15; }

const char* ModeError(const vqm_cu_format& f) {
    if (f.family == 0) return nullptr;
    switch (f.matrix) {
        case 0: case 2: case 1: case 4: case 5: case 6: case 7: case 8: case 9: case 12:
            break;
        case 10: case 13:
            if (!IsBt709Curve(f.transfer))
                return "constant-luminance matrix coefficients require the BT.709 transfer";
            break;
        case 14:
            if (!(f.transfer == 16 || f.transfer == 18) || f.primaries != 9)
                return "ICtCp requires the ST 2084 or ARIB B67 transfer and BT.2020 primaries";
            break;
        default:
            return "unsupported matrix coefficients";
    }
    if (f.family != 0 && f.primaries == 10) {
        const bool derived = f.matrix == 12 || f.matrix == 13;
        if (derived || f.transfer == 18)
            return "XYZ color primaries do not define the chromaticity this conversion needs";
    }
    return nullptr;
}

// ---- zimg colorimetry (input.cc:262-587), same operation order ----

double Det2(double a00, double a01, double a10, double a11) { return a00 * a11 - a01 * a10; }
Matrix3 Inverse(const Matrix3& m) {
    double det = 0.0;
    det += m[0] * Det2(m[4], m[5], m[7], m[8]);
    det -= m[1] * Det2(m[3], m[5], m[6], m[8]);
    det += m[2] * Det2(m[3], m[4], m[6], m[7]);
    Matrix3 r{};
    r[0] = Det2(m[4], m[5], m[7], m[8]) / det;
    r[1] = Det2(m[2], m[1], m[8], m[7]) / det;
    r[2] = Det2(m[1], m[2], m[4], m[5]) / det;
    r[3] = Det2(m[5], m[3], m[8], m[6]) / det;
    r[4] = Det2(m[0], m[2], m[6], m[8]) / det;
    r[5] = Det2(m[2], m[0], m[5], m[3]) / det;
    r[6] = Det2(m[3], m[4], m[6], m[7]) / det;
    r[7] = Det2(m[1], m[0], m[7], m[6]) / det;
    r[8] = Det2(m[0], m[1], m[3], m[4]) / det;
    return r;
}
Matrix3 Mul3(const Matrix3& a, const Matrix3& b) {
    Matrix3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 3; ++k) acc += a[i * 3 + k] * b[k * 3 + j];
            r[i * 3 + j] = acc;
        }
    return r;
}
Vec3 MulV(const Matrix3& m, const Vec3& v) {
    return {m[0] * v[0] + m[1] * v[1] + m[2] * v[2], m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
            m[6] * v[0] + m[7] * v[1] + m[8] * v[2]};
}
double Dot(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
Vec3 Cross(const Vec3& a, const Vec3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
Matrix3 Identity() { return {1, 0, 0, 0, 1, 0, 0, 0, 1}; }
Vec3 XyToXyz(double x, double y) { return {x / y, 1.0, (1.0 - x - y) / y}; }

struct Chromaticities {
    double xy[3][2];
};
bool PrimariesXy(uint8_t p, Chromaticities& out) {
    static const Chromaticities k470M{{{0.670, 0.330}, {0.210, 0.710}, {0.140, 0.080}}};
    static const Chromaticities k470Bg{{{0.640, 0.330}, {0.290, 0.600}, {0.150, 0.060}}};
    static const Chromaticities kSmpteC{{{0.630, 0.340}, {0.310, 0.595}, {0.155, 0.070}}};
    static const Chromaticities k709{{{0.640, 0.330}, {0.300, 0.600}, {0.150, 0.060}}};
    static const Chromaticities kFilm{{{0.681, 0.319}, {0.243, 0.692}, {0.145, 0.049}}};
    static const Chromaticities k2020{{{0.708, 0.292}, {0.170, 0.797}, {0.131, 0.046}}};
    static const Chromaticities kP3{{{0.680, 0.320}, {0.265, 0.690}, {0.150, 0.060}}};
    static const Chromaticities kEbu{{{0.630, 0.340}, {0.295, 0.605}, {0.155, 0.077}}};
    switch (p) {
        case 4: out = k470M; return true;
        case 5: out = k470Bg; return true;
        case 6: case 7: out = kSmpteC; return true;
        case 1: out = k709; return true;
        case 8: out = kFilm; return true;
        case 9: out = k2020; return true;
        case 11: case 12: out = kP3; return true;
        case 22: out = kEbu; return true;
    }
    return false;
}
Vec3 WhitePoint(uint8_t p) {
    switch (p) {
        case 4: case 8: return XyToXyz(0.31, 0.316);
        case 10: return XyToXyz(1.0 / 3.0, 1.0 / 3.0);
        case 11: return XyToXyz(0.314, 0.351);
        default: return XyToXyz(0.3127, 0.3290);
    }
}
Matrix3 PrimariesXyz(uint8_t p) {
    Chromaticities c;
    if (!PrimariesXy(p, c)) throw std::invalid_argument("color primaries do not define chromaticities");
    const Vec3 r = XyToXyz(c.xy[0][0], c.xy[0][1]);
    const Vec3 g = XyToXyz(c.xy[1][0], c.xy[1][1]);
    const Vec3 b = XyToXyz(c.xy[2][0], c.xy[2][1]);
    return {r[0], g[0], b[0], r[1], g[1], b[1], r[2], g[2], b[2]};
}
void KrKbFromPrimaries(uint8_t p, double& kr, double& kb) {
    if (p == 1) { kr = 0.2126; kb = 0.0722; return; }
    if (p == 9) { kr = 0.2627; kb = 0.0593; return; }
    Chromaticities c;
    if (!PrimariesXy(p, c)) throw std::invalid_argument("color primaries do not define chromaticities");
    const Vec3 r = XyToXyz(c.xy[0][0], c.xy[0][1]);
    const Vec3 g = XyToXyz(c.xy[1][0], c.xy[1][1]);
    const Vec3 b = XyToXyz(c.xy[2][0], c.xy[2][1]);
    const Vec3 white = WhitePoint(p);
    const double den = Dot({r[0], g[0], b[0]}, Cross({r[1], g[1], b[1]}, {r[2], g[2], b[2]}));
    kr = Dot(white, Cross(g, b)) / den;
    kb = Dot(white, Cross(r, g)) / den;
}
Matrix3 YuvFromKrKb(double kr, double kb) {
    const double kg = 1.0 - kr - kb;
    const double us = 1.0 / (2.0 - 2.0 * kb);
    const double vs = 1.0 / (2.0 - 2.0 * kr);
    return {kr, kg, kb, -kr * us, -kg * us, (1.0 - kb) * us, (1.0 - kr) * vs, -kg * vs, -kb * vs};
}
void KrKbFromMatrix(uint8_t m, double& kr, double& kb) {
    switch (m) {
        case 4: kr = 0.3; kb = 0.11; return;
        case 7: kr = 0.212; kb = 0.087; return;
        case 5: case 6: kr = 0.299; kb = 0.114; return;
        case 1: kr = 0.2126; kb = 0.0722; return;
        case 9: case 10: kr = 0.2627; kb = 0.0593; return;
    }
    throw std::invalid_argument("matrix coefficients have no luma weights");
}
Matrix3 RgbToYuv(uint8_t m) {
    if (m == 8) return {0.25, 0.5, 0.25, -0.25, 0.5, -0.25, 0.5, 0.0, -0.5};
    double kr = 0, kb = 0;
    KrKbFromMatrix(m, kr, kb);
    return YuvFromKrKb(kr, kb);
}
Matrix3 YuvToRgbFromPrimaries(uint8_t p) {
    if (p == 1) return Inverse(RgbToYuv(1));
    if (p == 9) return Inverse(RgbToYuv(9));
    double kr = 0, kb = 0;
    KrKbFromPrimaries(p, kr, kb);
    return Inverse(YuvFromKrKb(kr, kb));
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
    const Vec3 s = MulV(Inverse(m), WhitePoint(p));
    Matrix3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i * 3 + j] = m[i * 3 + j] * s[j];
    return r;
}
Matrix3 Gamut(uint8_t from, uint8_t to) {
    const Matrix3 to_rgb = to == 10 ? Identity() : Inverse(RgbToXyz(to));
    return Mul3(to_rgb, RgbToXyz(from));
}
Matrix3 LmsToRgb() {
    return Inverse({1688.0 / 4096.0, 2146.0 / 4096.0, 262.0 / 4096.0, 683.0 / 4096.0,
                    2951.0 / 4096.0, 462.0 / 4096.0, 99.0 / 4096.0, 309.0 / 4096.0,
                    3688.0 / 4096.0});
}
double Rec709Oetf(double x) {
    x = std::max(x, 0.0);
    return x < 0.018053968510807 ? x * 4.5
                                 : 1.09929682680944 * std::pow(x, 0.45) - (1.09929682680944 - 1.0);
}

int SelectMode(const vqm_cu_format& f) {
    if (f.family == 0) return 0;
    if (f.matrix == 10 || f.matrix == 13) return 1;
    if (f.matrix == 14) return 2;
    return 0;
}
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
void ScaleOffset(const vqm_cu_format& f, bool chroma, bool alpha, float& scale, float& offset) {
    const bool is_float = f.type == 2 || f.type == 3;
    const int depth = EffectiveDepth(f);
    if (depth < 1 || depth > TypeDepth(f.type))
        throw std::invalid_argument("invalid bit depth for pixel type");
    if (is_float) { scale = 1.0f; offset = 0.0f; return; }
    const bool full = alpha || f.range == 1;
    const bool ycgco = f.matrix == 8;
    const double numeric_max = static_cast<double>((1u << depth) - 1u);
    const double range =
        full ? numeric_max
             : static_cast<double>(chroma && !ycgco ? 224u << (depth - 8) : 219u << (depth - 8));
    double off = 0.0;
    if (alpha) off = 0.0;
    else if (chroma) off = static_cast<double>(1u << (depth - 1));
    else if (!full) off = static_cast<double>(16u << (depth - 8));
    scale = static_cast<float>(1.0 / range);
    offset = static_cast<float>(-off / range);
}
void LumaWeights(const vqm_cu_format& f, double& kr, double& kg, double& kb) {
    kr = 0.0; kg = 1.0; kb = 0.0;
    const int mode = SelectMode(f);
    if (f.family == 0) return;
    if (mode == 1) {
        if (f.matrix == 13) KrKbFromPrimaries(f.primaries, kr, kb);
        else KrKbFromMatrix(f.matrix, kr, kb);
    } else if (f.transfer == 18) {
        KrKbFromPrimaries(f.primaries, kr, kb);
    } else {
        return;
    }
    kg = 1.0 - kr - kb;
}

// The per-channel transfer decode in float, for the 8-bit table: the same
// formulas and rounding as the device path (ss2_decode.cuh) and color.glsl.
float HostPow(float a, float b) { return ss2dm::pow(a, b); }
float Rec709InvOetfF(float x) {
    x = std::max(x, 0.0f);
    const float alpha = 1.09929682680944f, beta = 0.018053968510807f;
    return x < 4.5f * beta ? x / 4.5f : HostPow((x + (alpha - 1.0f)) / alpha, 1.0f / 0.45f);
}
float St2084EotfF(float x) {
    if (x <= 0.0f) return 0.0f;
    const float xp = HostPow(x, 1.0f / 78.84375f);
    const float num = std::max(xp - 0.8359375f, 0.0f);
    const float den = std::max(18.8515625f - 18.6875f * xp, 1.17549435e-38f);
    return HostPow(num / den, 1.0f / 0.1593017578125f);
}
float TransferF(int id, float tl, float v) {
    switch (id) {
        case 0: return v;
        case 1: return v < 0.0f ? 0.0f : ss2dm::powf_gamma(v, 2.4f);
        case 2: return v < 0.0f ? 0.0f : ss2dm::powf_gamma(v, 2.2f);
        case 3: return v < 0.0f ? 0.0f : ss2dm::powf_gamma(v, 2.8f);
        case 4: return v <= 0.04045f ? v / 12.92f : HostPow((v + 0.055f) / 1.055f, 2.4f);
        case 5: return v <= 0.0f ? 0.01f : HostPow(10.0f, 2.0f * (v - 1.0f));
        case 6: return v <= 0.0f ? 0.00316227766f : HostPow(10.0f, 2.5f * (v - 1.0f));
        case 7:
            return v >= 0.0f && v <= 1.0f ? HostPow(v, 2.4f)
                                          : (v < 0.0f ? -Rec709InvOetfF(-v) : Rec709InvOetfF(v));
        case 8:
            if (v >= 0.0f && v <= 1.0f) return HostPow(v, 2.4f);
            return v >= 0.0f ? Rec709InvOetfF(v) : -Rec709InvOetfF(-4.0f * v) / 4.0f;
        case 9: return tl * St2084EotfF(v);
        case 10: return v < 0.0f ? 0.0f : (52.37f / 48.0f) * HostPow(v, 2.6f);
    }
    return v;
}

// score.cc:38-87.
const double kWeightTable[108] = {
    0.0, 0.0007376606707406586, 0.0, 0.0, 0.0007793481682867309, 0.0,
    0.0, 0.0004371155730107379, 0.0, 1.1041726426657346, 0.00066284834129271, 0.00015231632783718752,
    0.0, 0.0016406437456599754, 0.0, 1.8422455520539298, 11.441172603757666, 0.0,
    0.0007989109436015163, 0.000176816438078653, 0.0, 1.8787594979546387, 10.94906990605142, 0.0,
    0.0007289346991508072, 0.9677937080626833, 0.0, 0.00014003424285435884, 0.9981766977854967, 0.00031949755934435053,
    0.0004550992113792063, 0.0, 0.0, 0.0013648766163243398, 0.0, 0.0,
    0.0, 0.0, 0.0, 7.466890328078848, 0.0, 17.445833984131262,
    0.0006235601634041466, 0.0, 0.0, 6.683678146179332, 0.00037724407979611296, 1.027889937768264,
    225.20515300849274, 0.0, 0.0, 19.213238186143016, 0.0011401524586618361, 0.001237755635509985,
    176.39317598450694, 0.0, 0.0, 24.43300999870476, 0.28520802612117757, 0.0004485436923833408,
    0.0, 0.0, 0.0, 34.77906344483772, 44.835625328877896, 0.0,
    0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
    0.0, 0.0008680556573291698, 0.0, 0.0, 0.0, 0.0,
    0.0, 0.0005313191874358747, 0.0, 0.00016533814161379112, 0.0, 0.0,
    0.0, 0.0, 0.0, 0.0004179171803251336, 0.0017290828234722833, 0.0,
    0.0020827005846636437, 0.0, 0.0, 8.826982764996862, 23.19243343998926, 0.0,
    95.1080498811086, 0.9863978034400682, 0.9834382792465353, 0.0012286405048278493, 171.2667255897307, 0.9807858872435379,
    0.0, 0.0, 0.0, 0.0005130064588990679, 0.0, 0.00010854057858411537,
};

}  // namespace

std::array<PlaneGeometry, 4> PlaneLayout(const vqm_cu_format& f, uint32_t w, uint32_t h) {
    std::array<PlaneGeometry, 4> layout{};
    const size_t sb = SampleBytes(f.type);
    if (sb == 0) throw std::invalid_argument("invalid pixel type");
    if (f.subsample_w > 2 || f.subsample_h > 2)
        throw std::invalid_argument("subsampling greater than 4x is not supported");
    size_t cursor = 0;
    for (int p = 0; p < 4; ++p) {
        const bool chroma = p == 1 || p == 2;
        const bool present = p == 0 || (chroma && f.family != 0) || (p == 3 && f.alpha != 0);
        if (!present) continue;
        layout[p].width = chroma ? (w >> f.subsample_w) : w;
        layout[p].height = chroma ? (h >> f.subsample_h) : h;
        layout[p].sample_bytes = sb;
        layout[p].offset = cursor;
        cursor = (cursor + layout[p].width * layout[p].height * sb + 3) / 4 * 4;
    }
    return layout;
}

size_t RequiredBytes(const vqm_cu_format& f, uint32_t w, uint32_t h) {
    const auto layout = PlaneLayout(f, w, h);
    size_t total = 0;
    for (const auto& p : layout)
        if (p.present()) total = p.offset + p.width * p.height * p.sample_bytes;
    return (total + 3) / 4 * 4;
}

void ValidateFormat(const vqm_cu_format& f, uint32_t w, uint32_t h, const char* name) {
    const auto fail = [name](const char* message) {
        throw std::invalid_argument(std::string(name) + ": " + message);
    };
    if (SampleBytes(f.type) == 0) fail("invalid pixel type");
    if (f.range > 1) fail("invalid pixel range");
    if (f.alpha > 2) fail("invalid alpha type");
    if (f.chroma_location > 5) fail("invalid chroma location");
    if (!KnownMatrix(f.matrix)) fail("invalid matrix coefficients");
    if (!KnownPrimaries(f.primaries)) fail("invalid color primaries");
    const int depth = EffectiveDepth(f);
    if (f.depth > TypeDepth(f.type)) fail("bit depth exceeds the pixel type");
    if (f.subsample_w > 2 || f.subsample_h > 2) fail("subsampling greater than 4x is not supported");
    if (w % (1u << f.subsample_w) != 0 || h % (1u << f.subsample_h) != 0)
        fail("image dimensions must be divisible by the subsampling");
    if (f.range == 0 && depth < 8) fail("limited range requires a bit depth of at least 8");
    switch (f.family) {
        case 0:
            if (f.subsample_w != 0 || f.subsample_h != 0)
                fail("subsampled greyscale images are not supported");
            if (f.matrix == 0) fail("greyscale images cannot declare RGB matrix coefficients");
            break;
        case 1:
            if (f.subsample_w != 0 || f.subsample_h != 0) fail("subsampled RGB images are not supported");
            if (f.matrix != 0 && f.matrix != 2) fail("RGB images cannot declare YUV matrix coefficients");
            break;
        case 2:
            if (f.matrix == 0) fail("YUV images cannot declare RGB matrix coefficients");
            if (f.matrix == 2) fail("matrix coefficients are required for YUV input");
            break;
        default:
            fail("invalid color family");
    }
    if (const char* reason = TransferError(f.transfer)) fail(reason);
    if (f.family != 0 && f.primaries == 2) fail("color primaries are required");
    if (const char* reason = ModeError(f)) fail(reason);
}

namespace {

// The device's BilinearPhase (ss2_decode.cuh, color.glsl:288-299) in the
// same single-precision steps.
void HostBilinearPhase(uint32_t out_pos, float inv_scale, float shift, int centre, int& s0,
                       float& w0, float& w1) {
    const auto round_halfup = [](float x) {
        return x < 0.0f ? std::floor(x + 0.5f) : std::floor(x + 0.49999997f);
    };
    const float pos = (static_cast<float>(out_pos) + 0.5f) * inv_scale + shift;
    const float base = round_halfup(pos - 1.0f) + 0.5f;
    const float t = pos - base;
    s0 = static_cast<int>(std::floor(base)) - centre + 1;
    w0 = 1.0f - t;
    w1 = t;
}

// DevSource's YUV fast-path fields: set when the format qualifies and every
// block's bilinear phases are those of its parity (checked over block
// indices across the whole coordinate range).
// Sets the YUV fast path's constants (d.yuv_fast = 1 when it applies) and
// returns a bound on the magnitude of the YUV matrix's outputs over every
// sample code (infinity when the path does not apply).
double FastYuvConstants(const vqm_cu_format& f, int mode, int tid, uint32_t chroma_filter,
                        DevSource& d) {
    const double none = HUGE_VAL;
    d.yuv_fast = 0;
    d.chroma_pattern = 0;
    d.gamma = 0.0f;
    std::memset(d.cslot, 0, sizeof(d.cslot));
    std::memset(d.cweight, 0, sizeof(d.cweight));
    if (!(f.family == 2 && f.type <= 1 && f.alpha == 0 && mode == 0 && tid >= 1 && tid <= 3 &&
          f.subsample_w <= 1 && f.subsample_h <= 1 && (!d.chroma_variant || chroma_filter == 0)))
        return none;
    const float gammas[4] = {0.0f, 2.4f, 2.2f, 2.8f};  // TransferDecode cases 1-3
    d.gamma = gammas[tid];
    float w[2][2][2];  // [axis][parity][tap]
    static const uint32_t kBlocks[] = {0, 1, 2, 3, 5, 77, 1000, 4095, 16383, 32767};
    for (int axis = 0; axis < 2; ++axis) {
        const int sub = axis ? f.subsample_h : f.subsample_w;
        const float inv = 1.0f / static_cast<float>(1u << sub);
        const float shift = axis ? d.shift_y : d.shift_x;
        for (int par = 0; par < 2; ++par) {
            int s_ref = 0;
            float w0_ref = 0.0f, w1_ref = 0.0f;
            for (size_t k = 0; k < sizeof(kBlocks) / sizeof(kBlocks[0]); ++k) {
                const uint32_t b = kBlocks[k];
                int s0;
                float w0, w1;
                HostBilinearPhase(2 * b + par, inv, shift, static_cast<int>((2 * b) >> sub), s0,
                                  w0, w1);
                if (k == 0) {
                    s_ref = s0;
                    w0_ref = w0;
                    w1_ref = w1;
                } else if (s0 != s_ref || std::memcmp(&w0, &w0_ref, 4) ||
                           std::memcmp(&w1, &w1_ref, 4)) {
                    return none;
                }
            }
            // Slot 2 (an axis that is not subsampled) puts the second tap past
            // the 3x3 window, where the generic decode reads 0.
            if (s_ref < 0 || s_ref > 2) return none;
            d.cslot[axis][par] = static_cast<int8_t>(s_ref);
            w[axis][par][0] = w0_ref;
            w[axis][par][1] = w1_ref;
        }
    }
    // 4:2:0 axes whose phases are one of the two compiled patterns (the
    // device's ChromaFixed): offset 0 gives slots 0, 1 and weights
    // (1/4, 3/4), (3/4, 1/4); offset 1/4 gives slots 1, 1 and (1, 0),
    // (1/2, 1/2).
    d.chroma_pattern = 0;
    if (f.subsample_w == 1 && f.subsample_h == 1) {
        int type[2] = {-1, -1};
        for (int axis = 0; axis < 2; ++axis) {
            const auto is = [&](int s0, float a0, float b0, int s1, float a1, float b1) {
                return d.cslot[axis][0] == s0 && w[axis][0][0] == a0 && w[axis][0][1] == b0 &&
                       d.cslot[axis][1] == s1 && w[axis][1][0] == a1 && w[axis][1][1] == b1;
            };
            if (is(0, 0.25f, 0.75f, 1, 0.75f, 0.25f)) type[axis] = 0;
            else if (is(1, 1.0f, 0.0f, 1, 0.5f, 0.5f)) type[axis] = 1;
        }
        if (type[0] >= 0 && type[1] >= 0)
            d.chroma_pattern = static_cast<uint8_t>(1 + type[0] + 2 * type[1]);
    }
    for (int yp = 0; yp < 2; ++yp)
        for (int xp = 0; xp < 2; ++xp) {
            // BilinearTap's products, in single precision.
            d.cweight[yp][xp][0] = w[0][xp][0] * w[1][yp][0];
            d.cweight[yp][xp][1] = w[0][xp][1] * w[1][yp][0];
            d.cweight[yp][xp][2] = w[0][xp][0] * w[1][yp][1];
            d.cweight[yp][xp][3] = w[0][xp][1] * w[1][yp][1];
        }
    // The device's two-lane power takes every input from 2^-30 up without a
    // range check: every sample code the container can hold (whatever the
    // declared depth) must keep the YUV matrix's outputs below the power's
    // fast-range limit (with a margin for their float rounding). Valid
    // formats stay far below it (|R'G'B'| < 5; 9-bit codes filling 16 bits
    // reach a few hundred).
    const double code_max = f.type == 0 ? 255.0 : 65535.0;
    double lim[3];
    for (int p = 0; p < 3; ++p) {
        const int q = p == 0 ? 0 : 1;
        lim[p] = std::max(std::fabs(static_cast<double>(d.offset[q])),
                          std::fabs(code_max * d.scale[q] + d.offset[q]));
    }
    double max_bound = 0.0;
    for (int row = 0; row < 3; ++row) {
        double bound = d.identity1 ? lim[row] : 0.0;
        if (!d.identity1)
            for (int j = 0; j < 3; ++j)
                bound += std::fabs(static_cast<double>(d.m1[3 * row + j])) * lim[j];
        if (!(bound < 0.5 * ss2dm::kGammaMaxX)) return none;
        max_bound = std::max(max_bound, bound);
    }
    d.yuv_fast = 1;
    return max_bound;
}

}  // namespace

void BuildSourceConstants(const vqm_cu_format& f, uint32_t chroma_filter, float background,
                          DevSource& d) {
    d.type = f.type;
    d.family = f.family;
    d.alpha = f.alpha;
    d.sub_w = f.subsample_w;
    d.sub_h = f.subsample_h;
    const int mode = SelectMode(f);
    d.mode = static_cast<uint8_t>(mode);
    int tid = 0;
    float tls = 1.0f;
    SelectTransfer(f.transfer, tid, tls);
    d.transfer = static_cast<uint8_t>(tid);
    d.to_linear = tls;
    d.filter = static_cast<uint8_t>(chroma_filter);
    d.chroma_variant = (f.subsample_w != 0 || f.subsample_h != 0) ? 1 : 0;
    ScaleOffset(f, false, false, d.scale[0], d.offset[0]);
    ScaleOffset(f, f.family == 2, false, d.scale[1], d.offset[1]);
    ScaleOffset(f, false, true, d.scale[2], d.offset[2]);
    Matrix3 m1 = Identity();
    bool id1 = true;
    if (mode == 1) {
        id1 = true;
    } else if (mode == 2) {
        m1 = Inverse(LmsToIctCp(f.transfer));
        id1 = false;
    } else if (f.family != 0 && f.matrix != 0 && f.matrix != 2) {
        m1 = f.matrix == 12 ? YuvToRgbFromPrimaries(f.primaries) : Inverse(RgbToYuv(f.matrix));
        id1 = false;
    }
    Matrix3 m2 = Identity();
    bool id2 = true;
    if (f.family == 0 || f.primaries == 1) {
        id2 = true;
    } else if (mode == 2) {
        m2 = Mul3(Gamut(f.primaries, 1), LmsToRgb());
        id2 = false;
    } else {
        m2 = Gamut(f.primaries, 1);
        id2 = false;
    }
    for (int i = 0; i < 9; ++i) {
        d.m1[i] = static_cast<float>(m1[i]);
        d.m2[i] = static_cast<float>(m2[i]);
    }
    d.identity1 = id1 ? 1 : 0;
    d.identity2 = id2 ? 1 : 0;
    double kr, kg, kb;
    LumaWeights(f, kr, kg, kb);
    d.kr = static_cast<float>(kr);
    d.kg = static_cast<float>(kg);
    d.kb = static_cast<float>(kb);
    double sx = 0.0, sy = 0.0;
    if (f.family == 2 && d.chroma_variant) {
        // vulkan_source.cc:44-73: zimg's chroma offsets, negated.
        const double rw = 1.0 / static_cast<double>(1u << f.subsample_w);
        const double rh = 1.0 / static_cast<double>(1u << f.subsample_h);
        const double left = 0.5 - 0.5 * rw, top = 0.5 - 0.5 * rh, bottom = -(0.5 - 0.5 * rh);
        switch (f.chroma_location) {
            case 0: sx = left; break;
            case 2: sx = left; sy = top; break;
            case 3: sy = top; break;
            case 4: sx = left; sy = bottom; break;
            case 5: sy = bottom; break;
            default: break;
        }
    }
    d.shift_x = static_cast<float>(sx);
    d.shift_y = static_cast<float>(sy);
    for (int i = 0; i < 4; ++i) d.cl[i] = 0.0f;
    if (mode == 1) {
        d.cl[0] = static_cast<float>(Rec709Oetf(1.0 - kb));
        d.cl[1] = static_cast<float>(1.0 - Rec709Oetf(kb));
        d.cl[2] = static_cast<float>(Rec709Oetf(1.0 - kr));
        d.cl[3] = static_cast<float>(1.0 - Rec709Oetf(kr));
    }
    d.background = background;
    const double yuv_bound = FastYuvConstants(f, mode, tid, chroma_filter, d);
    // 8-bit grey/RGB without alpha: every sample decodes independently of its
    // neighbours, so one table per image holds the whole transfer decode.
    d.lut = (f.type == 0 && (f.family == 0 || f.family == 1) && f.alpha == 0 && mode == 0 &&
             tid != 11)
                ? 1
                : 0;
    // Power-law YUV without a primaries matrix: the transfer maps every
    // value to >= 0, and the matrix's output bound caps the linear values
    // (its power, with room for the power's rounding).
    d.in_range = d.yuv_fast && d.identity2 &&
                         std::pow(yuv_bound, static_cast<double>(d.gamma)) * (1.0 + 1e-6) <=
                             static_cast<double>(kInRangeLinearMax)
                     ? 1
                     : 0;
    if (!d.lut) {
        std::memset(d.srgb_lut, 0, sizeof(d.srgb_lut));
        return;
    }
    // The table depends only on the transfer and the luma scale and offset;
    // it is built once per distinct triple and reused.
    static std::mutex mu;
    static std::map<std::array<uint32_t, 4>, std::array<float, 256>> cache;
    uint32_t sb, ob, tb;
    std::memcpy(&sb, &d.scale[0], 4);
    std::memcpy(&ob, &d.offset[0], 4);
    std::memcpy(&tb, &tls, 4);
    const std::array<uint32_t, 4> key{static_cast<uint32_t>(tid), sb, ob, tb};
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it == cache.end()) {
        std::array<float, 256> table{};
        for (int v = 0; v < 256; ++v)
            table[v] = TransferF(tid, tls, std::fma(static_cast<float>(v), d.scale[0], d.offset[0]));
        it = cache.emplace(key, table).first;
    }
    std::memcpy(d.srgb_lut, it->second.data(), sizeof(d.srgb_lut));
    // Non-negative linear samples (and averages of them) mixed by the
    // all-positive opsin rows plus the bias stay in the cube root's direct
    // range; a primaries matrix could make them negative.
    bool in_range = d.identity2 != 0;
    for (float v : d.srgb_lut) in_range = in_range && v >= 0.0f && v <= kInRangeLinearMax;
    d.in_range = in_range ? 1 : 0;
}

bool ChannelPruned(int channel, int scale, int scales) {
    if (channel >= 3 || scale >= scales || scales > kMaxLevels) return false;
    const double* w = kWeightTable + (channel * scales + scale) * 6;
    double m = w[0];
    for (int i = 1; i < 6; ++i) m = std::max(m, w[i]);
    return m <= 0.01;
}

ScalePlan PlanScales(uint32_t width, uint32_t height) {
    if (width < kMinDimension || height < kMinDimension)
        throw std::invalid_argument("minimum image size is 8x8 pixels");
    ScalePlan plan;
    uint32_t w = width, h = height;
    while (plan.count < kMaxLevels && w >= kMinDimension && h >= kMinDimension) {
        if (plan.count != 0) {
            w = w / 2 + w % 2;
            h = h / 2 + h % 2;
        }
        plan.w[plan.count] = w;
        plan.h[plan.count] = h;
        ++plan.count;
    }
    for (int l = 0; l < plan.count; ++l) {
        plan.mask[l] = 0;
        for (int c = 0; c < 3; ++c)
            if (!ChannelPruned(c, l, plan.count)) plan.mask[l] |= 1u << c;
    }
    return plan;
}

std::array<float, kTaps> GaussianTaps() {
    double w[kTaps];
    double sum = 0.0;
    for (int i = 0; i < kTaps; ++i) {
        const double offset = static_cast<double>(i) - kRadius;
        w[i] = std::exp(-0.5 * (offset / 1.5) * (offset / 1.5));
        sum += w[i];
    }
    std::array<float, kTaps> out{};
    for (int i = 0; i < kTaps; ++i) out[i] = static_cast<float>(w[i] / sum);
    return out;
}

// Cloudinary's ssimulacra2 (github.com/cloudinary/ssimulacra2, 81feacf6)
// blurs with libjxl's recursive Gaussian (lib/jxl/gauss_blur.cc at libjxl
// e47d2a2b), the third-order method of D. Charalampidis, "Recursive
// Implementation of the Gaussian Filter Using Truncated Cosine Functions",
// IEEE Trans. Signal Processing 64(14), 2016. Restated here from the method:
//
// - window half-width N = nearest integer to 3.2795 sigma + 0.2546 (5 for
//   sigma 1.5) and frequencies w_k = (2k + 1) pi / (2N), k = 0, 1, 2, so
//   that cos(w_k N) = 0;
// - impulse response h(m) = sum_k beta_k cos(w_k m) for |m| <= N, 0 outside
//   (h(+-N) = 0 too, so 2N - 1 = 9 taps are nonzero);
// - beta: unit gain (sum_m h(m) = 1) and variance sigma^2
//   (sum_m m^2 h(m) = sigma^2), and of the coefficient vectors that meet both
//   the one closest to the Gaussian's cosine-series coefficients
//   rho_k = exp(-sigma^2 w_k^2 / 2) / N.
//
// Its recursion runs, for each k, S_k[n] = 2 cos(w_k) S_k[n-1] - S_k[n-2]
// + (-1)^k sin(w_k) (x[n+N-1] + x[n-N-1]) from zero state over zero-padded
// input, with y[n] = sum_k beta_k S_k[n]: exactly the zero-padded
// convolution with h (the windowed cosine times 1 - 2 cos(w) z^-1 + z^-2
// leaves only the two boundary terms). The kernels evaluate that
// convolution directly with these taps, rounded to float once as VQM rounds
// its sampled taps; the oracle's FP64 mode runs the recursion itself.
std::array<float, kTaps> RecursiveGaussianTaps() {
    constexpr double kPi = 3.14159265358979323846;
    const double sigma = 1.5;
    const int n = static_cast<int>(std::lround(3.2795 * sigma + 0.2546));
    static_assert(kRadius >= 5, "the recursive Gaussian's support fits the taps");
    double w[3], rho[3], p[2][3];
    for (int k = 0; k < 3; ++k) {
        w[k] = (2 * k + 1) * kPi / (2.0 * n);
        rho[k] = std::exp(-0.5 * sigma * sigma * w[k] * w[k]) / n;
        p[0][k] = p[1][k] = 0.0;
        for (int m = -n; m <= n; ++m) {
            const double c = std::cos(w[k] * m);
            p[0][k] += c;
            p[1][k] += static_cast<double>(m) * m * c;
        }
    }
    // beta = rho + P^T (P P^T)^-1 (g - P rho): the nearest point to rho on
    // the two constraints P beta = g = (1, sigma^2).
    const double g[2] = {1.0, sigma * sigma};
    double r[2], a[2][2];
    for (int i = 0; i < 2; ++i) {
        r[i] = g[i];
        for (int k = 0; k < 3; ++k) r[i] -= p[i][k] * rho[k];
        for (int j = 0; j < 2; ++j) {
            a[i][j] = 0.0;
            for (int k = 0; k < 3; ++k) a[i][j] += p[i][k] * p[j][k];
        }
    }
    const double det = a[0][0] * a[1][1] - a[0][1] * a[1][0];
    const double l0 = (a[1][1] * r[0] - a[0][1] * r[1]) / det;
    const double l1 = (a[0][0] * r[1] - a[1][0] * r[0]) / det;
    double beta[3];
    for (int k = 0; k < 3; ++k) beta[k] = rho[k] + p[0][k] * l0 + p[1][k] * l1;
    std::array<float, kTaps> out{};
    for (int m = -(n - 1); m <= n - 1; ++m) {
        double h = 0.0;
        for (int k = 0; k < 3; ++k) h += beta[k] * std::cos(w[k] * m);
        out[m + kRadius] = static_cast<float>(h);
    }
    return out;
}

std::array<float, kTaps> BlurTaps(uint32_t blur) {
    if (blur == VQM_CU_SS2_BLUR_SAMPLED) return GaussianTaps();
    if (blur == VQM_CU_SS2_BLUR_RECURSIVE) return RecursiveGaussianTaps();
    throw std::invalid_argument("Ssimulacra2Config: unknown blur mode");
}

const double* ScoreWeights() { return kWeightTable; }

double Score(const double* norms, int scales) {
    if (scales > kMaxLevels) throw std::invalid_argument("Ssimulacra2Result has too many scales");
    double error = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int s = 0; s < scales; ++s) {
            const double* w = kWeightTable + (c * scales + s) * 6;
            const double* ssim = norms + s * 18;
            const double* edge = norms + s * 18 + 6;
            error += w[0] * std::abs(ssim[c * 2 + 0]);
            error += w[1] * std::abs(edge[c * 4 + 0]);
            error += w[2] * std::abs(edge[c * 4 + 2]);
            error += w[3] * std::abs(ssim[c * 2 + 1]);
            error += w[4] * std::abs(edge[c * 4 + 1]);
            error += w[5] * std::abs(edge[c * 4 + 3]);
        }
    if (!std::isfinite(error))
        throw std::invalid_argument("Ssimulacra2Result contains nonfinite or overflowing norms");
    const double scaled = error * 0.9562382616834844;
    const double mapped = 2.326765642916932 * scaled - 0.020884521182843837 * scaled * scaled +
                          6.248496625763138e-05 * scaled * scaled * scaled;
    if (!std::isfinite(mapped)) throw std::invalid_argument("Ssimulacra2Result score mapping overflowed");
    if (mapped > 0.0) return 100.0 - 10.0 * std::pow(mapped, 0.6276336467831387);
    return 100.0;
}

}  // namespace vqm_b200
