// The host code of the library (vqm_b200/csrc/ss2_host.cc: formats, layout,
// decode constants, scale plan, taps, score) and the CPU oracle, built with
// AddressSanitizer and UndefinedBehaviorSanitizer by tests/test_sanitizers.py
// and run over odd sizes, every pixel type and family, alpha, chroma
// subsampling and filters, both blur modes and the three oracle precisions.
// Any report aborts the run (-fno-sanitize-recover); it prints "sanitize ok".
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../oracle/ss2_oracle.h"
#include "../../vqm_b200/csrc/ss2_host.h"

namespace {

uint64_t g_state = 0x9E3779B97F4A7C15ull;
uint32_t Next() {
    g_state ^= g_state << 13;
    g_state ^= g_state >> 7;
    g_state ^= g_state << 17;
    return static_cast<uint32_t>(g_state >> 11);
}

uint16_t HalfOf(float v) {  // v in [0, 1]: a normal or zero binary16 by truncation
    if (v <= 0.0f) return 0;
    uint32_t b;
    std::memcpy(&b, &v, 4);
    const int e = static_cast<int>((b >> 23) & 255) - 127 + 15;
    if (e <= 0) return 0;
    return static_cast<uint16_t>((e << 10) | ((b >> 13) & 1023));
}

// Random samples of a valid format, each plane filled within its range.
std::vector<uint8_t> Pixels(const vqm_cu_format& f, uint32_t w, uint32_t h) {
    std::vector<uint8_t> data(vqm_b200::RequiredBytes(f, w, h), 0);
    const auto layout = vqm_b200::PlaneLayout(f, w, h);
    const int depth = f.depth ? f.depth : (f.type == 0 ? 8 : 16);
    for (const auto& g : layout) {
        if (!g.present()) continue;
        for (size_t i = 0; i < g.width * g.height; ++i) {
            uint8_t* at = data.data() + g.offset + i * g.sample_bytes;
            const float u = static_cast<float>(Next() % 1000001u) / 1000000.0f;
            if (f.type == 0) {
                *at = static_cast<uint8_t>(Next() & 255u);
            } else if (f.type == 1) {
                const uint16_t v = static_cast<uint16_t>(Next() & ((1u << depth) - 1u));
                std::memcpy(at, &v, 2);
            } else if (f.type == 2) {
                const uint16_t v = HalfOf(u);
                std::memcpy(at, &v, 2);
            } else {
                std::memcpy(at, &u, 4);
            }
        }
    }
    return data;
}

ss2o_image OracleImage(const vqm_cu_format& f, uint32_t w, uint32_t h,
                       const std::vector<uint8_t>& data) {
    ss2o_image img{};
    img.width = w;
    img.height = h;
    std::memcpy(&img.format, &f, sizeof(f));
    img.data = data.data();
    img.bytes = data.size();
    return img;
}

vqm_cu_format Format(uint8_t type, uint8_t family, uint8_t alpha, uint8_t range, uint8_t matrix,
                     uint8_t transfer, uint8_t primaries, uint8_t sub_w, uint8_t sub_h,
                     uint8_t depth, uint8_t location = 0) {
    vqm_cu_format f{};
    f.type = type;
    f.family = family;
    f.alpha = alpha;
    f.range = range;
    f.matrix = matrix;
    f.transfer = transfer;
    f.primaries = primaries;
    f.chroma_location = location;
    f.subsample_w = sub_w;
    f.subsample_h = sub_h;
    f.depth = depth;
    return f;
}

int failures = 0;

void Expect(bool ok, const char* what) {
    if (!ok) {
        std::fprintf(stderr, "FAIL: %s\n", what);
        ++failures;
    }
}

}  // namespace

int main() {
    // Formats: sRGB bytes; straight-alpha floats; premultiplied halves;
    // grey words; 10-bit 4:2:0 BT.709; 12-bit 4:2:2 BT.2020 HLG; 4:4:4 PQ
    // with alpha; 4:1:1 bytes with BT.601 primaries; ICtCp; constant
    // luminance; xvYCC.
    const std::vector<vqm_cu_format> formats = {
        Format(0, 1, 0, 1, 0, 13, 1, 0, 0, 0),
        Format(3, 1, 1, 1, 0, 13, 1, 0, 0, 0),
        Format(2, 1, 2, 1, 0, 8, 1, 0, 0, 0),
        Format(1, 0, 0, 1, 1, 13, 1, 0, 0, 16),
        Format(1, 2, 0, 0, 1, 1, 1, 1, 1, 10),
        Format(1, 2, 0, 0, 9, 18, 9, 1, 0, 12, 2),
        Format(1, 2, 1, 1, 9, 16, 9, 0, 0, 10),
        Format(0, 2, 0, 0, 6, 6, 6, 2, 0, 0),
        Format(1, 2, 0, 0, 14, 16, 9, 1, 1, 12),
        Format(1, 2, 0, 0, 10, 14, 9, 1, 1, 10, 4),
        Format(0, 2, 0, 0, 1, 11, 1, 1, 1, 0),
    };
    const uint32_t sizes[][2] = {{8, 8}, {13, 9}, {33, 17}, {64, 36}, {65, 65}};
    int scored = 0, rejected = 0;
    for (const auto& s : sizes) {
        const vqm_b200::ScalePlan plan = vqm_b200::PlanScales(s[0], s[1]);
        Expect(plan.count >= 1 && plan.count <= 6, "scale plan");
        for (const auto& f : formats) {
            try {
                vqm_b200::ValidateFormat(f, s[0], s[1], "image");
            } catch (const std::invalid_argument&) {
                ++rejected;  // odd sizes with subsampled chroma
                continue;
            }
            for (uint32_t filter = 0; filter < 3; ++filter) {
                vqm_b200::DevSource src{};
                vqm_b200::BuildSourceConstants(f, filter, 0.25f, src);
            }
            const std::vector<uint8_t> a = Pixels(f, s[0], s[1]), b = Pixels(f, s[0], s[1]);
            const ss2o_image oa = OracleImage(f, s[0], s[1], a), ob = OracleImage(f, s[0], s[1], b);
            for (int precision : {32, 64, 16})
                for (int blur : {0, 1}) {
                    double norms[108], score = 0.0;
                    uint32_t scales = 0;
                    const int rc = ss2o_compute(&oa, &ob, 0.3f, (precision / 16) % 3, precision,
                                                blur, norms, &scales, &score);
                    // High-dynamic-range linear light overflows binary16
                    // planes: the half-plane score is then rejected as
                    // nonfinite, as VQM's Score rejects it.
                    if (rc != SS2O_OK && precision == 16) continue;
                    if (rc != SS2O_OK || scales != static_cast<uint32_t>(plan.count)) {
                        std::fprintf(stderr, "FAIL: oracle compute %ux%u type %d family %d "
                                     "precision %d blur %d: rc %d scales %u of %d\n",
                                     s[0], s[1], f.type, f.family, precision, blur, rc, scales,
                                     plan.count);
                        ++failures;
                        continue;
                    }
                    double host = vqm_b200::Score(norms, static_cast<int>(scales));
                    Expect(!(std::isfinite(score) && std::isfinite(host)) ||
                               std::fabs(host - score) < 1e-9,
                           "host score equals the oracle's");
                    ++scored;
                }
            double identity_norms[108], identity = 0.0;
            uint32_t scales = 0;
            Expect(ss2o_compute(&oa, &oa, 0.5f, 0, 32, 0, identity_norms, &scales, &identity) ==
                           SS2O_OK &&
                       identity == 100.0,
                   "identity scores 100");
        }
    }
    for (uint32_t blur : {0u, 1u}) {
        const auto taps = vqm_b200::BlurTaps(blur);
        double sum = 0.0;
        for (float t : taps) sum += t;
        Expect(std::fabs(sum - 1.0) < 1e-5, "taps sum to one");
    }
    bool threw = false;
    try {
        (void)vqm_b200::BlurTaps(7);
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    Expect(threw, "an unknown blur mode throws");
    std::printf("scored %d, rejected %d\n", scored, rejected);
    if (failures) return 1;
    std::printf("sanitize ok\n");
    return 0;
}
