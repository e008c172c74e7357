// Exercises include/vqm_cuda.hpp the way a VQM C++ caller would.
//
//   facade_check host   checks that need no device (sizes, Score, errors)
//   facade_check gpu    scores the 32x32 gradient pairs (tests/support.h
//                       MakeGradient) through Pipeline, Upload and Pool and
//                       prints one JSON object per result on stdout
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "vqm_cuda.hpp"

namespace v = vqm::cuda;

namespace {

int failures = 0;

void Expect(bool ok, const char* what) {
    if (!ok) {
        std::fprintf(stderr, "FAIL: %s\n", what);
        ++failures;
    }
}

template <class E, class F>
void ExpectThrow(F&& f, const char* what) {
    try {
        f();
    } catch (const E&) {
        return;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "FAIL: %s threw the wrong type: %s\n", what, e.what());
        ++failures;
        return;
    }
    std::fprintf(stderr, "FAIL: %s did not throw\n", what);
    ++failures;
}

v::ImageFormat Srgb8() {
    v::ImageFormat f;
    f.type = v::PixelType::Byte;
    return f;
}

// MakeGradient (tests/support.h:259-289): 0 gradient, 1 checkerboard +16
// red, 2 3-bit truncation.
v::Image Gradient(int variant) {
    const int side = 32;
    v::Image img;
    img.size = {side, side};
    img.format = Srgb8();
    img.data.resize(3 * side * side);
    for (int y = 0; y < side; ++y)
        for (int x = 0; x < side; ++x) {
            int r = x * 255 / (side - 1), g = y * 255 / (side - 1);
            int b = ((x * 7 + y * 11) * 13) & 255;
            if (variant == 1 && ((x + y) & 1) == 0) r = std::min(r + 16, 255);
            if (variant == 2) { r &= 0xF8; g &= 0xF8; b &= 0xF8; }
            const int i = y * side + x;
            img.data[i] = static_cast<std::uint8_t>(r);
            img.data[side * side + i] = static_cast<std::uint8_t>(g);
            img.data[2 * side * side + i] = static_cast<std::uint8_t>(b);
        }
    return img;
}

void Print(const char* path, int variant, const v::Ssimulacra2Result& r) {
    std::printf("{\"path\": \"%s\", \"variant\": %d, \"score\": %.17g, \"norms\": [", path,
                variant, r.Score());
    bool first = true;
    for (const auto& s : r.scales) {
        for (double n : s.avg_ssim) { std::printf(first ? "%.17g" : ", %.17g", n); first = false; }
        for (double n : s.avg_edgediff) std::printf(", %.17g", n);
    }
    std::printf("]}\n");
}

// image_view_test.cc:17-83: CopyImage packs padded planes, each plane's
// tail zero up to a 4-byte boundary.
void Views() {
    std::array<std::array<std::byte, 10>, 3> planes{};
    for (std::size_t p = 0; p < 3; ++p)
        for (std::size_t y = 0; y < 2; ++y)
            for (std::size_t x = 0; x < 3; ++x)
                planes[p][y * 5 + x] = static_cast<std::byte>(p * 20 + y * 3 + x + 1);
    v::ImageView view;
    view.size = {3, 2};
    view.format = Srgb8();
    for (std::size_t p = 0; p < 3; ++p) view.planes[p] = {planes[p].data(), 5};
    const v::Image image = v::CopyImage(view);
    Expect(image.size == view.size &&
               image.data == std::vector<std::uint8_t>({1, 2, 3, 4, 5, 6, 0, 0, 21, 22, 23, 24,
                                                        25, 26, 0, 0, 41, 42, 43, 44, 45, 46,
                                                        0, 0}),
           "CopyImage of padded planes");
    std::array<std::byte, 24> y{}, alpha{};
    std::array<std::byte, 8> u{}, w{};
    for (std::size_t r = 0; r < 4; ++r)
        for (std::size_t c = 0; c < 4; ++c) {
            y[r * 6 + c] = static_cast<std::byte>(r * 4 + c);
            alpha[r * 6 + c] = static_cast<std::byte>(200 + r * 4 + c);
        }
    for (std::size_t r = 0; r < 2; ++r)
        for (std::size_t c = 0; c < 2; ++c) {
            u[r * 4 + c] = static_cast<std::byte>(30 + r * 2 + c);
            w[r * 4 + c] = static_cast<std::byte>(60 + r * 2 + c);
        }
    v::ImageView yuv;
    yuv.size = {4, 4};
    yuv.format.type = v::PixelType::Byte;
    yuv.format.family = v::ColorFamily::Yuv;
    yuv.format.alpha = v::AlphaType::Straight;
    yuv.format.matrix = v::MatrixCoefficients::Bt709;
    yuv.format.subsample_w = yuv.format.subsample_h = 1;
    yuv.planes = {{{y.data(), 6}, {u.data(), 4}, {w.data(), 4}, {alpha.data(), 6}}};
    std::vector<std::uint8_t> want;
    for (int i = 0; i < 16; ++i) want.push_back(static_cast<std::uint8_t>(i));
    for (int i : {30, 31, 32, 33, 60, 61, 62, 63}) want.push_back(static_cast<std::uint8_t>(i));
    for (int i = 0; i < 16; ++i) want.push_back(static_cast<std::uint8_t>(200 + i));
    Expect(v::CopyImage(yuv).data == want, "CopyImage of subsampled planes and alpha");
    v::ImageView short_stride = view;
    short_stride.planes[1].stride_bytes = 2;
    ExpectThrow<std::invalid_argument>([&] { (void)v::CopyImage(short_stride); },
                                       "a short stride");
    v::ImageView missing = view;
    missing.planes[2].data = nullptr;
    ExpectThrow<std::invalid_argument>([&] { (void)v::CopyImage(missing); }, "a missing plane");
    v::ImageView empty = view;
    empty.size = {0, 2};
    ExpectThrow<std::invalid_argument>([&] { (void)v::CopyImage(empty); }, "an empty view");
}

void Host() {
    Views();
    Expect(v::RequiredBytes(Srgb8(), {32, 32}) == 3 * 32 * 32, "RequiredBytes srgb8");
    v::ImageFormat yuv;
    yuv.type = v::PixelType::Word;
    yuv.family = v::ColorFamily::Yuv;
    yuv.range = v::PixelRange::Limited;
    yuv.matrix = v::MatrixCoefficients::Bt709;
    yuv.transfer = v::TransferCharacteristics::Bt709;
    yuv.subsample_w = yuv.subsample_h = 1;
    yuv.depth = 10;
    Expect(v::RequiredBytes(yuv, {64, 32}) == 64 * 32 * 2 + 2 * 32 * 16 * 2,
           "RequiredBytes yuv420 10-bit");
    ExpectThrow<std::invalid_argument>([&] { v::ValidateFormat(yuv, {63, 32}, "original"); },
                                       "odd width with 4:2:0");

    v::Ssimulacra2Result perfect;
    perfect.scales.resize(6);
    Expect(perfect.Score() == 100.0, "all-zero norms score 100");
    v::Ssimulacra2Result seven;
    seven.scales.resize(7);
    ExpectThrow<std::invalid_argument>([&] { (void)seven.Score(); }, "seven scales");
    v::Ssimulacra2Result bad;
    bad.scales.resize(1);
    bad.scales[0].avg_ssim[0] = NAN;
    ExpectThrow<std::invalid_argument>([&] { (void)bad.Score(); }, "nonfinite norm");

    v::MetricsConfig none;
    none.size = {32, 32};
    ExpectThrow<std::invalid_argument>([&] { v::Metrics m(none); }, "no metric selected");

    v::Ssimulacra2Config unknown;
    unknown.size = {32, 32};
    unknown.blur = static_cast<v::Ssimulacra2Blur>(7);
    ExpectThrow<std::invalid_argument>([&] { v::Ssimulacra2Pipeline p(unknown); },
                                       "unknown blur mode");
}

void GpuMetrics() {
    v::MetricsConfig mc;
    mc.size = {32, 32};
    mc.original_format = mc.distorted_format = Srgb8();
    mc.ssimulacra2 = v::Ssimulacra2Config{};
    v::Metrics metrics(mc);
    const v::Image base = Gradient(0);
    // metrics_test.cc:376-411: SSIMULACRA 2 alone; the pipeline's memory
    // is the scratch entry, the other metrics have none.
    {
        const v::MetricsMemoryUsage usage = metrics.GetMemoryUsage();
        v::Ssimulacra2Config single;
        single.size = mc.size;
        single.gpu_resident_images = 0;
        v::Ssimulacra2Pipeline standalone(single);
        Expect(usage.spatial && usage.scratch && !usage.vmaf_v0 && !usage.vmaf_v1 &&
                   usage.scratch->arena.allocation_bytes ==
                       standalone.GetMemoryUsage().arena.allocation_bytes,
               "metrics memory usage");
        const auto r = metrics.Compute(base, Gradient(1));
        Expect(r && r->ssimulacra2 && !r->butteraugli && !r->vmaf_v0 && !r->vmaf_v1 &&
                   *r->ssimulacra2 == standalone.Compute(base, Gradient(1)).Score(),
               "SSIMULACRA 2 alone through Metrics");
        Expect(!metrics.Flush(), "nothing left to flush");
        metrics.Reset();
    }
    for (int variant = 0; variant < 3; ++variant) {
        const auto r = metrics.Compute(base, Gradient(variant));
        Expect(r.has_value() && r->frame_index == static_cast<std::uint64_t>(variant),
               "frame index");
        std::printf("{\"path\": \"metrics\", \"variant\": %d, \"score\": %.17g}\n", variant,
                    *r->ssimulacra2);
    }
    ExpectThrow<std::logic_error>([&] { (void)metrics.ComputeImage(base, base); },
                                  "ComputeImage inside a sequence");
    const v::MetricsFinalResult fin = metrics.Finalize();
    Expect(fin.frames == 3 && !fin.last_frame, "Finalize frames");
    ExpectThrow<std::logic_error>([&] { (void)metrics.Compute(base, base); },
                                  "Compute after Finalize");
    metrics.Reset();
    const v::MetricsResult still = metrics.ComputeImage(base, Gradient(1));
    Expect(still.frame_index == 0, "still frame index");
    std::printf("{\"path\": \"metrics_image\", \"variant\": 1, \"score\": %.17g}\n",
                *still.ssimulacra2);
    v::Image grey = Gradient(0);
    grey.format.family = v::ColorFamily::Grey;
    grey.data.resize(32 * 32);
    ExpectThrow<std::invalid_argument>([&] { (void)metrics.Compute(grey, grey); },
                                       "format differs from configured");
    // metrics_test.cc:439-475, 555-574: a rejected input does not consume a
    // frame or fail the sequence; packed spans must have the exact size.
    metrics.Reset();
    v::Image wrong = Gradient(1);
    wrong.format.transfer = v::TransferCharacteristics::Bt709;
    ExpectThrow<std::invalid_argument>([&] { (void)metrics.Compute(base, wrong); },
                                       "transfer differs from configured");
    v::Image narrow = Gradient(1);
    narrow.size.width -= 1;
    ExpectThrow<std::invalid_argument>([&] { (void)metrics.Compute(base, narrow); },
                                       "size differs from configured");
    v::Image short_data = Gradient(1);
    short_data.data.pop_back();
    ExpectThrow<std::invalid_argument>([&] { (void)metrics.Compute(base, short_data); },
                                       "short image data");
    const auto frame0 = metrics.Compute(base, Gradient(1));
    Expect(frame0 && frame0->frame_index == 0, "rejected inputs consume no frame");
    metrics.Reset();
    const v::Image d1 = Gradient(1);
    const auto ob = std::as_bytes(std::span(base.data));
    const auto db = std::as_bytes(std::span(d1.data));
    ExpectThrow<std::invalid_argument>(
        [&] { (void)metrics.Compute(ob.first(ob.size() - 1), db); }, "short packed original");
    ExpectThrow<std::invalid_argument>(
        [&] { (void)metrics.Compute(ob, db.first(db.size() - 1)); }, "short packed distorted");
    const auto packed = metrics.ComputeImage(ob, db);
    const auto image = metrics.ComputeImage(base, d1);
    Expect(packed.frame_index == 0 && image.frame_index == 0 &&
               *packed.ssimulacra2 == *image.ssimulacra2,
           "packed spans and images agree");
}

void Gpu() {
    // vqm_device.h: the devices, and the default device by UUID.
    const auto devices = v::ListDevices();
    Expect(!devices.empty() && !devices[0].name.empty(), "ListDevices");
    if (!devices.empty()) v::SetDefaultDevice(devices[0].uuid);
    v::DeviceUuid unknown{};
    unknown.fill(0xEE);
    ExpectThrow<std::invalid_argument>([&] { v::SetDefaultDevice(unknown); }, "an unknown UUID");
    v::Ssimulacra2Config config;
    config.size = {32, 32};
    v::Ssimulacra2Pipeline pipeline(config);
    const v::Image base = Gradient(0);
    for (int variant = 0; variant < 3; ++variant) {
        const v::Image dist = Gradient(variant);
        Print("pipeline", variant, pipeline.Compute(base, dist));
    }
    const v::UploadedImage up = pipeline.Upload(base);
    Print("uploaded", 1, pipeline.Compute(up, Gradient(1)));
    pipeline.Release(up);
    v::Image small = Gradient(0);
    small.size = {16, 16};
    small.data.resize(3 * 16 * 16);
    ExpectThrow<std::invalid_argument>([&] { (void)pipeline.Compute(base, small); },
                                       "size mismatch");
    ExpectThrow<std::invalid_argument>([&] { (void)pipeline.Finish(12345); }, "unknown token");
    // While a submission is in flight that is reported before a bad image
    // (pipeline_test.cc:385-395).
    const std::uint64_t token = pipeline.Submit(base, Gradient(1));
    ExpectThrow<std::logic_error>([&] { (void)pipeline.Submit(base, small); },
                                  "in flight before a bad image");
    ExpectThrow<std::logic_error>([&] { (void)pipeline.Upload(small); },
                                  "in flight before a bad upload");
    (void)pipeline.Finish(token);
    ExpectThrow<std::invalid_argument>([&] { (void)pipeline.Submit(base, small); },
                                       "bad image once idle");
    // vqm_alpha.h: an opaque pair once at the default background; with alpha
    // on either side, the lower of the dark and bright scores.
    const v::Image check = Gradient(1);
    Expect(v::ComputeWorstBackground(pipeline, base, check).Score() ==
               pipeline.Compute(base, check).Score(),
           "worst background of an opaque pair");
    v::Image translucent = Gradient(1);
    translucent.format.alpha = v::AlphaType::Straight;
    translucent.data.resize(4 * 32 * 32, 96);
    const double dark = pipeline.Compute(base, translucent, 0.1f).Score();
    const double bright = pipeline.Compute(base, translucent, 0.9f).Score();
    Expect(dark != bright, "the background matters with alpha");
    Expect(v::ComputeWorstBackground(pipeline, base, translucent).Score() == std::min(dark, bright),
           "worst background with alpha on one side");

    {
        // pipeline_test.cc:179-216: caller-owned buffers written through
        // the mapping score like the packed images; while a submission is
        // in flight the pool cannot change; two buffers fill this pool.
        v::Ssimulacra2Config owned = config;
        const std::size_t per_image = v::RequiredBytes(base.format, base.size);
        owned.input_bytes = 2 * per_image;
        owned.memory_policy = v::MemoryPolicy::Staged;
        v::Ssimulacra2Pipeline p(owned);
        const v::Image dist = Gradient(2);
        const double expected = p.Compute(base, dist).Score();
        const v::ImageBuffer a = p.AllocateImage(base.format);
        const v::ImageBuffer b = p.AllocateImage(dist.format);
        Expect(a.bytes == per_image && b.bytes == per_image, "buffer sizes");
        const v::PipelineMemoryUsage usage = p.GetMemoryUsage();
        Expect(usage.uses_staging && usage.staging.allocation_bytes >= 2 * per_image &&
                   usage.input_bytes >= 4 * per_image &&
                   usage.arena.allocation_bytes >= usage.pyramid_bytes &&
                   usage.arena.allocation_bytes + usage.staging.allocation_bytes ==
                       usage.total_bytes,
               "memory usage: device arena and pinned pool");
        std::memcpy(p.MapImage(a), base.data.data(), base.data.size());
        std::memcpy(p.MapImage(b), dist.data.data(), dist.data.size());
        Expect(p.Compute(a, b).Score() == expected, "caller-owned buffers");
        const std::uint64_t pending = p.Submit(a, b);
        ExpectThrow<std::logic_error>([&] { p.Release(a); }, "Release in flight");
        ExpectThrow<std::logic_error>([&] { (void)p.MapImage(a); }, "MapImage in flight");
        ExpectThrow<std::logic_error>([&] { (void)p.AllocateImage(base.format); },
                                      "AllocateImage in flight");
        Expect(p.Finish(pending).Score() == expected, "submitted buffers");
        p.Release(a);
        ExpectThrow<std::invalid_argument>([&] { (void)p.Compute(a, b); }, "released buffer");
        p.Release(b);
        const v::ImageBuffer c = p.AllocateImage(base.format);
        const v::ImageBuffer d = p.AllocateImage(base.format);
        ExpectThrow<std::invalid_argument>([&] { (void)p.AllocateImage(base.format); },
                                           "a third buffer");
        p.Release(c);
        p.Release(d);
    }

    {
        // vqm_views.h Score, and padded views through the pool with one
        // invalid view in the list (pool_test.cc:112-182).
        const v::Image dist = Gradient(2);
        std::array<std::vector<std::byte>, 3> ob, db;
        const auto padded = [](const v::Image& img, std::array<std::vector<std::byte>, 3>& st) {
            v::ImageView view;
            view.size = img.size;
            view.format = img.format;
            for (std::size_t p = 0; p < 3; ++p) {
                st[p].assign(39 * 32, std::byte{0});
                for (std::size_t r = 0; r < 32; ++r)
                    std::memcpy(st[p].data() + r * 39, img.data.data() + p * 1024 + r * 32, 32);
                view.planes[p] = {st[p].data(), 39};
            }
            return view;
        };
        const v::ImageView vo = padded(base, ob), vd = padded(dist, db);
        const double expected = pipeline.Compute(base, dist).Score();
        Expect(v::Score(pipeline, vo, vd) == expected, "Score of padded views");
        v::ImageView other = vd;
        other.size = {16, 16};
        ExpectThrow<std::invalid_argument>([&] { (void)v::Score(pipeline, vo, other); },
                                           "views of different sizes");
        v::Ssimulacra2Pool views(config, 2, 1);
        const std::vector<v::ImageViewPair> vp{{vo, vd}, {vd, vo}};
        const auto scores = views.ScoreMany(std::span<const v::ImageViewPair>(vp));
        Expect(scores[0] == expected && scores[1] == pipeline.Compute(dist, base).Score(),
               "pool of padded views");
        v::ImageView invalid = vd;
        invalid.planes[0].stride_bytes = 1;
        const std::vector<v::ImageViewPair> bad{{vo, vd}, {vd, vo}, {vo, invalid}};
        ExpectThrow<std::invalid_argument>(
            [&] { (void)views.ComputeMany(std::span<const v::ImageViewPair>(bad)); },
            "an invalid view in a pool list");
        Expect(views.ScoreMany(std::span<const v::ImageViewPair>(vp).first(1))[0] == expected,
               "the pool after an invalid view");
    }

    v::Ssimulacra2Pool pool(config, 2, 2);
    const v::Image d1 = Gradient(1), d2 = Gradient(2);
    const std::vector<v::ImagePair> pairs{{base, base}, {base, d1}, {base, d2}};
    const auto results = pool.ComputeMany(std::span<const v::ImagePair>(pairs));
    for (std::size_t i = 0; i < results.size(); ++i) Print("pool", static_cast<int>(i), results[i]);
    // pool_test.cc:17-61: no workers is an error; an empty list gives no
    // results; ScoreMany matches ComputeMany; a moved-from pool has no
    // workers and refuses work, the pool it moved into keeps scoring.
    ExpectThrow<std::invalid_argument>([&] { v::Ssimulacra2Pool none(config, 0); },
                                       "pool of zero workers");
    Expect(pool.ComputeMany(std::span<const v::ImagePair>{}).empty(), "empty list");
    const auto scores = pool.ScoreMany(std::span<const v::ImagePair>(pairs));
    for (std::size_t i = 0; i < pairs.size(); ++i)
        Expect(scores[i] == results[i].Score(), "ScoreMany equals ComputeMany");
    const std::span<const v::ImagePair> first_pair(pairs.data(), 1);
    v::Ssimulacra2Pool moved(std::move(pool));
    Expect(pool.Workers() == 0 && moved.Workers() == 2, "workers after a move");
    ExpectThrow<std::logic_error>([&] { (void)pool.ScoreMany(first_pair); }, "moved-from pool");
    Expect(moved.ScoreMany(first_pair)[0] == results[0].Score(), "moved pool scores");
    v::Ssimulacra2Pool assigned(config, 1, 2);
    assigned = std::move(moved);
    Expect(assigned.Workers() == 2 && moved.Workers() == 0, "workers after assignment");
    Expect(assigned.ScoreMany(first_pair)[0] == results[0].Score(), "assigned pool scores");
    ExpectThrow<std::logic_error>([&] { (void)moved.ComputeMany(first_pair); },
                                  "moved-from pool after assignment");

    // The opt-in recursive blur, through the pipeline and the pool.
    v::Ssimulacra2Config rec = config;
    rec.blur = v::Ssimulacra2Blur::Recursive;
    v::Ssimulacra2Pipeline rpipe(rec);
    for (int variant = 1; variant < 3; ++variant)
        Print("recursive", variant, rpipe.Compute(base, Gradient(variant)));
    v::Ssimulacra2Pool rpool(rec, 1, 2);
    const std::vector<v::ImagePair> rpairs{{base, d1}, {base, d2}};
    const auto rres = rpool.ComputeMany(std::span<const v::ImagePair>(rpairs));
    for (std::size_t i = 0; i < rres.size(); ++i)
        Print("recursive_pool", static_cast<int>(i) + 1, rres[i]);
}

}  // namespace

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "host";
    try {
        if (mode == "host") Host();
        else if (mode == "gpu") {
            Gpu();
            GpuMetrics();
        }
        else {
            std::fprintf(stderr, "usage: facade_check host|gpu\n");
            return 2;
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "FAIL: unexpected exception: %s\n", e.what());
        return 1;
    }
    return failures ? 1 : 0;
}
