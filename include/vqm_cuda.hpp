// vqm_cuda.hpp -- VQM's SSIMULACRA 2 C++ API on the B200 scorer.
//
// Header-only C++ layer over the C ABI in vqm_cu_ss2.h: the classes, member
// functions, argument meanings and exception types of the reference's
// include/ssimulacra2.h, include/vqm_image.h, include/vqm_views.h,
// include/vqm_pool.h and, for SSIMULACRA 2, include/vqm_metrics.h
// (GreatValueCreamSoda/vqm), with CUDA device buffers
// (CudaBufferView) in place of Vulkan buffers. A VQM caller switches by
// including this header and linking libvqm_ss2.so; every call crosses into
// CUDA through the C ABI only.
//
// Status codes map back to the reference's exceptions:
//   VQM_CU_INVALID_ARGUMENT -> std::invalid_argument
//   VQM_CU_LOGIC_ERROR      -> std::logic_error
//   VQM_CU_OVERFLOW_ERROR   -> std::overflow_error
//   VQM_CU_RUNTIME_ERROR    -> std::runtime_error
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "vqm_cu_ss2.h"

namespace vqm::cuda {

// ---- vqm_image.h ------------------------------------------------------------

struct Size {
    std::size_t width = 0;
    std::size_t height = 0;
    constexpr bool operator==(const Size&) const noexcept = default;
};

enum class PixelType : std::uint8_t { Byte = 0, Word = 1, Half = 2, Float = 3 };
enum class PixelRange : std::uint8_t { Limited = 0, Full = 1 };
enum class ColorFamily : std::uint8_t { Grey = 0, Rgb = 1, Yuv = 2 };
enum class AlphaType : std::uint8_t { None = 0, Straight = 1, Premultiplied = 2 };
enum class ChromaLocation : std::uint8_t {
    Left = 0, Center = 1, TopLeft = 2, Top = 3, BottomLeft = 4, Bottom = 5
};
enum class MatrixCoefficients : std::uint8_t {
    Rgb = 0, Bt709 = 1, Unspecified = 2, Fcc = 4, Bt470Bg = 5, St170M = 6, St240M = 7,
    YCgCo = 8, Bt2020Ncl = 9, Bt2020Cl = 10, St2085YDzDx = 11, ChromaticityDerivedNcl = 12,
    ChromaticityDerivedCl = 13, Bt2100ICtCp = 14, St2128IptC2 = 15, YCgCoRe = 16, YCgCoRo = 17
};
enum class TransferCharacteristics : std::uint8_t {
    Bt709 = 1, Unspecified = 2, Bt470M = 4, Bt470Bg = 5, Bt601 = 6, St240M = 7, Linear = 8,
    Log100 = 9, Log316 = 10, Iec61966_2_4 = 11, Bt1361 = 12, Srgb = 13, Bt2020_10 = 14,
    Bt2020_12 = 15, St2084 = 16, St428 = 17, AribB67 = 18
};
enum class ColorPrimaries : std::uint8_t {
    Bt709 = 1, Unspecified = 2, Bt470M = 4, Bt470Bg = 5, St170M = 6, St240M = 7, Film = 8,
    Bt2020 = 9, St428 = 10, St431_2 = 11, St432_1 = 12, Ebu3213E = 22
};
enum class ChromaFilter : std::uint8_t { Bilinear = 0, Bicubic = 1, Lanczos = 2 };
// The blur (no counterpart in VQM's config): Sampled is VQM's 13-tap
// Gaussian; Recursive, opt-in, is the recursive Gaussian of Cloudinary's
// ssimulacra2 (VQM_CU_SS2_BLUR_RECURSIVE), whose scores are not VQM's.
enum class Ssimulacra2Blur : std::uint32_t { Sampled = 0, Recursive = 1 };

struct ImageFormat {
    PixelType type = PixelType::Float;
    ColorFamily family = ColorFamily::Rgb;
    AlphaType alpha = AlphaType::None;
    PixelRange range = PixelRange::Full;
    MatrixCoefficients matrix = MatrixCoefficients::Rgb;
    TransferCharacteristics transfer = TransferCharacteristics::Srgb;
    ColorPrimaries primaries = ColorPrimaries::Bt709;
    ChromaLocation chroma_location = ChromaLocation::Left;
    std::uint8_t subsample_w = 0;
    std::uint8_t subsample_h = 0;
    std::uint8_t depth = 0;
};

// Packed planes (Y/R, U/G, V/B, alpha), each on a 4-byte boundary.
struct Image {
    Size size;
    ImageFormat format;
    std::vector<std::uint8_t> data;
    [[nodiscard]] bool HasAlpha() const noexcept { return format.alpha != AlphaType::None; }
};

struct UploadedImage {
    std::uint64_t slot = 0;  // 0 == invalid
    Size size;
};

struct ImageBuffer {
    std::uint64_t slot = 0;  // 0 == invalid
    Size size;
    std::size_t bytes = 0;
};

// ---- vqm_views.h --------------------------------------------------------------

struct PlaneView {
    const std::byte* data = nullptr;
    std::size_t stride_bytes = 0;
};

struct ImageView {
    Size size;
    ImageFormat format;
    std::array<PlaneView, 4> planes{};
};

// The CUDA counterpart of VulkanBufferView (include/vqm_vulkan.h): planes in
// caller-owned device memory, read in place; 0 strides mean packed rows.
struct CudaBufferView {
    Size size;
    ImageFormat format;
    std::array<const void*, 4> planes{};
    std::array<std::size_t, 4> strides{};
};

// The counterpart of VulkanSubmitSync: events the pair's work waits for
// before it starts and records when it is done (cudaEvent_t as void*).
struct CudaSubmitSync {
    std::vector<void*> wait_events;
    std::vector<void*> signal_events;
};

namespace detail {

inline void Check(int status) {
    if (status == VQM_CU_OK) return;
    const std::string message = vqm_cu_last_error();
    switch (status) {
        case VQM_CU_INVALID_ARGUMENT: throw std::invalid_argument(message);
        case VQM_CU_LOGIC_ERROR: throw std::logic_error(message);
        case VQM_CU_OVERFLOW_ERROR: throw std::overflow_error(message);
        default: throw std::runtime_error(message);
    }
}

inline vqm_cu_format ToC(const ImageFormat& f) {
    vqm_cu_format c{};
    c.type = static_cast<std::uint8_t>(f.type);
    c.family = static_cast<std::uint8_t>(f.family);
    c.alpha = static_cast<std::uint8_t>(f.alpha);
    c.range = static_cast<std::uint8_t>(f.range);
    c.matrix = static_cast<std::uint8_t>(f.matrix);
    c.transfer = static_cast<std::uint8_t>(f.transfer);
    c.primaries = static_cast<std::uint8_t>(f.primaries);
    c.chroma_location = static_cast<std::uint8_t>(f.chroma_location);
    c.subsample_w = f.subsample_w;
    c.subsample_h = f.subsample_h;
    c.depth = f.depth;
    return c;
}

inline std::uint32_t Dim(std::size_t v) {
    if (v > 0xffffffffull) throw std::overflow_error("image dimension exceeds 32 bits");
    return static_cast<std::uint32_t>(v);
}

}  // namespace detail

// RequiredBytes (include/vqm_image.h:360-363).
[[nodiscard]] inline std::size_t RequiredBytes(const ImageFormat& format, Size size) {
    std::size_t bytes = 0;
    const vqm_cu_format f = detail::ToC(format);
    detail::Check(vqm_cu_required_bytes(&f, detail::Dim(size.width), detail::Dim(size.height),
                                        &bytes));
    return bytes;
}

// ValidateFormat (src/input.cc): throws std::invalid_argument with the
// reference's message, prefixed by `name`.
inline void ValidateFormat(const ImageFormat& format, Size size, const char* name) {
    const vqm_cu_format f = detail::ToC(format);
    detail::Check(vqm_cu_validate_format(&f, detail::Dim(size.width), detail::Dim(size.height),
                                         name));
}

namespace detail {

// Plane p of vqm::Image's packed layout (input.cc:114-145): whether it is
// present, its offset, samples per row and rows, and bytes per sample.
struct PlaneGeometry {
    bool present = false;
    std::size_t offset = 0, width = 0, height = 0, sample_bytes = 0;
};
inline std::array<PlaneGeometry, 4> Layout(const ImageFormat& f, Size size) {
    std::array<PlaneGeometry, 4> out{};
    const std::size_t sb = f.type == PixelType::Byte ? 1 : f.type == PixelType::Float ? 4 : 2;
    std::size_t cursor = 0;
    for (int p = 0; p < 4; ++p) {
        const bool chroma = p == 1 || p == 2;
        PlaneGeometry& g = out[p];
        g.present = p == 0 || (chroma && f.family != ColorFamily::Grey) ||
                    (p == 3 && f.alpha != AlphaType::None);
        if (!g.present) continue;
        g.width = chroma ? size.width >> f.subsample_w : size.width;
        g.height = chroma ? size.height >> f.subsample_h : size.height;
        g.sample_bytes = sb;
        g.offset = cursor;
        cursor = (cursor + g.width * g.height * sb + 3) / 4 * 4;
    }
    return out;
}

// Plane addresses of a packed Image.
inline vqm_cu_image ToC(const Image& img, const char* name) {
    const std::size_t expected = RequiredBytes(img.format, img.size);
    if (img.data.size() != expected)
        throw std::invalid_argument(std::string(name) +
                                    ": data size does not match the image format (expected " +
                                    std::to_string(expected) + " bytes)");
    vqm_cu_image c{};
    c.width = Dim(img.size.width);
    c.height = Dim(img.size.height);
    c.format = ToC(img.format);
    c.memory = VQM_CU_MEMORY_HOST;
    const auto layout = Layout(img.format, img.size);
    for (int p = 0; p < 4; ++p)
        if (layout[p].present) c.planes[p] = img.data.data() + layout[p].offset;
    return c;
}

// DescribeImageView (src/image_view.cc:16-45): a non-empty size, a valid
// format, and every present plane with data and a stride of at least a row.
inline std::array<PlaneGeometry, 4> CheckView(const ImageView& v) {
    if (v.size.width == 0 || v.size.height == 0)
        throw std::invalid_argument("image view: size must be non-zero");
    const vqm_cu_format f = ToC(v.format);
    Check(vqm_cu_validate_format(&f, Dim(v.size.width), Dim(v.size.height), "image view"));
    const auto layout = Layout(v.format, v.size);
    for (int p = 0; p < 4; ++p) {
        const PlaneGeometry& g = layout[p];
        if (!g.present) continue;
        const std::size_t row = g.width * g.sample_bytes;
        if (v.planes[p].data == nullptr || v.planes[p].stride_bytes < row)
            throw std::invalid_argument("image view: missing plane or short stride");
        const auto max_offset = static_cast<std::size_t>(PTRDIFF_MAX);
        if (row > max_offset ||
            (g.height > 1 && v.planes[p].stride_bytes > (max_offset - row) / (g.height - 1)))
            throw std::overflow_error("image view: plane stride is too large");
    }
    return layout;
}

inline vqm_cu_image ToC(const ImageView& v) {
    (void)CheckView(v);
    vqm_cu_image c{};
    c.width = Dim(v.size.width);
    c.height = Dim(v.size.height);
    c.format = ToC(v.format);
    c.memory = VQM_CU_MEMORY_HOST;
    for (int p = 0; p < 4; ++p) {
        c.planes[p] = v.planes[p].data;
        c.strides[p] = v.planes[p].stride_bytes;
    }
    return c;
}

inline vqm_cu_image ToC(const CudaBufferView& v) {
    vqm_cu_image c{};
    c.width = Dim(v.size.width);
    c.height = Dim(v.size.height);
    c.format = ToC(v.format);
    c.memory = VQM_CU_MEMORY_DEVICE;
    for (int p = 0; p < 4; ++p) {
        c.planes[p] = v.planes[p];
        c.strides[p] = v.strides[p];
    }
    return c;
}

}  // namespace detail

// ---- ssimulacra2.h ----------------------------------------------------------

struct Ssimulacra2Scale {
    static constexpr std::size_t kSsimNormCount = 6;
    static constexpr std::size_t kEdgeNormCount = 12;
    std::array<double, kSsimNormCount> avg_ssim{};     // [channel * 2 + norm]
    std::array<double, kEdgeNormCount> avg_edgediff{}; // [channel * 4 + n]
};

struct Ssimulacra2Result {
    std::vector<Ssimulacra2Scale> scales;
    // Ssimulacra2Result::Score (score.cc:118-163): throws
    // std::invalid_argument for more than six scales, nonfinite norms or an
    // overflowing mapping.
    [[nodiscard]] double Score() const {
        std::vector<double> flat(std::max<std::size_t>(scales.size(), 1) * 18, 0.0);
        for (std::size_t s = 0; s < scales.size(); ++s) {
            for (int k = 0; k < 6; ++k) flat[s * 18 + k] = scales[s].avg_ssim[k];
            for (int k = 0; k < 12; ++k) flat[s * 18 + 6 + k] = scales[s].avg_edgediff[k];
        }
        double score = 0.0;
        detail::Check(vqm_cu_ss2_score(flat.data(), static_cast<std::uint32_t>(scales.size()),
                                       &score));
        return score;
    }

    static Ssimulacra2Result FromNorms(const double* norms, std::uint32_t count) {
        Ssimulacra2Result r;
        r.scales.resize(count);
        for (std::uint32_t s = 0; s < count; ++s) {
            for (int k = 0; k < 6; ++k) r.scales[s].avg_ssim[k] = norms[s * 18 + k];
            for (int k = 0; k < 12; ++k) r.scales[s].avg_edgediff[k] = norms[s * 18 + 6 + k];
        }
        return r;
    }
};

// vqm_memory_types.h:12-14: Automatic and Direct read the AllocateImage pool
// in place from pinned host memory; Staged copies its spans to a device
// mirror at submit.
enum class MemoryPolicy : std::uint8_t { Automatic, Direct, Staged };

struct Ssimulacra2Config {
    Size size;
    std::size_t gpu_resident_images = 2;
    bool half_planes = false;
    ChromaFilter chroma_filter = ChromaFilter::Bilinear;
    std::size_t input_bytes = 0;
    bool streaming_inputs = true;
    MemoryPolicy memory_policy = MemoryPolicy::Automatic;
    int device = -1;  // CUDA ordinal; -1 = the current device
    Ssimulacra2Blur blur = Ssimulacra2Blur::Sampled;
};

// vqm_memory_types.h:17-33. The arena is the device memory a pipeline
// holds; staging is the pinned host memory of its AllocateImage pool, which
// the kernels read in place. Memory types and heaps are 0 (device) and 1
// (host). The five byte counts break the same memory down by use.
struct MemoryAllocation {
    std::uint64_t buffer_bytes = 0;
    std::uint64_t allocation_bytes = 0;
    std::uint32_t memory_type = 0;
    std::uint32_t heap = 0;
};
struct PipelineMemoryUsage {
    bool uses_staging = false;
    MemoryAllocation arena;
    MemoryAllocation staging;
    std::vector<MemoryAllocation> auxiliary = {};
    std::uint64_t pyramid_bytes = 0, resident_bytes = 0, input_bytes = 0, scratch_bytes = 0,
                  total_bytes = 0;
};

class Ssimulacra2Pipeline {
public:
    explicit Ssimulacra2Pipeline(Ssimulacra2Config config) : config_(config) {
        vqm_cu_ss2_config c{};
        c.width = detail::Dim(config.size.width);
        c.height = detail::Dim(config.size.height);
        if (config.gpu_resident_images > 0xffffffffull)
            throw std::invalid_argument("gpu_resident_images is limited to 4095 slots");
        c.gpu_resident_images = static_cast<std::uint32_t>(config.gpu_resident_images);
        c.half_planes = config.half_planes ? 1 : 0;
        c.chroma_filter = static_cast<std::uint32_t>(config.chroma_filter);
        c.streaming_inputs = config.streaming_inputs ? 1 : 0;
        c.input_bytes = config.input_bytes;
        c.device = config.device;
        c.blur = static_cast<std::uint32_t>(config.blur);
        c.memory_policy = static_cast<std::uint32_t>(config.memory_policy);
        vqm_cu_ss2_pipeline* p = nullptr;
        detail::Check(vqm_cu_ss2_create(&c, &p));
        p_.reset(p);
    }
    Ssimulacra2Pipeline(Ssimulacra2Pipeline&&) noexcept = default;
    Ssimulacra2Pipeline& operator=(Ssimulacra2Pipeline&&) noexcept = default;

    [[nodiscard]] Ssimulacra2Result Compute(const Image& o, const Image& d, float background = 0.5f) {
        return Finish(Submit(o, d, background));
    }
    [[nodiscard]] Ssimulacra2Result Compute(const ImageView& o, const ImageView& d,
                                            float background = 0.5f) {
        return Finish(Submit(o, d, background));
    }
    [[nodiscard]] Ssimulacra2Result Compute(const UploadedImage& o, const UploadedImage& d,
                                            float background = 0.5f) {
        return Finish(Submit(o, d, background));
    }
    [[nodiscard]] Ssimulacra2Result Compute(const UploadedImage& o, const Image& d,
                                            float background = 0.5f) {
        return Finish(Submit(o, d, background));
    }
    [[nodiscard]] Ssimulacra2Result Compute(const ImageBuffer& o, const ImageBuffer& d,
                                            float background = 0.5f) {
        return Finish(Submit(o, d, background));
    }
    [[nodiscard]] Ssimulacra2Result Compute(const CudaBufferView& o, const CudaBufferView& d,
                                            float background = 0.5f) {
        return Finish(Submit(o, d, background));
    }

    [[nodiscard]] std::uint64_t Submit(const Image& o, const Image& d, float background = 0.5f) {
        vqm_cu_image a{}, b{};
        IdleFirst([&] {
            Geometry(o.size, "original");
            Geometry(d.size, "distorted");
            a = detail::ToC(o, "original");
            b = detail::ToC(d, "distorted");
        });
        return SubmitC(a, b, background);
    }
    [[nodiscard]] std::uint64_t Submit(const ImageView& o, const ImageView& d,
                                       float background = 0.5f) {
        vqm_cu_image a{}, b{};
        IdleFirst([&] {
            a = detail::ToC(o);
            b = detail::ToC(d);
        });
        return SubmitC(a, b, background);
    }
    [[nodiscard]] std::uint64_t Submit(const UploadedImage& o, const UploadedImage& d,
                                       float background = 0.5f) {
        std::uint64_t token = 0;
        detail::Check(vqm_cu_ss2_submit_resident(p_.get(), o.slot, d.slot, background, &token));
        return token;
    }
    [[nodiscard]] std::uint64_t Submit(const UploadedImage& o, const Image& d,
                                       float background = 0.5f) {
        vqm_cu_image b{};
        IdleFirst([&] {
            Geometry(d.size, "distorted");
            b = detail::ToC(d, "distorted");
        });
        std::uint64_t token = 0;
        detail::Check(vqm_cu_ss2_submit_resident_image(p_.get(), o.slot, &b, background, &token));
        return token;
    }
    [[nodiscard]] std::uint64_t Submit(const ImageBuffer& o, const ImageBuffer& d,
                                       float background = 0.5f) {
        std::uint64_t token = 0;
        detail::Check(vqm_cu_ss2_submit_buffers(p_.get(), o.slot, d.slot, background, &token));
        return token;
    }
    [[nodiscard]] std::uint64_t Submit(const CudaBufferView& o, const CudaBufferView& d,
                                       float background = 0.5f) {
        return SubmitC(detail::ToC(o), detail::ToC(d), background);
    }
    [[nodiscard]] std::uint64_t Submit(const CudaBufferView& o, const CudaBufferView& d,
                                       const CudaSubmitSync& sync, float background = 0.5f) {
        const vqm_cu_image a = detail::ToC(o), b = detail::ToC(d);
        std::uint64_t token = 0;
        detail::Check(vqm_cu_ss2_submit_sync(
            p_.get(), &a, &b, sync.wait_events.data(),
            static_cast<std::uint32_t>(sync.wait_events.size()), sync.signal_events.data(),
            static_cast<std::uint32_t>(sync.signal_events.size()), background, &token));
        return token;
    }

    [[nodiscard]] Ssimulacra2Result Finish(std::uint64_t token) {
        double norms[VQM_CU_SS2_MAX_NORMS];
        std::uint32_t scales = 0;
        detail::Check(vqm_cu_ss2_finish(p_.get(), token, norms, &scales));
        return Ssimulacra2Result::FromNorms(norms, scales);
    }

    [[nodiscard]] UploadedImage Upload(const Image& image) {
        vqm_cu_image c{};
        IdleFirst([&] {
            Geometry(image.size, "image");
            c = detail::ToC(image, "image");
        });
        std::uint64_t handle = 0;
        detail::Check(vqm_cu_ss2_upload(p_.get(), &c, &handle));
        return UploadedImage{handle, image.size};
    }
    void Release(UploadedImage image) { detail::Check(vqm_cu_ss2_release(p_.get(), image.slot)); }

    [[nodiscard]] ImageBuffer AllocateImage(const ImageFormat& format) {
        const vqm_cu_format f = detail::ToC(format);
        std::uint64_t handle = 0;
        std::size_t bytes = 0;
        detail::Check(vqm_cu_ss2_allocate_image(p_.get(), &f, &handle, &bytes));
        return ImageBuffer{handle, config_.size, bytes};
    }
    // The buffer's bytes in pinned host memory, written with memcpy as in
    // VQM (ssimulacra2.h:174-176) and read by the kernels in place.
    [[nodiscard]] std::byte* MapImage(ImageBuffer buffer) {
        void* ptr = nullptr;
        detail::Check(vqm_cu_ss2_map_image(p_.get(), buffer.slot, &ptr));
        return static_cast<std::byte*>(ptr);
    }
    void Release(ImageBuffer buffer) {
        detail::Check(vqm_cu_ss2_release_image(p_.get(), buffer.slot));
    }

    [[nodiscard]] PipelineMemoryUsage GetMemoryUsage() const {
        vqm_cu_memory_usage c{};
        detail::Check(vqm_cu_ss2_memory_usage(p_.get(), &c));
        PipelineMemoryUsage u;
        const std::uint64_t device = c.total_bytes - c.host_bytes;
        u.arena = {device, device, 0, 0};
        u.staging = {c.host_bytes, c.host_bytes, 1, 1};
        u.uses_staging = c.uses_staging != 0;
        u.pyramid_bytes = c.pyramid_bytes;
        u.resident_bytes = c.resident_bytes;
        u.input_bytes = c.input_bytes;
        u.scratch_bytes = c.scratch_bytes;
        u.total_bytes = c.total_bytes;
        return u;
    }
    void SetStream(void* stream) { detail::Check(vqm_cu_ss2_set_stream(p_.get(), stream)); }

private:
    struct Deleter {
        void operator()(vqm_cu_ss2_pipeline* p) const noexcept { vqm_cu_ss2_destroy(p); }
    };
    void Geometry(Size s, const char* name) const {
        if (!(s == config_.size))
            throw std::invalid_argument(std::string(name) +
                                        ": image size does not match the pipeline geometry");
    }
    // The host-side image checks (geometry, data size) run before the
    // library sees the call; VQM reports a call made while a submission is
    // in flight first (vulkan_runtime.h:275-285), so a failed check defers
    // to that.
    template <class F>
    void IdleFirst(F&& checks) const {
        try {
            checks();
        } catch (const std::invalid_argument&) {
            std::uint32_t busy = 0;
            if (vqm_cu_ss2_in_flight(p_.get(), &busy) == VQM_CU_OK && busy)
                throw std::logic_error(
                    "cuda: a submission is already in flight; Finish it first");
            throw;
        }
    }
    std::uint64_t SubmitC(const vqm_cu_image& a, const vqm_cu_image& b, float background) {
        std::uint64_t token = 0;
        detail::Check(vqm_cu_ss2_submit(p_.get(), &a, &b, background, &token));
        return token;
    }
    Ssimulacra2Config config_;
    std::unique_ptr<vqm_cu_ss2_pipeline, Deleter> p_;
};

// ---- vqm_device.h -------------------------------------------------------------

using DeviceUuid = std::array<std::uint8_t, 16>;
enum class DeviceType { Other, IntegratedGpu, DiscreteGpu, VirtualGpu, Cpu };
struct DeviceInfo {
    DeviceUuid uuid;
    std::string name;
    DeviceType type;
};

// ListDevices / SetDefaultDevice (include/vqm_device.h): CUDA devices in
// ordinal order; the default device is the one a config's device = -1 uses.
[[nodiscard]] inline std::vector<DeviceInfo> ListDevices() {
    std::uint32_t n = 0;
    detail::Check(vqm_cu_device_count(&n));
    std::vector<DeviceInfo> out;
    for (std::uint32_t i = 0; i < n; ++i) {
        char name[256];
        DeviceInfo d{};
        std::uint32_t type = 0;
        detail::Check(vqm_cu_device_info(i, name, sizeof(name), d.uuid.data(), &type));
        d.name = name;
        d.type = static_cast<DeviceType>(type);
        out.push_back(std::move(d));
    }
    return out;
}
inline void SetDefaultDevice(const DeviceUuid& uuid) {
    detail::Check(vqm_cu_set_default_device(uuid.data()));
}

// ---- vqm_views.h helpers --------------------------------------------------------

// CopyImage (include/vqm_views.h:36, src/image_view.cc:82-90): the view's
// planes packed into a vqm::Image, each plane's trailing bytes up to a 4-byte
// boundary zero.
[[nodiscard]] inline Image CopyImage(const ImageView& view) {
    const auto layout = detail::CheckView(view);
    Image image;
    image.size = view.size;
    image.format = view.format;
    image.data.assign(RequiredBytes(view.format, view.size), 0);
    for (int p = 0; p < 4; ++p) {
        const auto& g = layout[p];
        if (!g.present) continue;
        const std::size_t row = g.width * g.sample_bytes;
        for (std::size_t y = 0; y < g.height; ++y)
            std::memcpy(image.data.data() + g.offset + y * row,
                        view.planes[p].data + y * view.planes[p].stride_bytes, row);
    }
    return image;
}

// Score (include/vqm_views.h:37-41, src/image_view.cc:92-100).
[[nodiscard]] inline double Score(Ssimulacra2Pipeline& pipeline, const ImageView& original,
                                  const ImageView& distorted, float background = 0.5f) {
    if (!(original.size == distorted.size))
        throw std::invalid_argument("image views must have the same size");
    return pipeline.Compute(original, distorted, background).Score();
}

// ---- vqm_alpha.h --------------------------------------------------------------

// ComputeWorstBackground (include/vqm_alpha.h:12-28), the CLI's alpha policy
// for callers: a pair with no alpha on either side is scored once at the
// default background; otherwise it is scored over a dark (0.1) and a bright
// (0.9) background and the lower score's result is returned. Frame is any
// image kind the pipeline's Compute takes (Image, ImageView, CudaBufferView).
template <typename Frame>
[[nodiscard]] Ssimulacra2Result ComputeWorstBackground(Ssimulacra2Pipeline& pipeline,
                                                       const Frame& original,
                                                       const Frame& distorted) {
    if (original.format.alpha == AlphaType::None && distorted.format.alpha == AlphaType::None)
        return pipeline.Compute(original, distorted);
    Ssimulacra2Result dark = pipeline.Compute(original, distorted, 0.1f);
    Ssimulacra2Result bright = pipeline.Compute(original, distorted, 0.9f);
    return bright.Score() < dark.Score() ? bright : dark;
}

// ---- vqm_pool.h ---------------------------------------------------------------

struct ImagePair {
    const Image& original;
    const Image& distorted;
};
struct ImageViewPair {
    const ImageView& original;
    const ImageView& distorted;
};
struct CudaBufferPair {
    const CudaBufferView& original;
    const CudaBufferView& distorted;
};

// Ssimulacra2Pool (include/vqm_pool.h:51-87): results in input order. The
// reference round-robins pairs over `workers` one-in-flight pipelines of one
// geometry; here every `chunk` pairs (any sizes) are one batched submission,
// one launch per stage over all of them, with `workers` batch scorers in
// flight at once.
class Ssimulacra2Pool {
public:
    Ssimulacra2Pool(Ssimulacra2Config config, std::size_t workers, std::size_t chunk = 64)
        : chroma_filter_(config.chroma_filter), chunk_(chunk ? chunk : 1) {
        if (workers == 0) throw std::invalid_argument("pool needs at least one worker");
        for (std::size_t i = 0; i < workers; ++i) {
            vqm_cu_ss2_batch_config c{};
            c.chroma_filter = static_cast<std::uint32_t>(config.chroma_filter);
            c.device = config.device;
            c.max_pairs = static_cast<std::uint32_t>(chunk_);
            c.half_planes = config.half_planes ? 1 : 0;
            c.blur = static_cast<std::uint32_t>(config.blur);
            vqm_cu_ss2_batch* b = nullptr;
            detail::Check(vqm_cu_ss2_batch_create(&c, &b));
            batches_.emplace_back(b);
        }
    }
    // A moved-from pool has no workers and refuses work (pool.cc:118-122).
    Ssimulacra2Pool(Ssimulacra2Pool&& other) noexcept
        : chroma_filter_(other.chroma_filter_),
          chunk_(other.chunk_),
          batches_(std::move(other.batches_)),
          poisoned_(other.poisoned_) {
        other.batches_.clear();
        other.moved_from_ = true;
    }
    Ssimulacra2Pool& operator=(Ssimulacra2Pool&& other) noexcept {
        if (this != &other) {
            chroma_filter_ = other.chroma_filter_;
            chunk_ = other.chunk_;
            batches_ = std::move(other.batches_);
            poisoned_ = other.poisoned_;
            moved_from_ = other.moved_from_;
            other.batches_.clear();
            other.moved_from_ = true;
        }
        return *this;
    }
    [[nodiscard]] std::size_t Workers() const noexcept { return batches_.size(); }

    [[nodiscard]] std::vector<Ssimulacra2Result> ComputeMany(std::span<const ImagePair> pairs,
                                                             float background = 0.5f) {
        Ready();
        std::vector<vqm_cu_image> o, d;
        for (const auto& p : pairs) {
            o.push_back(detail::ToC(p.original, "original"));
            d.push_back(detail::ToC(p.distorted, "distorted"));
        }
        return Run(o, d, background);
    }
    [[nodiscard]] std::vector<Ssimulacra2Result> ComputeMany(std::span<const ImageViewPair> pairs,
                                                             float background = 0.5f) {
        Ready();
        std::vector<vqm_cu_image> o, d;
        for (const auto& p : pairs) {
            o.push_back(detail::ToC(p.original));
            d.push_back(detail::ToC(p.distorted));
        }
        return Run(o, d, background);
    }
    [[nodiscard]] std::vector<Ssimulacra2Result> ComputeMany(std::span<const CudaBufferPair> pairs,
                                                             float background = 0.5f) {
        Ready();
        std::vector<vqm_cu_image> o, d;
        for (const auto& p : pairs) {
            o.push_back(detail::ToC(p.original));
            d.push_back(detail::ToC(p.distorted));
        }
        return Run(o, d, background);
    }
    template <class Pairs>
    [[nodiscard]] std::vector<double> ScoreMany(const Pairs& pairs, float background = 0.5f) {
        std::vector<double> scores;
        for (const auto& r : ComputeMany(pairs, background)) scores.push_back(r.Score());
        return scores;
    }

private:
    struct Deleter {
        void operator()(vqm_cu_ss2_batch* b) const noexcept { vqm_cu_ss2_batch_destroy(b); }
    };
    void Ready() const {
        if (moved_from_) throw std::logic_error("pool has been moved from");
        if (poisoned_) throw std::logic_error("pool cannot be reused after a failed drain");
    }
    std::vector<Ssimulacra2Result> Run(const std::vector<vqm_cu_image>& o,
                                       const std::vector<vqm_cu_image>& d, float background) {
        Ready();
        const std::size_t n = o.size();
        std::vector<Ssimulacra2Result> out(n);
        std::vector<std::pair<std::uint64_t, std::size_t>> pending(batches_.size(), {0, 0});
        std::vector<std::size_t> first(batches_.size(), 0);
        std::vector<double> norms(chunk_ * VQM_CU_SS2_MAX_NORMS);
        std::vector<std::uint32_t> scales(chunk_);
        auto drain = [&](std::size_t w) {
            const std::size_t count = pending[w].second;
            if (!count) return;
            pending[w].second = 0;  // a finish consumes the submission, failed or not
            detail::Check(vqm_cu_ss2_batch_finish(batches_[w].get(), pending[w].first,
                                                  norms.data(), scales.data(), nullptr));
            for (std::size_t i = 0; i < count; ++i)
                out[first[w] + i] = Ssimulacra2Result::FromNorms(
                    norms.data() + i * VQM_CU_SS2_MAX_NORMS, scales[i]);
        };
        std::size_t w = 0;
        try {
            for (std::size_t at = 0; at < n; at += chunk_, w = (w + 1) % batches_.size()) {
                drain(w);
                const std::size_t count = std::min(chunk_, n - at);
                std::uint64_t token = 0;
                // The images outlive the call, so their uploads may run
                // behind it and queue back to back across workers.
                detail::Check(vqm_cu_ss2_batch_submit_borrowed(batches_[w].get(),
                                                      static_cast<std::uint32_t>(count),
                                                      o.data() + at, d.data() + at, background,
                                                      &token));
                pending[w] = {token, count};
                first[w] = at;
            }
            for (std::size_t k = 0; k < batches_.size(); ++k) drain(k);
        } catch (...) {
            // Drain what was submitted before rethrowing the error that
            // interrupted the list (pool.cc:64-72). If a drain itself fails,
            // the workers are released and the pool refuses further use
            // (pool.cc:94-109): no submission of this list outlives the call.
            bool drain_failed = false;
            for (std::size_t k = 0; k < batches_.size(); ++k) {
                if (!pending[k].second) continue;
                if (vqm_cu_ss2_batch_finish(batches_[k].get(), pending[k].first, nullptr,
                                            nullptr, nullptr) != VQM_CU_OK)
                    drain_failed = true;
                pending[k].second = 0;
            }
            if (drain_failed) {
                batches_.clear();
                poisoned_ = true;
            }
            throw;
        }
        return out;
    }
    ChromaFilter chroma_filter_;
    std::size_t chunk_;
    std::vector<std::unique_ptr<vqm_cu_ss2_batch, Deleter>> batches_;
    bool poisoned_ = false;
    bool moved_from_ = false;
};

// ---- vqm_metrics.h (SSIMULACRA 2 only) ---------------------------------------

struct MetricsConfig {
    Size size;
    ImageFormat original_format{};
    ImageFormat distorted_format{};
    bool streaming_inputs = true;
    MemoryPolicy memory_policy = MemoryPolicy::Automatic;
    float background = 0.5f;
    // The one metric this library computes; leaving it empty is the
    // reference's "select at least one metric" error.
    std::optional<Ssimulacra2Config> ssimulacra2 = std::nullopt;
};

// vqm_metrics.h:50-61; the other metrics' fields stay empty here.
struct MetricsResult {
    std::uint64_t frame_index = 0;
    std::optional<double> ssimulacra2;
    std::optional<double> butteraugli;
    std::optional<double> vmaf_v0;
    std::optional<double> vmaf_v1;
    std::optional<double> cvvdp;
    std::optional<double> psnr_hvs;
};

struct MetricsFinalResult {
    std::optional<MetricsResult> last_frame;
    std::uint64_t frames = 0;
    std::optional<MetricsResult> penultimate_frame;
};

// vqm_metrics.h:63-75: `scratch` holds the pipeline's memory (its device
// arena and pinned pool); `spatial`, the SSIMULACRA 2 entry, holds what it
// keeps beside that, which is nothing; the other metrics' entries are empty.
struct MetricsMemoryUsage {
    std::optional<PipelineMemoryUsage> spatial;
    std::optional<PipelineMemoryUsage> vmaf_v0;
    std::optional<PipelineMemoryUsage> vmaf_v1;
    std::optional<PipelineMemoryUsage> cvvdp;
    std::optional<PipelineMemoryUsage> psnr_hvs;
    std::optional<PipelineMemoryUsage> scratch;
};

// Metrics (include/vqm_metrics.h:147-217, src/metrics/metrics.cc:83-396) with
// SSIMULACRA 2 as the selected metric. SSIMULACRA 2 has no lookahead, so
// Compute returns each frame's result at once and Flush returns nothing; the
// sequence rules are the reference's: after a failed call only Reset helps,
// after Flush/Finalize the sequence is finished until Reset, and ComputeImage
// needs a fresh sequence and resets it afterwards.
class Metrics {
public:
    explicit Metrics(MetricsConfig config) : config_(config) {
        if (!config_.ssimulacra2)
            throw std::invalid_argument("metrics: select at least one metric");
        Ssimulacra2Config c = *config_.ssimulacra2;
        c.size = config_.size;
        c.streaming_inputs = config_.streaming_inputs;
        c.memory_policy = config_.memory_policy;
        c.gpu_resident_images = 0;
        c.input_bytes = 0;
        pipeline_.emplace(c);
    }

    [[nodiscard]] std::optional<MetricsResult> Compute(const Image& o, const Image& d) {
        return Run([&] { return pipeline_->Compute(o, d, config_.background); },
                   [&] { Storage(o, "original"), Storage(d, "distorted"); }, o.size, o.format,
                   d.size, d.format, true);
    }
    [[nodiscard]] std::optional<MetricsResult> Compute(const ImageView& o, const ImageView& d) {
        return Run([&] { return pipeline_->Compute(o, d, config_.background); },
                   [&] { Storage(o, "original"), Storage(d, "distorted"); }, o.size, o.format,
                   d.size, d.format, true);
    }
    // Tightly packed planes in the configured formats, exactly RequiredBytes
    // each.
    [[nodiscard]] std::optional<MetricsResult> Compute(std::span<const std::byte> o,
                                                       std::span<const std::byte> d) {
        const Image a = Packed(o, config_.original_format, "original");
        const Image b = Packed(d, config_.distorted_format, "distorted");
        return Compute(a, b);
    }
    [[nodiscard]] std::optional<MetricsResult> Compute(const CudaBufferView& o,
                                                       const CudaBufferView& d) {
        return Run([&] { return pipeline_->Compute(o, d, config_.background); },
                   [&] { Storage(o, "original"), Storage(d, "distorted"); }, o.size, o.format,
                   d.size, d.format, false);
    }

    [[nodiscard]] MetricsResult ComputeImage(const Image& o, const Image& d) {
        return Still([&] { return Compute(o, d); });
    }
    [[nodiscard]] MetricsResult ComputeImage(const ImageView& o, const ImageView& d) {
        return Still([&] { return Compute(o, d); });
    }
    [[nodiscard]] MetricsResult ComputeImage(std::span<const std::byte> o,
                                             std::span<const std::byte> d) {
        return Still([&] { return Compute(o, d); });
    }
    [[nodiscard]] MetricsResult ComputeImage(const CudaBufferView& o, const CudaBufferView& d) {
        return Still([&] { return Compute(o, d); });
    }

    [[nodiscard]] std::optional<MetricsResult> Flush() {
        if (failed_) throw std::logic_error("metrics: previous call failed; call Reset");
        finished_ = true;
        return std::nullopt;
    }
    [[nodiscard]] MetricsFinalResult Finalize() {
        (void)Flush();
        MetricsFinalResult r;
        r.frames = next_index_;
        return r;
    }
    void Reset() {
        next_index_ = 0;
        failed_ = false;
        finished_ = false;
    }
    [[nodiscard]] MetricsMemoryUsage GetMemoryUsage() const {
        MetricsMemoryUsage u;
        u.scratch = pipeline_->GetMemoryUsage();
        u.spatial = PipelineMemoryUsage{};
        return u;
    }

private:
    static bool SameFormat(const ImageFormat& a, const ImageFormat& b) {
        return a.type == b.type && a.family == b.family && a.alpha == b.alpha &&
               a.range == b.range && a.matrix == b.matrix && a.transfer == b.transfer &&
               a.primaries == b.primaries && a.chroma_location == b.chroma_location &&
               a.subsample_w == b.subsample_w && a.subsample_h == b.subsample_h &&
               a.depth == b.depth;
    }
    Image Packed(std::span<const std::byte> bytes, const ImageFormat& f, const char* name) const {
        (void)name;
        if (bytes.size() != RequiredBytes(f, config_.size))
            throw std::invalid_argument("metrics: packed input has incorrect size");
        Image img;
        img.size = config_.size;
        img.format = f;
        img.data.resize(bytes.size());
        std::memcpy(img.data.data(), bytes.data(), bytes.size());
        return img;
    }
    // Checks of the inputs' storage (metrics.cc:46-58): made before the
    // frame is attempted, so a rejected input does not fail the sequence.
    static void Storage(const Image& img, const char* name) {
        ValidateFormat(img.format, img.size, name);
        (void)detail::ToC(img, name);
    }
    static void Storage(const ImageView& v, const char*) { (void)detail::CheckView(v); }
    static void Storage(const CudaBufferView& v, const char* name) {
        ValidateFormat(v.format, v.size, name);
    }
    template <class F, class S>
    std::optional<MetricsResult> Run(F&& compute, S&& storage, Size os, const ImageFormat& of,
                                     Size ds, const ImageFormat& df, bool host) {
        if (failed_) throw std::logic_error("metrics: previous call failed; call Reset");
        if (finished_) throw std::logic_error("metrics: sequence finished; call Reset");
        if (next_index_ == ~std::uint64_t{0})
            throw std::overflow_error("metrics: too many frames");
        if (!(os == config_.size) || !(ds == config_.size))
            throw std::invalid_argument("metrics: image size differs from configured size");
        if (!SameFormat(of, config_.original_format) || !SameFormat(df, config_.distorted_format))
            throw std::invalid_argument("metrics: image format differs from configured format");
        storage();
        if (host && !config_.streaming_inputs)
            throw std::invalid_argument("metrics: streaming inputs are disabled");
        try {
            MetricsResult r;
            r.frame_index = next_index_;
            r.ssimulacra2 = compute().Score();
            ++next_index_;
            return r;
        } catch (...) {
            failed_ = true;
            throw;
        }
    }
    template <class F>
    MetricsResult Still(F&& first) {
        if (failed_) throw std::logic_error("metrics: previous call failed; call Reset");
        if (finished_) throw std::logic_error("metrics: sequence finished; call Reset");
        if (next_index_ != 0)
            throw std::logic_error("metrics: reset the active sequence before ComputeImage");
        std::optional<MetricsResult> r = first();
        Reset();
        return *r;
    }

    MetricsConfig config_;
    std::optional<Ssimulacra2Pipeline> pipeline_;
    std::uint64_t next_index_ = 0;
    bool failed_ = false;
    bool finished_ = false;
};

}  // namespace vqm::cuda
