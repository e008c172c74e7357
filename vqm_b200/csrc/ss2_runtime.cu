// Host runtime of the SSIMULACRA 2.1 scorer and its C ABI (vqm_cu_ss2.h).
//
// Two objects sit behind the ABI:
//   Pipeline  one geometry, one pair in flight: VQM's Ssimulacra2Pipeline
//             (include/ssimulacra2.h:83-215) with CUDA in place of Vulkan.
//             Its device tables never change after construction, so each
//             pair is one CUDA-graph replay of [descriptor upload, prepare,
//             blur, finalize, result read-back].
//   Batch     any number of pairs of any sizes and formats, scored by one
//             launch per stage over all of them (the batched path).
//
// Handles and tokens follow VQM's src/handles.h: a process-wide incarnation
// counter packed with a 12-bit slot index, so stale or foreign handles never
// alias a live one.

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/vqm_cu_ss2.h"
#include "ss2_device.cuh"
#include "ss2_host.h"
#include "ss2_kernels.h"
#include "ss2_layout.h"

namespace vqm_b200 {
namespace {

thread_local std::string g_last_error;

struct CudaFailure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void Check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw CudaFailure(std::string("cuda: ") + what + ": " + cudaGetErrorString(e));
}
#define VQM_CK(call) Check((call), #call)

constexpr uint32_t kIndexBits = 12;
constexpr uint64_t kIndexMask = (1u << kIndexBits) - 1u;
constexpr uint64_t kIncarnationMax = UINT64_MAX >> kIndexBits;

std::atomic<uint64_t> g_incarnation{0};

// handles.h:27-30: never wraps, never reused.
uint64_t NextIncarnation() {
    const uint64_t v = g_incarnation.fetch_add(1) + 1;
    if (v > kIncarnationMax) throw std::overflow_error("handle identifiers exhausted");
    return v;
}

// An NVTX range (a named span on the Nsight Systems timeline) over a scope:
// the host side of a submission, or the wait for its results. Without a tool
// attached, NVTX v3 calls return at once.
class TraceRange {
public:
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

constexpr const char* kCapacityError =
    "resident image capacity exhausted; raise gpu_resident_images";

// Per-device one-time constant upload (score weights).
void EnsureDevice(int device) {
    static std::mutex mu;
    static std::vector<bool> ready;
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0) throw std::invalid_argument("cuda: invalid device ordinal");
    if (ready.size() <= static_cast<size_t>(device)) ready.resize(device + 1, false);
    if (ready[device]) return;
    VQM_CK(cudaSetDevice(device));
    VQM_CK(SetConstants(ScoreWeights()));
    // Kernels load lazily on their first launch otherwise: a first batch,
    // or the first that selects a new blur variant, would pay for it.
    VQM_CK(PreloadPrepare());
    VQM_CK(PreloadBlur());
    ready[device] = true;
}

// The device a config's device = -1 names once SetDefaultDevice chose one
// (process-wide, as VQM's default device is); -1: the thread's current one.
std::atomic<int> g_default_device{-1};

int ResolveDevice(int32_t requested) {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        throw std::runtime_error("cuda: no usable compute device");
    int device = requested;
    if (device < 0) device = g_default_device.load();
    if (device < 0) VQM_CK(cudaGetDevice(&device));
    if (device >= count) throw std::invalid_argument("cuda: invalid device ordinal");
    return device;
}

// Device allocation that only grows.
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) {
        o.ptr_ = nullptr;
        o.bytes_ = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&&) = delete;
    ~DeviceBuffer() { reset(); }
    void reset() {
        if (ptr_) cudaFree(ptr_);
        ptr_ = nullptr;
        bytes_ = 0;
    }
    // The size ensure(bytes) leaves: unchanged if it suffices, else bytes,
    // and at least half again the old size when one was held.
    size_t grown(size_t bytes) const {
        if (bytes <= bytes_) return bytes_;
        return bytes_ ? std::max(bytes, bytes_ + bytes_ / 2) : bytes;
    }
    // Returns true when the address changed. A buffer that has to grow
    // grows by half again at least, so a scorer fed batches of varying sizes
    // reallocates (and synchronises the device) a few times, not per batch.
    bool ensure(size_t bytes) {
        if (bytes <= bytes_) return false;
        bytes = grown(bytes);
        reset();
        if (cudaMalloc(&ptr_, bytes) != cudaSuccess) {
            ptr_ = nullptr;
            cudaGetLastError();
            throw std::runtime_error("cuda: device allocation of " + std::to_string(bytes) +
                                     " bytes failed");
        }
        bytes_ = bytes;
        return true;
    }
    template <class T>
    T* as() const { return static_cast<T*>(ptr_); }
    size_t bytes() const { return bytes_; }

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
};

class PinnedBuffer {
public:
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() { reset(); }
    void reset() {
        if (ptr_) cudaFreeHost(ptr_);
        ptr_ = nullptr;
        bytes_ = 0;
    }
    bool ensure(size_t bytes) {
        if (bytes <= bytes_) return false;
        if (bytes_) bytes = std::max(bytes, bytes_ + bytes_ / 2);
        reset();
        if (cudaMallocHost(&ptr_, bytes) != cudaSuccess) {
            ptr_ = nullptr;
            cudaGetLastError();
            throw std::runtime_error("cuda: pinned host allocation failed");
        }
        bytes_ = bytes;
        return true;
    }
    template <class T>
    T* as() const { return static_cast<T*>(ptr_); }
    size_t bytes() const { return bytes_; }

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
};

size_t AlignUp(size_t v, size_t a) { return (v + a - 1) / a * a; }

// An IEEE binary16 value (its bits) as float; every binary16 is a float.
float HalfBitsToFloat(uint16_t h) {
    const uint32_t sign = static_cast<uint32_t>(h & 0x8000u) << 16;
    const uint32_t exp = (h >> 10) & 0x1fu, man = h & 0x3ffu;
    uint32_t bits;
    if (exp == 0x1fu) {
        bits = sign | 0x7f800000u | (man << 13);
    } else if (exp != 0) {
        bits = sign | ((exp + 112u) << 23) | (man << 13);
    } else if (man == 0) {
        bits = sign;
    } else {  // subnormal: man * 2^-24
        float f = static_cast<float>(man) * 5.9604644775390625e-8f;
        std::memcpy(&bits, &f, 4);
        bits |= sign;
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// ---------------------------------------------------------------------------
// Batch tables: pyramid plane offsets, work segments and prefix offsets.
// ---------------------------------------------------------------------------

// The blur kernel variant and its output tile.
struct BlurShape {
    int variant = kDefaultBlurVariant;
    int w = 32, h = 32;
    static BlurShape Of(int variant) {
        BlurShape s;
        s.variant = variant;
        BlurTileShape(variant, &s.w, &s.h);
        return s;
    }
    BlurShape() { BlurTileShape(variant, &w, &h); }
};

struct Tables {
    std::vector<DevPair> pairs;
    std::vector<DevSegment> segs;
    std::vector<DevPrepItem> prep_items;  // the images, by prepare group
    std::vector<uint32_t> prep_start;     // every group's prefix offsets
    uint32_t prep_count[kPrepGroups] = {}, prep_blocks[kPrepGroups] = {};
    std::vector<uint32_t> blur_start;
    std::vector<size_t> pyramid_first;  // float offset of each pair's planes
    size_t pyramid_floats = 0;
    size_t partials = 0;  // tile partial count
};

// Lays out pairs of the given sizes. Plane pointers are filled later, once
// the pyramid allocation is known (FillPointers).
Tables BuildTables(const std::vector<std::pair<uint32_t, uint32_t>>& sizes, BlurShape shape) {
    Tables t;
    t.pairs.resize(sizes.size());
    t.blur_start.push_back(0);
    uint64_t prep = 0, blur = 0;
    for (size_t i = 0; i < sizes.size(); ++i) {
        DevPair& P = t.pairs[i];
        std::memset(static_cast<void*>(&P), 0, sizeof(DevPair));
        const ScalePlan plan = PlanScales(sizes[i].first, sizes[i].second);
        P.levels = static_cast<uint32_t>(plan.count);
        size_t floats = 0;
        for (int l = 0; l < plan.count; ++l) {
            P.w[l] = plan.w[l];
            P.h[l] = plan.h[l];
            P.pitch[l] = RowPairPitch(plan.w[l]);
            P.mask[l] = plan.mask[l];
            for (int c = 0; c < 3; ++c) {
                if (!(plan.mask[l] & (1u << c))) continue;
                P.plane_off[l][c] = floats;
                floats += PlaneFloats(plan.w[l], plan.h[l]);
            }
        }
        P.image_stride = floats;
        t.pyramid_first.push_back(t.pyramid_floats);
        t.pyramid_floats += AlignUp(2 * floats, 64);
        P.prep_tiles_x = PrepTiles(sizes[i].first);
        P.prep_tiles_y = PrepTiles(sizes[i].second);
        prep += 2ull * P.prep_tiles_x * P.prep_tiles_y;
        P.seg_first = static_cast<uint32_t>(t.segs.size());
        for (int l = 0; l < plan.count; ++l)
            for (int c = 0; c < 3; ++c) {
                if (!(plan.mask[l] & (1u << c))) continue;
                DevSegment s{};
                s.pair = static_cast<uint32_t>(i);
                s.level = static_cast<uint32_t>(l);
                s.channel = static_cast<uint32_t>(c);
                s.tiles_x = (plan.w[l] + shape.w - 1) / shape.w;
                const uint32_t ty = (plan.h[l] + shape.h - 1) / shape.h;
                s.tiles = s.tiles_x * ty;
                s.partial_first = static_cast<uint32_t>(t.partials);
                s.partials = BlurBlocks(shape.variant, s.tiles_x, ty);
                t.partials += s.partials;
                blur += s.partials;
                t.segs.push_back(s);
                t.blur_start.push_back(static_cast<uint32_t>(blur));
            }
        P.seg_count = static_cast<uint32_t>(t.segs.size()) - P.seg_first;
    }
    if (prep > 0x7fffffffull || blur > 0x7fffffffull)
        throw std::invalid_argument("cuda: batch too large for one launch");
    t.prep_items.resize(2 * sizes.size());
    t.prep_start.resize(2 * sizes.size() + kPrepGroups);
    return t;
}

// The tile grids (columns, rows) of the default tile over every kept
// (pair, level, channel), in the blur's launch order.
std::vector<std::pair<uint32_t, uint32_t>> DefaultTileGrids(
    const std::vector<std::pair<uint32_t, uint32_t>>& sizes) {
    int tw = 0, th = 0;
    BlurTileShape(kDefaultBlurVariant, &tw, &th);
    std::vector<std::pair<uint32_t, uint32_t>> grids;
    for (const auto& wh : sizes) {
        const ScalePlan plan = PlanScales(wh.first, wh.second);
        for (int l = 0; l < plan.count; ++l)
            for (int c = 0; c < 3; ++c)
                if (plan.mask[l] & (1u << c))
                    grids.emplace_back((plan.w[l] + tw - 1) / tw, (plan.h[l] + th - 1) / th);
    }
    return grids;
}

int DeviceSms(int device) {
    int sms = 0;
    VQM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    return sms;
}

// Splits the images into the prepare groups (group[i][k]: PrepGroup of
// image k of pair i) and lays out each group's prefix tile offsets. The list
// sizes do not depend on the split. `skip_original`, when set, leaves every
// pair's image 0 out (its pyramid is already in place).
using PrepGroups = std::vector<std::array<uint8_t, 2>>;
void BuildPrepLists(Tables& t, const PrepGroups& group, bool skip_original = false) {
    uint32_t n[kPrepGroups] = {};
    for (size_t i = 0; i < t.pairs.size(); ++i)
        for (int k = skip_original ? 1 : 0; k < 2; ++k) ++n[group[i][k]];
    uint32_t first[kPrepGroups];   // the group's first item
    uint32_t* start[kPrepGroups];  // the group's prefix offsets
    uint32_t blocks[kPrepGroups] = {};
    for (uint32_t g = 0, items = 0; g < kPrepGroups; items += n[g], ++g) {
        first[g] = items;
        start[g] = t.prep_start.data() + items + g;
        start[g][0] = 0;
    }
    uint32_t at[kPrepGroups] = {};
    for (size_t i = 0; i < t.pairs.size(); ++i)
        for (uint32_t k = skip_original ? 1 : 0; k < 2; ++k) {
            const int g = group[i][k];
            const uint32_t pos = at[g]++;
            t.prep_items[first[g] + pos] = DevPrepItem{static_cast<uint32_t>(i), k};
            blocks[g] += t.pairs[i].prep_tiles_x * t.pairs[i].prep_tiles_y;
            start[g][pos + 1] = blocks[g];
        }
    for (int g = 0; g < kPrepGroups; ++g) {
        t.prep_count[g] = n[g];
        t.prep_blocks[g] = blocks[g];
    }
}

// The device tables of one batch: one table allocation, its pinned mirror,
// the pyramid, partials, segment sums and per-pair counters, and the pinned
// host blocks the results land in.
struct BatchMemory {
    DeviceBuffer table, pyramid, partials, seg_sums, pair_done;
    PinnedBuffer table_host, results_host;
    // Table layout: [pairs | prep items | prep starts | segments | blur
    // starts]. Everything a call can change (pair records, which images take
    // the table path) sits in the first `head_bytes`.
    size_t off_pairs = 0, off_items = 0, off_prep = 0, off_segs = 0, off_blur = 0;
    size_t head_bytes = 0, table_bytes = 0;
    DevBatch dev{};
    uint32_t pair_count = 0;
    size_t elem_bytes = 4;  // pyramid element: float, or binary16 with half planes

    // The blur mode's taps, carried by every launch of this memory's tables.
    void SetBlur(uint32_t blur) {
        const std::array<float, kTaps> taps = BlurTaps(blur);
        for (int i = 0; i < kTaps; ++i) dev.taps2[i] = make_float2(taps[i], taps[i]);
    }

    // Device bytes each buffer needs for `t`, in the order table, pyramid,
    // partials, segment sums, pair counters (and the table offsets).
    std::array<size_t, 5> Needs(const Tables& t) {
        off_pairs = 0;
        off_items = AlignUp(off_pairs + sizeof(DevPair) * t.pairs.size(), 16);
        off_prep = AlignUp(off_items + sizeof(DevPrepItem) * t.prep_items.size(), 16);
        head_bytes = AlignUp(off_prep + sizeof(uint32_t) * t.prep_start.size(), 256);
        off_segs = head_bytes;
        off_blur = AlignUp(off_segs + sizeof(DevSegment) * t.segs.size(), 256);
        table_bytes = AlignUp(off_blur + sizeof(uint32_t) * t.blur_start.size(), 256);
        return {table_bytes, std::max<size_t>(t.pyramid_floats, 64) * elem_bytes,
                std::max<size_t>(t.partials, 1) * 6 * sizeof(double),
                std::max<size_t>(t.segs.size(), 1) * 6 * sizeof(double),
                (t.pairs.size() + t.segs.size() + 2) * sizeof(uint32_t)};
    }
    std::array<DeviceBuffer*, 5> Buffers() {
        return {&table, &pyramid, &partials, &seg_sums, &pair_done};
    }
    // Device bytes held now.
    size_t DeviceBytes() {
        size_t n = 0;
        for (DeviceBuffer* b : Buffers()) n += b->bytes();
        return n;
    }
    void ReleaseDevice() {
        for (DeviceBuffer* b : Buffers()) b->reset();
    }

    // Sizes and uploads-to-be for `t`; returns true if any address moved.
    bool Layout(const Tables& t) {
        bool moved = false;
        const std::array<size_t, 5> need = Needs(t);
        moved |= table.ensure(need[0]);
        moved |= table_host.ensure(table_bytes);
        moved |= pyramid.ensure(need[1]);
        moved |= partials.ensure(need[2]);
        moved |= seg_sums.ensure(need[3]);
        if (pair_done.ensure(need[4])) {
            moved = true;
            // New counters start at zero; wait for it, as launches run on
            // streams that do not wait for the legacy stream's memset.
            VQM_CK(cudaMemset(pair_done.as<void>(), 0, pair_done.bytes()));
            VQM_CK(cudaStreamSynchronize(nullptr));
        }
        moved |= results_host.ensure(std::max<size_t>(t.pairs.size(), 1) * kResultDoubles * sizeof(double));
        pair_count = static_cast<uint32_t>(t.pairs.size());
        uint8_t* base = table.as<uint8_t>();
        dev.pairs = static_cast<uint32_t>(t.pairs.size());
        dev.segments = static_cast<uint32_t>(t.segs.size());
        dev.blur_blocks = t.blur_start.back();
        dev.pair = reinterpret_cast<const DevPair*>(base + off_pairs);
        dev.seg = reinterpret_cast<const DevSegment*>(base + off_segs);
        dev.prep_item = reinterpret_cast<const DevPrepItem*>(base + off_items);
        dev.prep_start = reinterpret_cast<const uint32_t*>(base + off_prep);
        dev.blur_start = reinterpret_cast<const uint32_t*>(base + off_blur);
        dev.partials = partials.as<double>();
        dev.seg_sums = seg_sums.as<double>();
        dev.pair_done = pair_done.as<uint32_t>();
        dev.seg_done = pair_done.as<uint32_t>() + t.pairs.size();
        dev.blur_queue = dev.seg_done + t.segs.size();
        dev.status = nullptr;
        dev.half = elem_bytes == 2 ? 1u : 0u;
        return moved;
    }

    // Writes the host mirror of the tables with device pointers filled in.
    void Stage(Tables& t) {
        for (size_t i = 0; i < t.pairs.size(); ++i) {
            t.pairs[i].pyramid =
                reinterpret_cast<float*>(pyramid.as<uint8_t>() + t.pyramid_first[i] * elem_bytes);
            // Pinned host memory, which the device reaches at the same
            // address: the blur's epilogue writes each result across the
            // bus once, and no copy follows the kernels.
            t.pairs[i].result = results_host.as<double>() + i * kResultDoubles;
        }
        uint8_t* h = table_host.as<uint8_t>();
        std::memcpy(h + off_pairs, t.pairs.data(), sizeof(DevPair) * t.pairs.size());
        std::memcpy(h + off_segs, t.segs.data(), sizeof(DevSegment) * t.segs.size());
        std::memcpy(h + off_blur, t.blur_start.data(), sizeof(uint32_t) * t.blur_start.size());
        StagePrep(t);
    }
    // The prepare lists (after BuildPrepLists) into the host mirror and the
    // kernel parameters.
    void StagePrep(const Tables& t) {
        uint8_t* h = table_host.as<uint8_t>();
        std::memcpy(h + off_items, t.prep_items.data(), sizeof(DevPrepItem) * t.prep_items.size());
        std::memcpy(h + off_prep, t.prep_start.data(), sizeof(uint32_t) * t.prep_start.size());
        for (int g = 0; g < kPrepGroups; ++g) {
            dev.prep_items[g] = t.prep_count[g];
            dev.prep_blocks[g] = t.prep_blocks[g];
        }
    }
    DevPair* HostPair(size_t i) {
        return reinterpret_cast<DevPair*>(table_host.as<uint8_t>() + off_pairs) + i;
    }

    void EnqueueUpload(size_t bytes, cudaStream_t s) {
        VQM_CK(cudaMemcpyAsync(table.as<void>(), table_host.as<void>(), bytes,
                               cudaMemcpyHostToDevice, s));
    }
    // ev, when given, holds 4 timing events recorded before prepare and
    // after prepare, blur and the (fused) finalize: the last two are back
    // to back, the finalize work being the blur's epilogue.
    void EnqueueKernels(BlurShape shape, cudaStream_t s, cudaEvent_t* ev = nullptr) {
        if (ev) VQM_CK(cudaEventRecord(ev[0], s));
        VQM_CK(LaunchPrepare(dev, s));
        if (ev) VQM_CK(cudaEventRecord(ev[1], s));
        VQM_CK(LaunchBlur(dev, shape.variant, s));
        if (ev) VQM_CK(cudaEventRecord(ev[2], s));
        if (ev) VQM_CK(cudaEventRecord(ev[3], s));
    }
};

// ---------------------------------------------------------------------------
// Image sources.
// ---------------------------------------------------------------------------

void CheckGeometry(const vqm_cu_image& img, uint32_t w, uint32_t h, const char* name) {
    if (img.width != w || img.height != h)
        throw std::invalid_argument(std::string(name) +
                                    ": image size does not match the pipeline geometry");
}

// Fills src's plane pointers and sizes for an image whose planes are at
// `planes` with byte strides `strides` (0 = packed rows).
void FillPlanes(DevSource& src, const vqm_cu_format& f, uint32_t w, uint32_t h,
                const void* const planes[4], const size_t strides[4], const char* name) {
    const auto layout = PlaneLayout(f, w, h);
    for (int p = 0; p < 4; ++p) {
        src.plane[p] = nullptr;
        src.row_bytes[p] = 0;
        src.plane_w[p] = static_cast<uint32_t>(layout[p].width);
        src.plane_h[p] = static_cast<uint32_t>(layout[p].height);
        if (!layout[p].present()) continue;
        if (planes[p] == nullptr)
            throw std::invalid_argument(std::string(name) + ": plane " + std::to_string(p) +
                                        " is null");
        const size_t row = layout[p].width * layout[p].sample_bytes;
        const size_t stride = strides[p] ? strides[p] : row;
        if (stride < row)
            throw std::invalid_argument(std::string(name) + ": plane stride is shorter than a row");
        if (stride % layout[p].sample_bytes != 0 ||
            reinterpret_cast<uintptr_t>(planes[p]) % layout[p].sample_bytes != 0)
            throw std::invalid_argument(std::string(name) +
                                        ": plane address or stride is not sample aligned");
        if (stride > 0xffffffffull) throw std::overflow_error("plane stride exceeds 32 bits");
        src.plane[p] = static_cast<const uint8_t*>(planes[p]);
        src.row_bytes[p] = static_cast<uint32_t>(stride);
    }
    src.width = w;
    src.height = h;
}

// Copies a host image into a packed device buffer (vqm::Image's layout).
// Planes whose rows are packed go as linear copies, and planes that also
// follow one another without a gap in both the host image and the packed
// layout (a vqm::Image buffer, for one) go as one copy: a 2D copy of short
// rows, or several copies of one image, leave the copy engine idle between
// rows and between copies.
void CopyHostImage(const vqm_cu_image& img, uint8_t* dst, cudaStream_t stream) {
    const auto layout = PlaneLayout(img.format, img.width, img.height);
    const uint8_t* run_src = nullptr;  // the pending linear run
    size_t run_offset = 0, run_bytes = 0;
    const auto flush = [&] {
        if (run_bytes)
            VQM_CK(cudaMemcpyAsync(dst + run_offset, run_src, run_bytes, cudaMemcpyHostToDevice,
                                   stream));
        run_bytes = 0;
    };
    for (int p = 0; p < 4; ++p) {
        if (!layout[p].present()) continue;
        const size_t row = layout[p].width * layout[p].sample_bytes;
        const size_t stride = img.strides[p] ? img.strides[p] : row;
        if (img.planes[p] == nullptr) throw std::invalid_argument("image: plane is null");
        if (stride < row) throw std::invalid_argument("image: plane stride is shorter than a row");
        const auto* src = static_cast<const uint8_t*>(img.planes[p]);
        if (stride != row) {
            flush();
            VQM_CK(cudaMemcpy2DAsync(dst + layout[p].offset, row, src, stride, row,
                                     layout[p].height, cudaMemcpyHostToDevice, stream));
            continue;
        }
        const size_t bytes = row * layout[p].height;
        if (run_bytes && run_src + run_bytes == src && run_offset + run_bytes == layout[p].offset) {
            run_bytes += bytes;
            continue;
        }
        flush();
        run_src = src;
        run_offset = layout[p].offset;
        run_bytes = bytes;
    }
    flush();
}

void PackedPlanes(const vqm_cu_format& f, uint32_t w, uint32_t h, const uint8_t* base,
                  const void* planes[4], size_t strides[4]) {
    const auto layout = PlaneLayout(f, w, h);
    for (int p = 0; p < 4; ++p) {
        planes[p] = layout[p].present() ? base + layout[p].offset : nullptr;
        strides[p] = 0;
    }
}

// ---------------------------------------------------------------------------
// Pipeline.
// ---------------------------------------------------------------------------

struct Slot {
    bool live = false;
    uint64_t generation = 0;
    DeviceBuffer memory;
    vqm_cu_format format{};
};

struct InputAlloc {
    bool live = false;
    uint64_t generation = 0;
    size_t offset = 0, bytes = 0;
    vqm_cu_format format{};
};

class Pipeline {
public:
    explicit Pipeline(const vqm_cu_ss2_config& cfg) : cfg_(cfg) {
        plan_ = PlanScales(cfg.width, cfg.height);
        if (cfg.gpu_resident_images > kIndexMask)
            throw std::invalid_argument("gpu_resident_images is limited to " +
                                        std::to_string(kIndexMask) + " slots");
        if (cfg.chroma_filter > 2) throw std::invalid_argument("invalid chroma filter");
        // Half planes (ssimulacra2.h:41-46): binary16 pyramid elements, FP32
        // arithmetic, the level averages rounded like the planes.
        mem_.elem_bytes = cfg.half_planes ? 2 : 4;
        mem_.SetBlur(cfg.blur);
        if (cfg.memory_policy > VQM_CU_MEMORY_POLICY_STAGED)
            throw std::invalid_argument("cuda: invalid memory policy");
        staged_ = cfg.memory_policy == VQM_CU_MEMORY_POLICY_STAGED;
        device_ = ResolveDevice(cfg.device);
        EnsureDevice(device_);
        VQM_CK(cudaSetDevice(device_));
        VQM_CK(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
        stream_ = own_stream_;
        VQM_CK(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming));
        VQM_CK(cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming));
        if (!cfg.half_planes)
            shape_ = BlurShape::Of(
                AutoBlurVariant(DefaultTileGrids({{cfg.width, cfg.height}}), DeviceSms(device_)));
        tables_ = BuildTables({{cfg.width, cfg.height}}, shape_);
        BuildPrepLists(tables_, {{0, 0}});
        mem_.Layout(tables_);
        mem_.Stage(tables_);
        VQM_CK(cudaMemcpy(mem_.table.as<void>(), mem_.table_host.as<void>(), mem_.table_bytes,
                          cudaMemcpyHostToDevice));
        slots_.resize(cfg.gpu_resident_images);
        if (cfg.input_bytes) pool_.ensure(cfg.input_bytes);
        if (cfg.input_bytes && staged_) pool_device_.ensure(cfg.input_bytes);
    }
    ~Pipeline() {
        cudaSetDevice(device_);
        if (stream_) cudaStreamSynchronize(stream_);
        for (auto& g : graph_exec_)
            if (g) cudaGraphExecDestroy(g);
        if (done_) cudaEventDestroy(done_);
        if (copied_) cudaEventDestroy(copied_);
        if (own_stream_) cudaStreamDestroy(own_stream_);
    }

    void SetStream(void* s) {
        RequireIdle();
        stream_ = s ? static_cast<cudaStream_t>(s) : own_stream_;
    }
    void* GetStream() const { return stream_; }
    // Submissions that reused the cached original's pyramid.
    uint64_t ReferenceReuses() const { return reference_reuses_; }
    bool InFlight() const { return in_flight_; }
    void SetGraphs(bool on) {
        RequireIdle();
        graphs_ = on;
    }

    void RequireIdle(const char* what = nullptr) const {
        if (!in_flight_) return;
        if (what)
            throw std::logic_error(std::string("cuda: ") + what +
                                   " while a submission is in flight; Finish it first");
        throw std::logic_error("cuda: a submission is already in flight; Finish it first");
    }

    uint64_t SubmitImages(const vqm_cu_image* o, const vqm_cu_image* d, float bg,
                          void* const* waits = nullptr, uint32_t nwaits = 0,
                          void* const* signals = nullptr, uint32_t nsignals = 0) {
        RequireIdle();
        const vqm_cu_image* imgs[2] = {o, d};
        const char* names[2] = {"original", "distorted"};
        for (int i = 0; i < 2; ++i) {
            if (!imgs[i]) throw std::invalid_argument(std::string(names[i]) + ": image is null");
            CheckGeometry(*imgs[i], cfg_.width, cfg_.height, names[i]);
            ValidateFormat(imgs[i]->format, imgs[i]->width, imgs[i]->height, names[i]);
            if (imgs[i]->memory != VQM_CU_MEMORY_HOST && imgs[i]->memory != VQM_CU_MEMORY_DEVICE)
                throw std::invalid_argument(std::string(names[i]) + ": invalid memory kind");
            if (imgs[i]->memory == VQM_CU_MEMORY_HOST && !cfg_.streaming_inputs)
                throw std::invalid_argument("cuda: streaming_inputs is false");
        }
        VQM_CK(cudaSetDevice(device_));
        for (uint32_t k = 0; k < nwaits; ++k)
            VQM_CK(cudaStreamWaitEvent(stream_, static_cast<cudaEvent_t>(waits[k]), 0));
        for (int i = 0; i < 2; ++i) {
            const vqm_cu_image& img = *imgs[i];
            DevSource& src = mem_.HostPair(0)->src[i];
            BuildSourceConstants(img.format, cfg_.chroma_filter, bg, src);
            if (img.memory == VQM_CU_MEMORY_HOST) {
                const size_t need = RequiredBytes(img.format, img.width, img.height);
                stream_in_[i].ensure(AlignUp(need, 256));
                CopyHostImage(img, stream_in_[i].as<uint8_t>(), stream_);
                const void* planes[4];
                size_t strides[4];
                PackedPlanes(img.format, img.width, img.height, stream_in_[i].as<uint8_t>(),
                             planes, strides);
                FillPlanes(src, img.format, img.width, img.height, planes, strides, names[i]);
            } else {
                FillPlanes(src, img.format, img.width, img.height, img.planes, img.strides,
                           names[i]);
            }
        }
        const bool host = o->memory == VQM_CU_MEMORY_HOST || d->memory == VQM_CU_MEMORY_HOST;
        if (host) VQM_CK(cudaEventRecord(copied_, stream_));
        const uint64_t token = Launch();
        for (uint32_t k = 0; k < nsignals; ++k)
            VQM_CK(cudaEventRecord(static_cast<cudaEvent_t>(signals[k]), stream_));
        // ssimulacra2.h:106-113: host samples only need to stay readable until
        // Submit returns, so wait for the copies (not the kernels) here.
        if (host) VQM_CK(cudaEventSynchronize(copied_));
        return token;
    }

    uint64_t SubmitResident(uint64_t a, uint64_t b, float bg) {
        RequireIdle();
        const Slot& sa = RequireSlot(a, "original");
        const Slot& sb = RequireSlot(b, "distorted");
        VQM_CK(cudaSetDevice(device_));
        const Slot* s[2] = {&sa, &sb};
        for (int i = 0; i < 2; ++i) SourceFromDevice(i, s[i]->format, s[i]->memory.as<uint8_t>(), bg);
        return LaunchWithOriginal(a, bg);
    }

    uint64_t SubmitResidentImage(uint64_t a, const vqm_cu_image* d, float bg) {
        RequireIdle();
        if (!cfg_.streaming_inputs) throw std::invalid_argument("cuda: streaming_inputs is false");
        const Slot& sa = RequireSlot(a, "original");
        if (!d) throw std::invalid_argument("distorted: image is null");
        CheckGeometry(*d, cfg_.width, cfg_.height, "distorted");
        ValidateFormat(d->format, d->width, d->height, "distorted");
        VQM_CK(cudaSetDevice(device_));
        SourceFromDevice(0, sa.format, sa.memory.as<uint8_t>(), bg);
        DevSource& src = mem_.HostPair(0)->src[1];
        BuildSourceConstants(d->format, cfg_.chroma_filter, bg, src);
        if (d->memory == VQM_CU_MEMORY_HOST) {
            const size_t need = RequiredBytes(d->format, d->width, d->height);
            stream_in_[1].ensure(AlignUp(need, 256));
            CopyHostImage(*d, stream_in_[1].as<uint8_t>(), stream_);
            const void* planes[4];
            size_t strides[4];
            PackedPlanes(d->format, d->width, d->height, stream_in_[1].as<uint8_t>(), planes,
                         strides);
            FillPlanes(src, d->format, d->width, d->height, planes, strides, "distorted");
            VQM_CK(cudaEventRecord(copied_, stream_));
            const uint64_t token = LaunchWithOriginal(a, bg);
            VQM_CK(cudaEventSynchronize(copied_));
            return token;
        }
        FillPlanes(src, d->format, d->width, d->height, d->planes, d->strides, "distorted");
        return LaunchWithOriginal(a, bg);
    }

    uint64_t SubmitBuffers(uint64_t a, uint64_t b, float bg) {
        RequireIdle();
        const InputAlloc& ia = RequireInput(a);
        const InputAlloc& ib = RequireInput(b);
        VQM_CK(cudaSetDevice(device_));
        const uint8_t* base = pool_.as<uint8_t>();
        if (staged_) {
            // The two spans to the device mirror, ahead of the kernels.
            for (const InputAlloc* in : {&ia, &ib})
                VQM_CK(cudaMemcpyAsync(pool_device_.as<uint8_t>() + in->offset, base + in->offset,
                                       in->bytes, cudaMemcpyHostToDevice, stream_));
            base = pool_device_.as<uint8_t>();
        }
        SourceFromDevice(0, ia.format, base + ia.offset, bg);
        SourceFromDevice(1, ib.format, base + ib.offset, bg);
        return Launch();
    }

    void Finish(uint64_t token, double* norms, uint32_t* scales) {
        if (!in_flight_ || token != token_)
            throw std::invalid_argument("cuda: no submission with that token");
        TraceRange trace("ss2 pipeline finish");
        VQM_CK(cudaSetDevice(device_));
        const cudaError_t e = cudaEventSynchronize(done_);
        in_flight_ = false;
        if (e != cudaSuccess) reference_valid_ = false;
        Check(e, "pair execution");
        VQM_CK(cudaGetLastError());
        const double* r = mem_.results_host.as<double>();
        const int n = static_cast<int>(r[kResultScales]);
        if (n != plan_.count) throw std::runtime_error("cuda: result block is incomplete");
        if (norms) {
            for (int i = 0; i < 108; ++i) norms[i] = i < 18 * n ? r[i] : 0.0;
        }
        if (scales) *scales = static_cast<uint32_t>(n);
    }

    uint64_t Upload(const vqm_cu_image* img) {
        RequireIdle("Upload");
        if (!img) throw std::invalid_argument("image: image is null");
        CheckGeometry(*img, cfg_.width, cfg_.height, "image");
        ValidateFormat(img->format, img->width, img->height, "image");
        size_t index = slots_.size();
        for (size_t i = 0; i < slots_.size(); ++i)
            if (!slots_[i].live) {
                index = i;
                break;
            }
        if (index == slots_.size()) throw std::invalid_argument(kCapacityError);
        const uint64_t generation = NextIncarnation();
        VQM_CK(cudaSetDevice(device_));
        Slot& s = slots_[index];
        const size_t need = RequiredBytes(img->format, img->width, img->height);
        s.memory.ensure(AlignUp(need, 256));
        if (img->memory == VQM_CU_MEMORY_HOST) {
            CopyHostImage(*img, s.memory.as<uint8_t>(), stream_);
        } else {
            const auto layout = PlaneLayout(img->format, img->width, img->height);
            for (int p = 0; p < 4; ++p) {
                if (!layout[p].present()) continue;
                const size_t row = layout[p].width * layout[p].sample_bytes;
                VQM_CK(cudaMemcpy2DAsync(s.memory.as<uint8_t>() + layout[p].offset, row,
                                         img->planes[p], img->strides[p] ? img->strides[p] : row,
                                         row, layout[p].height, cudaMemcpyDeviceToDevice,
                                         stream_));
            }
        }
        VQM_CK(cudaStreamSynchronize(stream_));
        s.live = true;
        s.generation = generation;
        s.format = img->format;
        return (generation << kIndexBits) | (index + 1);
    }

    void Release(uint64_t handle) {
        RequireIdle("Release");
        if (reference_valid_ && handle == reference_handle_) reference_valid_ = false;
        const uint64_t idx = handle & kIndexMask;
        if (idx == 0 || idx > slots_.size()) return;
        Slot& s = slots_[idx - 1];
        if (!s.live || s.generation != (handle >> kIndexBits)) return;
        s.live = false;
    }

    uint64_t AllocateImage(const vqm_cu_format& f, size_t* bytes) {
        RequireIdle("AllocateImage");
        ValidateFormat(f, cfg_.width, cfg_.height, "image buffer");
        if (cfg_.input_bytes == 0)
            throw std::invalid_argument(
                "cuda: the input pool size is 0, so AllocateImage has no memory; set it to the "
                "bytes your frames need and construct again");
        const size_t need = RequiredBytes(f, cfg_.width, cfg_.height);
        if (need > cfg_.input_bytes) throw std::invalid_argument("cuda: the input pool is full");
        // First fit over the live spans, starts 64-byte aligned.
        std::vector<std::pair<size_t, size_t>> used;
        for (const auto& a : inputs_)
            if (a.live) used.emplace_back(a.offset, a.bytes);
        std::sort(used.begin(), used.end());
        size_t at = 0;
        bool found = false;
        for (const auto& u : used) {
            if (at + need <= u.first) {
                found = true;
                break;
            }
            at = AlignUp(u.first + u.second, 64);
        }
        if (!found && at + need <= cfg_.input_bytes) found = true;
        if (!found)
            throw std::invalid_argument(
                "cuda: the input pool is full; Release a buffer or raise the configured input "
                "bytes");
        size_t index = inputs_.size();
        for (size_t i = 0; i < inputs_.size(); ++i)
            if (!inputs_[i].live) {
                index = i;
                break;
            }
        if (index == inputs_.size()) {
            if (index >= kIndexMask)
                throw std::invalid_argument("cuda: maximum number of live image buffers reached");
            inputs_.emplace_back();
        }
        InputAlloc& a = inputs_[index];
        a.live = true;
        a.generation = NextIncarnation();
        a.offset = at;
        a.bytes = need;
        a.format = f;
        *bytes = need;
        return (a.generation << kIndexBits) | (index + 1);
    }

    void* MapImage(uint64_t handle) {
        RequireIdle("MapImage");
        const InputAlloc& a = RequireInput(handle);
        return pool_.as<uint8_t>() + a.offset;
    }

    void ReleaseImage(uint64_t handle) {
        if (in_flight_)
            throw std::logic_error(
                "cuda: Release while a submission is in flight would hand the span to the next "
                "AllocateImage while it is still being read; Finish first");
        const uint64_t idx = handle & kIndexMask;
        if (idx == 0 || idx > inputs_.size()) return;
        InputAlloc& a = inputs_[idx - 1];
        if (!a.live || a.generation != (handle >> kIndexBits)) return;
        a.live = false;
    }

    void DebugPlane(uint32_t image, uint32_t level, uint32_t channel, float* out) {
        RequireIdle("debug_plane");
        if (image > 1 || level >= static_cast<uint32_t>(plan_.count) || channel > 2)
            throw std::invalid_argument("cuda: no such plane");
        if (!(plan_.mask[level] & (1u << channel)))
            throw std::invalid_argument("cuda: the channel is pruned at this level");
        const DevPair& P = tables_.pairs[0];
        const size_t eb = mem_.elem_bytes;
        const uint8_t* src = mem_.pyramid.as<uint8_t>() +
                             (tables_.pyramid_first[0] + image * P.image_stride +
                              P.plane_off[level][channel]) * eb;
        const uint32_t w = P.w[level], h = P.h[level], pitch = P.pitch[level];
        std::vector<uint8_t> pairs(PlaneFloats(w, h) * eb);
        VQM_CK(cudaSetDevice(device_));
        VQM_CK(cudaMemcpy(pairs.data(), src, pairs.size(), cudaMemcpyDeviceToHost));
        for (uint32_t y = 0; y < h; ++y)
            for (uint32_t x = 0; x < w; ++x) {
                const size_t i = PlaneIndex(pitch, x, y);
                float v;
                if (eb == 2) {
                    uint16_t hbits;
                    std::memcpy(&hbits, &pairs[i * 2], 2);
                    v = HalfBitsToFloat(hbits);
                } else {
                    std::memcpy(&v, &pairs[i * 4], 4);
                }
                out[static_cast<size_t>(y) * w + x] = v;
            }
    }

    void Usage(vqm_cu_memory_usage* u) const {
        std::memset(u, 0, sizeof(*u));
        u->pyramid_bytes = mem_.pyramid.bytes();
        for (const auto& s : slots_) u->resident_bytes += s.memory.bytes();
        u->input_bytes = pool_.bytes() + pool_device_.bytes() + stream_in_[0].bytes() +
                         stream_in_[1].bytes();
        u->scratch_bytes = mem_.table.bytes() + mem_.partials.bytes() + mem_.seg_sums.bytes() +
                           mem_.pair_done.bytes();
        u->total_bytes = u->pyramid_bytes + u->resident_bytes + u->input_bytes + u->scratch_bytes;
        u->host_bytes = pool_.bytes();
        u->uses_staging = staged_ ? 1u : 0u;
    }

private:
    const Slot& RequireSlot(uint64_t handle, const char* name) const {
        const uint64_t idx = handle & kIndexMask;
        if (idx == 0 || idx > slots_.size() || !slots_[idx - 1].live ||
            slots_[idx - 1].generation != (handle >> kIndexBits))
            throw std::invalid_argument(std::string(name) + ": not a live resident image");
        return slots_[idx - 1];
    }
    const InputAlloc& RequireInput(uint64_t handle) const {
        const uint64_t idx = handle & kIndexMask;
        if (idx == 0 || idx > inputs_.size() || !inputs_[idx - 1].live ||
            inputs_[idx - 1].generation != (handle >> kIndexBits))
            throw std::invalid_argument(
                "cuda: image buffer is not live (released or stale handle)");
        return inputs_[idx - 1];
    }
    void SourceFromDevice(int i, const vqm_cu_format& f, const uint8_t* base, float bg) {
        DevSource& src = mem_.HostPair(0)->src[i];
        BuildSourceConstants(f, cfg_.chroma_filter, bg, src);
        const void* planes[4];
        size_t strides[4];
        PackedPlanes(f, cfg_.width, cfg_.height, base, planes, strides);
        FillPlanes(src, f, cfg_.width, cfg_.height, planes, strides, i == 0 ? "original" : "distorted");
    }

    // The reference-pyramid reuse of vulkan.cc:238-243, 714-736: when the
    // original is the same resident slot (same handle, so the same image) as
    // in the previous submission, with the same background, its pyramid
    // planes are still in place and its prepare is skipped. Only resident
    // slots are immutable; any other kind of submission, a Release of the
    // slot or a failed run forgets the cached original.
    uint64_t LaunchWithOriginal(uint64_t handle, float bg) {
        const bool reuse =
            reference_valid_ && handle == reference_handle_ && bg == reference_background_;
        reference_valid_ = false;
        const uint64_t token = Launch(reuse);
        if (reuse) ++reference_reuses_;
        reference_valid_ = true;
        reference_handle_ = handle;
        reference_background_ = bg;
        return token;
    }

    // [upload the pair record, prepare, blur, finalize, read back], as one
    // graph replay when graphs are on. `skip_original` leaves the original's
    // prepare out (its pyramid is cached).
    uint64_t Launch(bool skip_original = false) {
        TraceRange trace("ss2 pipeline launch");
        if (!skip_original) reference_valid_ = false;
        // Each image's prepare group, and whether the original is prepared,
        // decide the prepare launches; one graph per combination.
        const DevPair* hp = mem_.HostPair(0);
        const uint8_t g0 = static_cast<uint8_t>(PrepGroup(hp->src[0]));
        const uint8_t g1 = static_cast<uint8_t>(PrepGroup(hp->src[1]));
        // The YUV prepare kernel (and its window) depends on the images'
        // chroma subsampling too.
        bool yuv420 = true;
        for (int k = skip_original ? 1 : 0; k < 2; ++k)
            if (PrepGroup(hp->src[k]) == 1 && !Yuv420Window(hp->src[k])) yuv420 = false;
        mem_.dev.yuv420 = yuv420 ? 1u : 0u;
        const int key = g0 + kPrepGroups * (g1 + kPrepGroups * ((skip_original ? 1 : 0) +
                                                                 2 * (yuv420 ? 1 : 0)));
        BuildPrepLists(tables_, {{g0, g1}}, skip_original);
        mem_.StagePrep(tables_);
        const size_t upload = mem_.head_bytes;
        // Stream capture needs a real stream; the legacy default stream runs
        // the same work launch by launch.
        if (graphs_ && stream_ != nullptr) {
            cudaGraphExec_t& exec = graph_exec_[key];
            if (!exec) {
                cudaGraph_t graph = nullptr;
                VQM_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
                try {
                    mem_.EnqueueUpload(upload, stream_);
                    mem_.EnqueueKernels(shape_, stream_);
                } catch (...) {
                    cudaStreamEndCapture(stream_, &graph);
                    if (graph) cudaGraphDestroy(graph);
                    throw;
                }
                VQM_CK(cudaStreamEndCapture(stream_, &graph));
                const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                Check(e, "cudaGraphInstantiate");
            }
            VQM_CK(cudaGraphLaunch(exec, stream_));
        } else {
            mem_.EnqueueUpload(upload, stream_);
            mem_.EnqueueKernels(shape_, stream_);
        }
        VQM_CK(cudaEventRecord(done_, stream_));
        token_ = NextIncarnation();
        in_flight_ = true;
        return token_;
    }

    vqm_cu_ss2_config cfg_;
    ScalePlan plan_;
    BlurShape shape_;
    int device_ = 0;
    cudaStream_t own_stream_ = nullptr, stream_ = nullptr;
    cudaEvent_t done_ = nullptr, copied_ = nullptr;
    cudaGraphExec_t graph_exec_[4 * kPrepGroups * kPrepGroups] = {};
    bool reference_valid_ = false;
    uint64_t reference_handle_ = 0;
    float reference_background_ = 0.0f;
    uint64_t reference_reuses_ = 0;
    bool graphs_ = true;
    Tables tables_;
    BatchMemory mem_;
    DeviceBuffer stream_in_[2];
    // The AllocateImage pool: pinned host memory the caller writes through
    // MapImage (as into VQM's host-visible arena) and the prepare kernels
    // read in place over the bus (unified addressing maps it on the device).
    PinnedBuffer pool_;
    // The STAGED memory policy's device mirror of the pool.
    DeviceBuffer pool_device_;
    bool staged_ = false;
    std::vector<Slot> slots_;
    std::vector<InputAlloc> inputs_;
    bool in_flight_ = false;
    uint64_t token_ = 0;
};

// ---------------------------------------------------------------------------
// Batch: many pairs of any sizes, one launch per stage.
// ---------------------------------------------------------------------------

class Batch {
public:
    explicit Batch(const vqm_cu_ss2_batch_config& cfg) : cfg_(cfg) {
        if (cfg.chroma_filter > 2) throw std::invalid_argument("invalid chroma filter");
        mem_.SetBlur(cfg.blur);
        if (cfg.variant) {
            if (cfg.variant > static_cast<uint32_t>(BlurTileCount()))
                throw std::invalid_argument("cuda: no such blur variant");
            shape_ = BlurShape::Of(static_cast<int>(cfg.variant) - 1);
        } else if (cfg.tile_w || cfg.tile_h) {
            // The one-tile-per-CTA variant with that tile.
            int found = -1;
            for (int i = 0; i < BlurTileCount() && found < 0; ++i) {
                int w, h;
                BlurTileShape(i, &w, &h);
                if (w == static_cast<int>(cfg.tile_w) && h == static_cast<int>(cfg.tile_h) &&
                    BlurTileStrip(i) == 1 && !BlurTilePersistent(i))
                    found = i;
            }
            if (found < 0) throw std::invalid_argument("cuda: blur tile shape is not compiled in");
            shape_ = BlurShape::Of(found);
        }
        if (cfg.half_planes) {
            // Half planes run the one-tile-per-CTA blur of the same tile (the
            // default tile when there is none), and the tables count its
            // blocks.
            mem_.elem_bytes = 2;
            const int v = HalfPlaneVariant(shape_.variant);
            shape_ = BlurShape::Of(v < 0 ? kDefaultBlurVariant : v);
        }
        // No variant chosen: each submit picks one for its tile count.
        auto_shape_ = !cfg.variant && !cfg.tile_w && !cfg.tile_h && !cfg.half_planes;
        device_ = ResolveDevice(cfg.device);
        EnsureDevice(device_);
        VQM_CK(cudaSetDevice(device_));
        sms_ = DeviceSms(device_);
        VQM_CK(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
        stream_ = own_stream_;
        VQM_CK(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
        VQM_CK(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming));
        VQM_CK(cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming));
        VQM_CK(cudaEventCreateWithFlags(&uploaded_, cudaEventDisableTiming));
        for (auto& e : stage_ev_) VQM_CK(cudaEventCreate(&e));
    }
    ~Batch() {
        cudaSetDevice(device_);
        if (stream_) cudaStreamSynchronize(stream_);
        if (copy_stream_) cudaStreamSynchronize(copy_stream_);
        for (cudaEvent_t e : {done_, copied_, uploaded_})
            if (e) cudaEventDestroy(e);
        for (auto& e : stage_ev_)
            if (e) cudaEventDestroy(e);
        if (copy_stream_) cudaStreamDestroy(copy_stream_);
        if (own_stream_) cudaStreamDestroy(own_stream_);
    }
    void SetStream(void* s) {
        if (in_flight_) throw std::logic_error("cuda: a batch is in flight; Finish it first");
        stream_ = s ? static_cast<cudaStream_t>(s) : own_stream_;
    }

    // Device bytes the batch holds now (pyramid, tables, partials, counters
    // and its copy of host inputs), reused from submit to submit.
    size_t DeviceBytes() { return mem_.DeviceBytes() + inputs_.bytes(); }

    // Device bytes the batch will hold once these pairs are submitted: its
    // buffers grown as Submit grows them (never shrunk). Validates the pairs
    // as Submit does; allocates nothing.
    size_t DeviceBytesAfter(uint32_t n, const vqm_cu_image* o, const vqm_cu_image* d) {
        std::vector<std::pair<uint32_t, uint32_t>> sizes;
        const size_t host_bytes = ValidatePairs(n, o, d, sizes);
        Tables t = BuildTables(sizes, ShapeFor(sizes));
        BatchMemory probe;  // offsets only; the sizes come from mem_
        probe.elem_bytes = mem_.elem_bytes;
        const std::array<size_t, 5> need = probe.Needs(t);
        const std::array<DeviceBuffer*, 5> buf = mem_.Buffers();
        size_t bytes = inputs_.grown(std::max<size_t>(host_bytes, 256));
        for (int i = 0; i < 5; ++i) bytes += buf[i]->grown(need[i]);
        return bytes;
    }

    // Frees the device memory an idle batch holds; the next submit
    // allocates what it needs again.
    void Trim() {
        if (in_flight_) throw std::logic_error("cuda: a batch is in flight; Finish it first");
        VQM_CK(cudaSetDevice(device_));
        VQM_CK(cudaStreamSynchronize(stream_));
        VQM_CK(cudaStreamSynchronize(copy_stream_));
        mem_.ReleaseDevice();
        inputs_.reset();
    }

    // `wait_copies` false leaves the host-to-device copies of host images in
    // flight: their planes are then borrowed until Finish.
    uint64_t Submit(uint32_t n, const vqm_cu_image* o, const vqm_cu_image* d, float bg,
                    bool wait_copies = true) {
        if (in_flight_) throw std::logic_error("cuda: a batch is in flight; Finish it first");
        TraceRange trace("ss2 batch submit");
        std::vector<std::pair<uint32_t, uint32_t>> sizes;
        const size_t host_bytes = ValidatePairs(n, o, d, sizes);
        VQM_CK(cudaSetDevice(device_));
        const BlurShape shape = ShapeFor(sizes);
        Tables t = BuildTables(sizes, shape);
        mem_.Layout(t);
        inputs_.ensure(std::max<size_t>(host_bytes, 256));
        size_t cursor = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const vqm_cu_image* imgs[2] = {&o[i], &d[i]};
            for (int k = 0; k < 2; ++k) {
                DevSource& src = t.pairs[i].src[k];
                const vqm_cu_image& img = *imgs[k];
                BuildSourceConstants(img.format, cfg_.chroma_filter, bg, src);
                const char* name = k == 0 ? "original" : "distorted";
                if (img.memory == VQM_CU_MEMORY_HOST) {
                    uint8_t* dst = inputs_.as<uint8_t>() + cursor;
                    cursor += AlignUp(RequiredBytes(img.format, img.width, img.height), 256);
                    CopyHostImage(img, dst, stream_);
                    const void* planes[4];
                    size_t strides[4];
                    PackedPlanes(img.format, img.width, img.height, dst, planes, strides);
                    FillPlanes(src, img.format, img.width, img.height, planes, strides, name);
                } else if (img.memory == VQM_CU_MEMORY_DEVICE) {
                    FillPlanes(src, img.format, img.width, img.height, img.planes, img.strides,
                               name);
                } else {
                    throw std::invalid_argument(std::string(name) + ": invalid memory kind");
                }
            }
        }
        PrepGroups group(n);
        bool yuv420 = true;
        for (uint32_t i = 0; i < n; ++i) {
            group[i] = {static_cast<uint8_t>(PrepGroup(t.pairs[i].src[0])),
                        static_cast<uint8_t>(PrepGroup(t.pairs[i].src[1]))};
            for (int k = 0; k < 2; ++k)
                if (group[i][k] == 1 && !Yuv420Window(t.pairs[i].src[k])) yuv420 = false;
        }
        mem_.dev.yuv420 = yuv420 ? 1u : 0u;
        BuildPrepLists(t, group);
        mem_.Stage(t);
        if (host_bytes) VQM_CK(cudaEventRecord(copied_, stream_));
        // The tables and counters go up on the batch's copy stream: they
        // depend on nothing on the launch stream (this batch's previous
        // submission has finished), so they overlap whatever runs there,
        // typically another batch's kernels. The results need no copy: the
        // blur writes them into pinned host memory.
        VQM_CK(cudaMemsetAsync(mem_.pair_done.as<void>(), 0,
                               sizeof(uint32_t) * (n + t.segs.size() + 2), copy_stream_));
        mem_.EnqueueUpload(mem_.table_bytes, copy_stream_);
        VQM_CK(cudaEventRecord(uploaded_, copy_stream_));
        VQM_CK(cudaStreamWaitEvent(stream_, uploaded_, 0));
        mem_.EnqueueKernels(shape, stream_, timing_ ? stage_ev_ : nullptr);
        timed_ = timing_;
        VQM_CK(cudaEventRecord(done_, stream_));
        count_ = n;
        token_ = NextIncarnation();
        in_flight_ = true;
        if (host_bytes && wait_copies) VQM_CK(cudaEventSynchronize(copied_));
        return token_;
    }

    void SetTiming(bool on) {
        if (in_flight_) throw std::logic_error("cuda: a batch is in flight; Finish it first");
        timing_ = on;
    }

private:
    // Validates a submission; fills `sizes` and returns the device bytes its
    // host images take once copied.
    size_t ValidatePairs(uint32_t n, const vqm_cu_image* o, const vqm_cu_image* d,
                         std::vector<std::pair<uint32_t, uint32_t>>& sizes) const {
        if (n == 0) throw std::invalid_argument("cuda: empty batch");
        if (!o || !d) throw std::invalid_argument("cuda: image arrays must not be null");
        if (cfg_.max_pairs && n > cfg_.max_pairs)
            throw std::invalid_argument("cuda: batch exceeds max_pairs");
        sizes.resize(n);
        size_t host_bytes = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const std::string no = "original[" + std::to_string(i) + "]";
            const std::string nd = "distorted[" + std::to_string(i) + "]";
            if (o[i].width != d[i].width || o[i].height != d[i].height)
                throw std::invalid_argument(nd + ": image size does not match the original");
            ValidateFormat(o[i].format, o[i].width, o[i].height, no.c_str());
            ValidateFormat(d[i].format, d[i].width, d[i].height, nd.c_str());
            sizes[i] = {o[i].width, o[i].height};
            if (o[i].memory == VQM_CU_MEMORY_HOST)
                host_bytes += AlignUp(RequiredBytes(o[i].format, o[i].width, o[i].height), 256);
            if (d[i].memory == VQM_CU_MEMORY_HOST)
                host_bytes += AlignUp(RequiredBytes(d[i].format, d[i].width, d[i].height), 256);
        }
        return host_bytes;
    }
    BlurShape ShapeFor(const std::vector<std::pair<uint32_t, uint32_t>>& sizes) const {
        return auto_shape_ ? BlurShape::Of(AutoBlurVariant(DefaultTileGrids(sizes), sms_))
                           : shape_;
    }

public:
    void StageMs(float* ms) const {
        if (in_flight_) throw std::logic_error("cuda: a batch is in flight; Finish it first");
        if (!timed_) throw std::logic_error("cuda: the last batch was not timed");
        for (int i = 0; i < 3; ++i) VQM_CK(cudaEventElapsedTime(&ms[i], stage_ev_[i], stage_ev_[i + 1]));
    }

    void Finish(uint64_t token, double* norms, uint32_t* scales, double* scores) {
        if (!in_flight_ || token != token_)
            throw std::invalid_argument("cuda: no submission with that token");
        TraceRange trace("ss2 batch finish");
        VQM_CK(cudaSetDevice(device_));
        const cudaError_t e = cudaEventSynchronize(done_);
        in_flight_ = false;
        Check(e, "batch execution");
        const double* r = mem_.results_host.as<double>();
        for (uint32_t i = 0; i < count_; ++i) {
            const double* ri = r + static_cast<size_t>(i) * kResultDoubles;
            const int n = static_cast<int>(ri[kResultScales]);
            if (norms)
                for (int k = 0; k < 108; ++k) norms[i * 108 + k] = k < 18 * n ? ri[k] : 0.0;
            if (scales) scales[i] = static_cast<uint32_t>(n);
            if (scores) scores[i] = ri[kResultScore];
        }
    }

private:
    vqm_cu_ss2_batch_config cfg_;
    BlurShape shape_;
    bool auto_shape_ = false;
    int sms_ = 0;
    int device_ = 0;
    cudaStream_t own_stream_ = nullptr, stream_ = nullptr;
    cudaStream_t copy_stream_ = nullptr;  // tables and counter resets
    cudaEvent_t done_ = nullptr, copied_ = nullptr;
    cudaEvent_t uploaded_ = nullptr;
    cudaEvent_t stage_ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    bool timing_ = false, timed_ = false;
    BatchMemory mem_;
    DeviceBuffer inputs_;
    bool in_flight_ = false;
    uint32_t count_ = 0;
    uint64_t token_ = 0;
};

// ---------------------------------------------------------------------------
// C ABI plumbing: exceptions to status codes.
// ---------------------------------------------------------------------------

template <class F>
int Guard(F&& f) {
    try {
        f();
        g_last_error.clear();
        return VQM_CU_OK;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return VQM_CU_INVALID_ARGUMENT;
    } catch (const std::logic_error& e) {
        g_last_error = e.what();
        return VQM_CU_LOGIC_ERROR;
    } catch (const std::overflow_error& e) {
        g_last_error = e.what();
        return VQM_CU_OVERFLOW_ERROR;
    } catch (const std::bad_alloc&) {
        g_last_error = "out of host memory";
        return VQM_CU_RUNTIME_ERROR;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return VQM_CU_RUNTIME_ERROR;
    }
}

void NotNull(const void* p, const char* what) {
    if (!p) throw std::invalid_argument(std::string(what) + " is null");
}

// The self-checks of the kernels' shorter arithmetic routes (CheckCbrt,
// CheckDivision) on the current device, as C ABI calls.
template <class Check>
int RunRouteCheck(Check check, uint32_t first_bits, uint32_t last_bits, uint64_t* mismatches,
                  uint32_t* first_bad) {
    return Guard([&] {
        NotNull(mismatches, "mismatches");
        NotNull(first_bad, "first_bad");
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("cuda: no usable compute device");
        }
        EnsureDevice(device);
        const cudaError_t e = check(first_bits, last_bits, mismatches, first_bad);
        if (e == cudaErrorInvalidValue) throw std::invalid_argument("empty or inverted range");
        if (e != cudaSuccess) throw std::runtime_error(std::string("cuda: ") + cudaGetErrorString(e));
    });
}

}  // namespace

int ResolveDeviceOrdinal(int32_t requested) { return ResolveDevice(requested); }

// The message vqm_cu_last_error() returns on this thread, for entry points
// defined in other translation units.
void SetLastErrorMessage(const char* message) { g_last_error = message ? message : ""; }

}  // namespace vqm_b200

using vqm_b200::Guard;
using vqm_b200::NotNull;

struct vqm_cu_ss2_pipeline {
    vqm_b200::Pipeline impl;
    explicit vqm_cu_ss2_pipeline(const vqm_cu_ss2_config& c) : impl(c) {}
};
struct vqm_cu_ss2_batch {
    vqm_b200::Batch impl;
    explicit vqm_cu_ss2_batch(const vqm_cu_ss2_batch_config& c) : impl(c) {}
};

extern "C" {

const char* vqm_cu_last_error(void) { return vqm_b200::g_last_error.c_str(); }
uint32_t vqm_cu_version(void) { return (1u << 16) | 5u; }

int vqm_cu_device_count(uint32_t* count) {
    return vqm_b200::Guard([&] {
        vqm_b200::NotNull(count, "count");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        *count = static_cast<uint32_t>(n);
    });
}

int vqm_cu_device_info(uint32_t index, char* name, size_t name_bytes, uint8_t* uuid16,
                       uint32_t* type) {
    return vqm_b200::Guard([&] {
        vqm_b200::NotNull(uuid16, "uuid");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        if (index >= static_cast<uint32_t>(n))
            throw std::invalid_argument("cuda: no device " + std::to_string(index));
        cudaDeviceProp prop{};
        const cudaError_t e = cudaGetDeviceProperties(&prop, static_cast<int>(index));
        if (e != cudaSuccess) throw std::runtime_error(std::string("cuda: ") + cudaGetErrorString(e));
        if (name && name_bytes) {
            std::strncpy(name, prop.name, name_bytes - 1);
            name[name_bytes - 1] = '\0';
        }
        std::memcpy(uuid16, prop.uuid.bytes, 16);
        if (type) *type = prop.integrated ? 1u : 2u;
    });
}

int vqm_cu_set_default_device(const uint8_t* uuid16) {
    return vqm_b200::Guard([&] {
        vqm_b200::NotNull(uuid16, "uuid");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        for (int i = 0; i < n; ++i) {
            cudaDeviceProp prop{};
            const cudaError_t e = cudaGetDeviceProperties(&prop, i);
            if (e != cudaSuccess)
                throw std::runtime_error(std::string("cuda: ") + cudaGetErrorString(e));
            if (std::memcmp(prop.uuid.bytes, uuid16, 16) == 0) {
                vqm_b200::g_default_device.store(i);
                return;
            }
        }
        throw std::invalid_argument("device UUID is not available");
    });
}

int vqm_cu_required_bytes(const vqm_cu_format* format, uint32_t width, uint32_t height,
                          size_t* bytes) {
    return Guard([&] {
        NotNull(format, "format");
        NotNull(bytes, "bytes");
        *bytes = vqm_b200::RequiredBytes(*format, width, height);
    });
}

int vqm_cu_validate_format(const vqm_cu_format* format, uint32_t width, uint32_t height,
                           const char* name) {
    return Guard([&] {
        NotNull(format, "format");
        vqm_b200::ValidateFormat(*format, width, height, name ? name : "image");
    });
}

int vqm_cu_ss2_plan_scales(uint32_t width, uint32_t height, uint32_t* sizes12, uint32_t* scales) {
    return Guard([&] {
        const auto plan = vqm_b200::PlanScales(width, height);
        for (int i = 0; i < 6; ++i) {
            if (sizes12) {
                sizes12[2 * i] = i < plan.count ? plan.w[i] : 0;
                sizes12[2 * i + 1] = i < plan.count ? plan.h[i] : 0;
            }
        }
        if (scales) *scales = static_cast<uint32_t>(plan.count);
    });
}

int vqm_cu_ss2_check_cbrt(uint32_t first_bits, uint32_t last_bits, uint64_t* mismatches,
                          uint32_t* first_bad) {
    return vqm_b200::RunRouteCheck(vqm_b200::CheckCbrt, first_bits, last_bits, mismatches,
                                   first_bad);
}

int vqm_cu_ss2_check_division(uint32_t first_bits, uint32_t last_bits, uint64_t* mismatches,
                              uint32_t* first_bad) {
    return vqm_b200::RunRouteCheck(vqm_b200::CheckDivision, first_bits, last_bits, mismatches,
                                   first_bad);
}

int vqm_cu_ss2_channel_pruned(uint32_t channel, uint32_t scale, uint32_t scales, int* pruned) {
    return Guard([&] {
        NotNull(pruned, "pruned");
        if (channel >= 3 || scales == 0 || scales > 6 || scale >= scales)
            throw std::invalid_argument("channel, scale or scale count out of range");
        *pruned = vqm_b200::ChannelPruned(static_cast<int>(channel), static_cast<int>(scale),
                                          static_cast<int>(scales))
                      ? 1
                      : 0;
    });
}

int vqm_cu_ss2_blur_taps(uint32_t blur, float* taps13) {
    return Guard([&] {
        NotNull(taps13, "taps13");
        const std::array<float, vqm_b200::kTaps> taps = vqm_b200::BlurTaps(blur);
        std::copy(taps.begin(), taps.end(), taps13);
    });
}

int vqm_cu_ss2_score(const double* norms, uint32_t scales, double* score) {
    return Guard([&] {
        NotNull(score, "score");
        if (scales > 0) NotNull(norms, "norms");
        *score = vqm_b200::Score(norms, static_cast<int>(scales));
    });
}

int vqm_cu_ss2_source_constants(const vqm_cu_format* format, uint32_t chroma_filter,
                                uint32_t* words) {
    return Guard([&] {
        NotNull(format, "format");
        NotNull(words, "words44");
        if (chroma_filter > 2) throw std::invalid_argument("invalid chroma filter");
        vqm_b200::DevSource d{};
        vqm_b200::BuildSourceConstants(*format, chroma_filter, 0.5f, d);
        std::memset(words, 0, 44 * sizeof(uint32_t));
        words[4] = uint32_t(format->type) | (uint32_t(format->family) << 2) |
                   (uint32_t(format->alpha) << 4) | (uint32_t(format->subsample_w) << 6) |
                   (uint32_t(format->subsample_h) << 8) | (uint32_t(d.transfer) << 10) |
                   (chroma_filter << 15) | (uint32_t(d.mode) << 17);
        words[5] = (d.identity1 ? 1u : 0u) | (d.identity2 ? 2u : 0u);
        auto put = [&](int i, float v) { std::memcpy(&words[i], &v, 4); };
        for (int i = 0; i < 3; ++i) {
            put(6 + i, d.scale[i]);
            put(9 + i, d.offset[i]);
        }
        for (int i = 0; i < 9; ++i) {
            put(12 + i, d.m1[i]);
            put(21 + i, d.m2[i]);
        }
        put(30, d.kr);
        put(31, d.kg);
        put(32, d.kb);
        put(33, d.to_linear);
        put(34, d.shift_x);
        put(35, d.shift_y);
        for (int i = 0; i < 4; ++i) put(36 + i, d.cl[i]);
    });
}

int vqm_cu_ss2_create(const vqm_cu_ss2_config* config, vqm_cu_ss2_pipeline** pipeline) {
    return Guard([&] {
        NotNull(config, "config");
        NotNull(pipeline, "pipeline");
        *pipeline = nullptr;
        *pipeline = new vqm_cu_ss2_pipeline(*config);
    });
}

int vqm_cu_ss2_destroy(vqm_cu_ss2_pipeline* pipeline) {
    return Guard([&] { delete pipeline; });
}

int vqm_cu_ss2_set_stream(vqm_cu_ss2_pipeline* p, void* stream) {
    return Guard([&] {
        NotNull(p, "pipeline");
        p->impl.SetStream(stream);
    });
}

int vqm_cu_ss2_get_stream(vqm_cu_ss2_pipeline* p, void** stream) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(stream, "stream");
        *stream = p->impl.GetStream();
    });
}

int vqm_cu_ss2_set_graphs(vqm_cu_ss2_pipeline* p, int enabled) {
    return Guard([&] {
        NotNull(p, "pipeline");
        p->impl.SetGraphs(enabled != 0);
    });
}

int vqm_cu_ss2_reference_reuses(vqm_cu_ss2_pipeline* p, uint64_t* count) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(count, "count");
        *count = p->impl.ReferenceReuses();
    });
}

int vqm_cu_ss2_in_flight(const vqm_cu_ss2_pipeline* p, uint32_t* in_flight) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(in_flight, "in_flight");
        *in_flight = p->impl.InFlight() ? 1u : 0u;
    });
}

int vqm_cu_ss2_submit(vqm_cu_ss2_pipeline* p, const vqm_cu_image* o, const vqm_cu_image* d,
                      float background, uint64_t* token) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(token, "token");
        *token = p->impl.SubmitImages(o, d, background);
    });
}

int vqm_cu_ss2_submit_resident(vqm_cu_ss2_pipeline* p, uint64_t o, uint64_t d, float background,
                               uint64_t* token) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(token, "token");
        *token = p->impl.SubmitResident(o, d, background);
    });
}

int vqm_cu_ss2_submit_resident_image(vqm_cu_ss2_pipeline* p, uint64_t o, const vqm_cu_image* d,
                                     float background, uint64_t* token) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(token, "token");
        *token = p->impl.SubmitResidentImage(o, d, background);
    });
}

int vqm_cu_ss2_submit_buffers(vqm_cu_ss2_pipeline* p, uint64_t o, uint64_t d, float background,
                              uint64_t* token) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(token, "token");
        *token = p->impl.SubmitBuffers(o, d, background);
    });
}

int vqm_cu_ss2_submit_sync(vqm_cu_ss2_pipeline* p, const vqm_cu_image* o, const vqm_cu_image* d,
                           void* const* waits, uint32_t nwaits, void* const* signals,
                           uint32_t nsignals, float background, uint64_t* token) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(token, "token");
        if (nwaits) NotNull(waits, "wait_events");
        if (nsignals) NotNull(signals, "signal_events");
        for (uint32_t i = 0; i < nwaits; ++i)
            if (!waits[i]) throw std::invalid_argument("cuda: invalid event list");
        for (uint32_t i = 0; i < nsignals; ++i)
            if (!signals[i]) throw std::invalid_argument("cuda: invalid event list");
        *token = p->impl.SubmitImages(o, d, background, waits, nwaits, signals, nsignals);
    });
}

int vqm_cu_ss2_finish(vqm_cu_ss2_pipeline* p, uint64_t token, double* norms108, uint32_t* scales) {
    return Guard([&] {
        NotNull(p, "pipeline");
        p->impl.Finish(token, norms108, scales);
    });
}

int vqm_cu_ss2_compute(vqm_cu_ss2_pipeline* p, const vqm_cu_image* o, const vqm_cu_image* d,
                       float background, double* norms108, uint32_t* scales, double* score) {
    return Guard([&] {
        NotNull(p, "pipeline");
        const uint64_t token = p->impl.SubmitImages(o, d, background);
        double local[108];
        double* out = norms108 ? norms108 : local;
        uint32_t n = 0;
        p->impl.Finish(token, out, &n);
        if (scales) *scales = n;
        if (score) *score = vqm_b200::Score(out, static_cast<int>(n));
    });
}

int vqm_cu_ss2_upload(vqm_cu_ss2_pipeline* p, const vqm_cu_image* image, uint64_t* handle) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(handle, "handle");
        *handle = p->impl.Upload(image);
    });
}

int vqm_cu_ss2_release(vqm_cu_ss2_pipeline* p, uint64_t handle) {
    return Guard([&] {
        NotNull(p, "pipeline");
        p->impl.Release(handle);
    });
}

int vqm_cu_ss2_allocate_image(vqm_cu_ss2_pipeline* p, const vqm_cu_format* format,
                              uint64_t* handle, size_t* bytes) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(format, "format");
        NotNull(handle, "handle");
        size_t b = 0;
        *handle = p->impl.AllocateImage(*format, &b);
        if (bytes) *bytes = b;
    });
}

int vqm_cu_ss2_map_image(vqm_cu_ss2_pipeline* p, uint64_t handle, void** device_ptr) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(device_ptr, "device_ptr");
        *device_ptr = p->impl.MapImage(handle);
    });
}

int vqm_cu_ss2_release_image(vqm_cu_ss2_pipeline* p, uint64_t handle) {
    return Guard([&] {
        NotNull(p, "pipeline");
        p->impl.ReleaseImage(handle);
    });
}

int vqm_cu_ss2_debug_plane(vqm_cu_ss2_pipeline* p, uint32_t image, uint32_t level,
                           uint32_t channel, float* out) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(out, "out");
        p->impl.DebugPlane(image, level, channel, out);
    });
}

int vqm_cu_ss2_memory_usage(vqm_cu_ss2_pipeline* p, vqm_cu_memory_usage* usage) {
    return Guard([&] {
        NotNull(p, "pipeline");
        NotNull(usage, "usage");
        p->impl.Usage(usage);
    });
}

int vqm_cu_ss2_batch_create(const vqm_cu_ss2_batch_config* config, vqm_cu_ss2_batch** batch) {
    return Guard([&] {
        NotNull(config, "config");
        NotNull(batch, "batch");
        *batch = nullptr;
        *batch = new vqm_cu_ss2_batch(*config);
    });
}

int vqm_cu_ss2_batch_destroy(vqm_cu_ss2_batch* batch) {
    return Guard([&] { delete batch; });
}

int vqm_cu_ss2_batch_set_stream(vqm_cu_ss2_batch* b, void* stream) {
    return Guard([&] {
        NotNull(b, "batch");
        b->impl.SetStream(stream);
    });
}

int vqm_cu_ss2_batch_submit(vqm_cu_ss2_batch* b, uint32_t n, const vqm_cu_image* o,
                            const vqm_cu_image* d, float background, uint64_t* token) {
    return Guard([&] {
        NotNull(b, "batch");
        NotNull(token, "token");
        if (n) {
            NotNull(o, "originals");
            NotNull(d, "distorteds");
        }
        *token = b->impl.Submit(n, o, d, background);
    });
}

int vqm_cu_ss2_batch_submit_borrowed(vqm_cu_ss2_batch* b, uint32_t n, const vqm_cu_image* o,
                                     const vqm_cu_image* d, float background, uint64_t* token) {
    return Guard([&] {
        NotNull(b, "batch");
        NotNull(token, "token");
        if (n) {
            NotNull(o, "originals");
            NotNull(d, "distorteds");
        }
        *token = b->impl.Submit(n, o, d, background, false);
    });
}

int vqm_cu_ss2_batch_finish(vqm_cu_ss2_batch* b, uint64_t token, double* norms, uint32_t* scales,
                            double* scores) {
    return Guard([&] {
        NotNull(b, "batch");
        b->impl.Finish(token, norms, scales, scores);
    });
}

int vqm_cu_ss2_decode_path(const vqm_cu_format* format, uint32_t chroma_filter,
                           uint32_t* path) {
    return Guard([&] {
        NotNull(format, "format");
        NotNull(path, "path");
        if (chroma_filter > 2) throw std::invalid_argument("invalid chroma filter");
        vqm_b200::ValidateFormat(*format, 4, 4, "format");
        vqm_b200::DevSource d{};
        vqm_b200::BuildSourceConstants(*format, chroma_filter, 0.5f, d);
        *path = d.lut ? (d.in_range ? VQM_CU_DECODE_TABLE_IN_RANGE : VQM_CU_DECODE_TABLE)
                      : (d.yuv_fast ? VQM_CU_DECODE_YUV : VQM_CU_DECODE_GENERIC);
    });
}

int vqm_cu_ss2_blur_variants(uint32_t* count, uint32_t* shapes) {
    return Guard([&] {
        NotNull(count, "count");
        *count = static_cast<uint32_t>(vqm_b200::BlurTileCount());
        if (shapes)
            for (int i = 0; i < vqm_b200::BlurTileCount(); ++i) {
                int w, h;
                vqm_b200::BlurTileShape(i, &w, &h);
                uint32_t* v = shapes + VQM_CU_SS2_VARIANT_WORDS * i;
                v[0] = static_cast<uint32_t>(w);
                v[1] = static_cast<uint32_t>(h);
                v[2] = static_cast<uint32_t>(vqm_b200::BlurTileThreads(i));
                v[3] = static_cast<uint32_t>(vqm_b200::BlurTileStrip(i));
                v[4] = vqm_b200::BlurTilePersistent(i) ? 1u : 0u;
            }
    });
}

int vqm_cu_ss2_auto_blur_variant(const uint32_t* sizes, uint32_t n, uint32_t sms,
                                 uint32_t* variant) {
    return Guard([&] {
        NotNull(variant, "variant");
        if (n == 0 || sms == 0) throw std::invalid_argument("no pairs or no SMs");
        NotNull(sizes, "sizes");
        std::vector<std::pair<uint32_t, uint32_t>> wh(n);
        for (uint32_t i = 0; i < n; ++i) {
            wh[i] = {sizes[2 * i], sizes[2 * i + 1]};
            if (wh[i].first < vqm_b200::kMinDimension || wh[i].second < vqm_b200::kMinDimension)
                throw std::invalid_argument("pair smaller than 8x8");
        }
        *variant = static_cast<uint32_t>(
            vqm_b200::AutoBlurVariant(vqm_b200::DefaultTileGrids(wh), static_cast<int>(sms)));
    });
}

int vqm_cu_ss2_batch_set_timing(vqm_cu_ss2_batch* b, int enabled) {
    return Guard([&] {
        NotNull(b, "batch");
        b->impl.SetTiming(enabled != 0);
    });
}

int vqm_cu_ss2_batch_stage_ms(vqm_cu_ss2_batch* b, float* ms3) {
    return Guard([&] {
        NotNull(b, "batch");
        NotNull(ms3, "stage_ms3");
        b->impl.StageMs(ms3);
    });
}

int vqm_cu_ss2_batch_device_bytes(vqm_cu_ss2_batch* b, uint64_t* held) {
    return Guard([&] {
        NotNull(b, "batch");
        NotNull(held, "held");
        *held = b->impl.DeviceBytes();
    });
}

int vqm_cu_ss2_batch_device_bytes_after(vqm_cu_ss2_batch* b, uint32_t n, const vqm_cu_image* o,
                                        const vqm_cu_image* d, uint64_t* bytes) {
    return Guard([&] {
        NotNull(b, "batch");
        NotNull(bytes, "bytes");
        *bytes = b->impl.DeviceBytesAfter(n, o, d);
    });
}

int vqm_cu_ss2_batch_trim(vqm_cu_ss2_batch* b) {
    return Guard([&] {
        NotNull(b, "batch");
        b->impl.Trim();
    });
}

int vqm_cu_ss2_batch_compute(vqm_cu_ss2_batch* b, uint32_t n, const vqm_cu_image* o,
                             const vqm_cu_image* d, float background, double* norms,
                             uint32_t* scales, double* scores) {
    return Guard([&] {
        NotNull(b, "batch");
        const uint64_t token = b->impl.Submit(n, o, d, background);
        b->impl.Finish(token, norms, scales, scores);
    });
}

}  // extern "C"
