// Scoring one pair without allocating any memory.
//
// The pipeline and batch objects allocate their device memory (pyramid
// planes, tile partials, tables) with cudaMalloc when they are created or
// grow. Some callers cannot let a library do that: applications that hand all
// device memory to their own pool or allocator and forbid other allocations,
// real-time loops where cudaMalloc/cudaFree would synchronize the device and
// stall unrelated streams, and plug-in hosts that give a plug-in a stream and
// buffers but no allocation rights. vqm_cu_ss2_compute_noalloc serves them:
// it runs the same prepare and blur kernels (the finalize is the blur's
// epilogue) on the caller's stream,
// with every piece of scratch (tables, counters, tile partials, segment sums
// and the XYB pyramid) placed in one file-scope __device__ array of fixed size
// that the CUDA module reserves when the library is loaded. The caller passes
// the device images to score and a device buffer for the result.
//
// Limits and rules:
//   * kScratchBytes (32 MiB) bounds the scratch one pair needs: its FP32
//     pyramid (rows padded to a multiple of 32 columns, so the need depends
//     on the width, not on the pixel count alone), tile partials and tables.
//     1920x1080, 1080x1920 and 2048x1200 fit; 1200x2048 (same area, narrow
//     rows padded more) and 2560x1440 do not. Pairs that need more are
//     rejected with VQM_CU_INVALID_ARGUMENT, naming the bytes they need.
//   * Image planes and the result must be device (or managed) memory of the
//     current device; anything else is rejected before a kernel runs.
//   * Every GPU that loads the library holds the 32 MiB until the process
//     exits.
//   * All calls share the one array and it keeps the last call's contents:
//     two calls whose work overlaps on the GPU (different streams, or a second
//     call before the first finished) race on it and corrupt each other.
//     Serialize them on one stream or wait between them.
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) and uploads the blur taps and score weights;
//     make that first call before any stream capture begins.

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
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

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxSegments = kMaxLevels * kChannels;

// The scratch itself. Host code must never dereference or pass this symbol:
// on the host it names a stand-in object, not device memory. Its device
// address comes from cudaGetSymbolAddress (ScratchAddress below).
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Everything the kernels read from tables, for one pair, passed to the
// staging kernel by value so no host buffer or copy is involved.
struct PairTables {
    DevPair pair;
    DevSegment seg[kMaxSegments];
    DevPrepItem item[2];
    uint32_t prep_start[2 + kPrepGroups];
    uint32_t blur_start[kMaxSegments + 1];
};
static_assert(sizeof(PairTables) < 30000, "kernel parameter space");

// `counters`: the pair's and every segment's completion counter, which the
// blur's epilogue counts up, and the blur's tile-queue words; they must
// start at zero whatever the last call left.
__global__ void StageTablesKernel(const PairTables tables, PairTables* dst, uint32_t* counters) {
    const uint32_t* from = reinterpret_cast<const uint32_t*>(&tables);
    uint32_t* to = reinterpret_cast<uint32_t*>(dst);
    for (uint32_t i = threadIdx.x; i < sizeof(PairTables) / 4; i += blockDim.x) to[i] = from[i];
    if (threadIdx.x < 3 + kMaxSegments) counters[threadIdx.x] = 0u;
}

struct DeviceState {
    bool ready = false;
    unsigned char* scratch = nullptr;
};

// Per-device set-up, once, with that device current.
unsigned char* ScratchAddress(int device) {
    static std::mutex mu;
    static std::vector<DeviceState> states;
    std::lock_guard<std::mutex> lock(mu);
    if (states.size() <= static_cast<size_t>(device)) states.resize(device + 1);
    DeviceState& st = states[device];
    if (st.ready) return st.scratch;
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error(std::string("cuda: cudaGetSymbolAddress of the scratch array: ") +
                                 cudaGetErrorString(e));
    }
    const cudaError_t c = SetConstants(ScoreWeights());
    if (c != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error(std::string("cuda: constant upload: ") + cudaGetErrorString(c));
    }
    st.scratch = static_cast<unsigned char*>(ptr);
    st.ready = true;
    return st.scratch;
}

size_t Align(size_t v, size_t a) { return (v + a - 1) / a * a; }

// A pointer the kernels may read or write: device or managed memory that
// belongs to `device`. Host memory, even pinned and mapped, is refused, so a
// caller's mistake is an error status and not a fault on the device.
void RequireDeviceMemory(const void* p, int device, const std::string& what) {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw std::invalid_argument(what + ": not a CUDA pointer");
    }
    const bool device_memory = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
    if (!device_memory || (a.type == cudaMemoryTypeDevice && a.device != device))
        throw std::invalid_argument(what + ": must be device memory of the current device");
}

void SourcePlanes(DevSource& src, const vqm_cu_image& img, const char* name) {
    if (img.memory != VQM_CU_MEMORY_DEVICE)
        throw std::invalid_argument(std::string(name) +
                                    ": the no-allocation entry point reads device images only");
    const auto layout = PlaneLayout(img.format, img.width, img.height);
    for (int p = 0; p < 4; ++p) {
        src.plane[p] = nullptr;
        src.row_bytes[p] = 0;
        src.plane_w[p] = static_cast<uint32_t>(layout[p].width);
        src.plane_h[p] = static_cast<uint32_t>(layout[p].height);
        if (!layout[p].present()) continue;
        if (img.planes[p] == nullptr)
            throw std::invalid_argument(std::string(name) + ": plane " + std::to_string(p) + " is null");
        const size_t row = layout[p].width * layout[p].sample_bytes;
        const size_t stride = img.strides[p] ? img.strides[p] : row;
        if (stride < row || stride % layout[p].sample_bytes != 0 || stride > 0xffffffffull ||
            reinterpret_cast<uintptr_t>(img.planes[p]) % layout[p].sample_bytes != 0)
            throw std::invalid_argument(std::string(name) + ": invalid plane stride or alignment");
        src.plane[p] = static_cast<const uint8_t*>(img.planes[p]);
        src.row_bytes[p] = static_cast<uint32_t>(stride);
    }
    src.width = img.width;
    src.height = img.height;
}

void Run(const vqm_cu_image* o, const vqm_cu_image* d, float background, uint32_t chroma_filter,
         void* stream_ptr, double* result) {
    if (!o || !d) throw std::invalid_argument("image is null");
    if (!result) throw std::invalid_argument("result is null");
    if (reinterpret_cast<uintptr_t>(result) % 8 != 0)
        throw std::invalid_argument("result must be 8-byte aligned device memory");
    if (chroma_filter > 2) throw std::invalid_argument("invalid chroma filter");
    if (d->width != o->width || d->height != o->height)
        throw std::invalid_argument("distorted: image size does not match the original");
    ValidateFormat(o->format, o->width, o->height, "original");
    ValidateFormat(d->format, d->width, d->height, "distorted");
    const ScalePlan plan = PlanScales(o->width, o->height);
    int tile_w = 0, tile_h = 0;  // the output tile of the blur kernel used
    BlurTileShape(kDefaultBlurVariant, &tile_w, &tile_h);
    const uint32_t tw = static_cast<uint32_t>(tile_w), th = static_cast<uint32_t>(tile_h);

    PairTables t;
    std::memset(static_cast<void*>(&t), 0, sizeof(t));
    DevPair& P = t.pair;
    P.levels = static_cast<uint32_t>(plan.count);
    size_t floats = 0;
    uint32_t nseg = 0, tiles = 0, blocks = 0;
    t.blur_start[0] = 0;
    for (int l = 0; l < plan.count; ++l) {
        P.w[l] = plan.w[l];
        P.h[l] = plan.h[l];
        P.pitch[l] = RowPairPitch(plan.w[l]);
        P.mask[l] = plan.mask[l];
        for (int c = 0; c < 3; ++c) {
            if (!(plan.mask[l] & (1u << c))) continue;
            P.plane_off[l][c] = floats;
            floats += PlaneFloats(plan.w[l], plan.h[l]);
            DevSegment& s = t.seg[nseg];
            s.pair = 0;
            s.level = static_cast<uint32_t>(l);
            s.channel = static_cast<uint32_t>(c);
            s.tiles_x = (plan.w[l] + tw - 1) / tw;
            const uint32_t ty = (plan.h[l] + th - 1) / th;
            s.tiles = s.tiles_x * ty;
            s.partial_first = tiles;
            s.partials = BlurBlocks(kDefaultBlurVariant, s.tiles_x, ty);
            tiles += s.partials;
            blocks += s.partials;
            ++nseg;
            t.blur_start[nseg] = blocks;
        }
    }
    P.image_stride = floats;
    P.prep_tiles_x = PrepTiles(o->width);
    P.prep_tiles_y = PrepTiles(o->height);
    P.seg_first = 0;
    P.seg_count = nseg;

    // Scratch layout: [tables | completion counters | segment sums | blur
    // partials | pyramid], each 256-byte aligned.
    const size_t off_tables = 0;
    const size_t off_done = Align(off_tables + sizeof(PairTables), 256);
    const size_t off_sums = Align(off_done + sizeof(uint32_t) * (3 + kMaxSegments), 256);
    const size_t off_partials = Align(off_sums + sizeof(double) * 6 * kMaxSegments, 256);
    const size_t off_pyramid = Align(off_partials + sizeof(double) * 6 * tiles, 256);
    const size_t need = off_pyramid + sizeof(float) * 2 * floats;
    if (need > kScratchBytes)
        throw std::invalid_argument(
            "cuda: a " + std::to_string(o->width) + "x" + std::to_string(o->height) +
            " pair needs " + std::to_string(need) +
            " bytes of scratch; the no-allocation entry point has " +
            std::to_string(kScratchBytes) +
            " (32 MiB: e.g. 1920x1080 or 2048x1200 fit; the need grows with the row width)");

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("cuda: no usable compute device");
    }
    BuildSourceConstants(o->format, chroma_filter, background, P.src[0]);
    BuildSourceConstants(d->format, chroma_filter, background, P.src[1]);
    SourcePlanes(P.src[0], *o, "original");
    SourcePlanes(P.src[1], *d, "distorted");
    for (int k = 0; k < 2; ++k)
        for (int p = 0; p < 4; ++p)
            if (P.src[k].plane[p])
                RequireDeviceMemory(P.src[k].plane[p], device,
                                    std::string(k ? "distorted" : "original") + " plane " +
                                        std::to_string(p));
    RequireDeviceMemory(result, device, "result");
    unsigned char* base = ScratchAddress(device);
    P.pyramid = reinterpret_cast<float*>(base + off_pyramid);
    P.result = result;

    // Prepare lists: the two images by prepare group (table, YUV, generic),
    // each group's prefix offsets after the previous group's.
    const uint32_t per_image = P.prep_tiles_x * P.prep_tiles_y;
    const int group[2] = {PrepGroup(P.src[0]), PrepGroup(P.src[1])};
    uint32_t n[kPrepGroups] = {};
    for (uint32_t k = 0; k < 2; ++k) ++n[group[k]];
    uint32_t item = 0, entry = 0;
    for (int g = 0; g < kPrepGroups; ++g) {
        t.prep_start[entry] = 0;
        for (uint32_t k = 0; k < 2; ++k) {
            if (group[k] != g) continue;
            t.item[item++] = DevPrepItem{0, k};
            t.prep_start[entry + 1] = t.prep_start[entry] + per_image;
            ++entry;
        }
        ++entry;
    }

    PairTables* dev_tables = reinterpret_cast<PairTables*>(base + off_tables);
    uint32_t* pair_done = reinterpret_cast<uint32_t*>(base + off_done);
    DevBatch b{};
    b.pairs = 1;
    b.segments = nseg;
    for (int g = 0; g < kPrepGroups; ++g) {
        b.prep_items[g] = n[g];
        b.prep_blocks[g] = n[g] * per_image;
    }
    b.blur_blocks = blocks;
    b.pair = &dev_tables->pair;
    b.seg = dev_tables->seg;
    b.prep_item = dev_tables->item;
    b.prep_start = dev_tables->prep_start;
    b.blur_start = dev_tables->blur_start;
    b.partials = reinterpret_cast<double*>(base + off_partials);
    b.seg_sums = reinterpret_cast<double*>(base + off_sums);
    b.pair_done = pair_done;
    b.seg_done = pair_done + 1;
    b.blur_queue = pair_done + 1 + kMaxSegments;
    b.status = nullptr;
    const std::array<float, kTaps> taps = GaussianTaps();
    for (int i = 0; i < kTaps; ++i) b.taps2[i] = make_float2(taps[i], taps[i]);

    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    StageTablesKernel<<<1, 256, 0, stream>>>(t, dev_tables, pair_done);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = LaunchPrepare(b, stream);
    if (e == cudaSuccess) e = LaunchBlur(b, kDefaultBlurVariant, stream);
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("cuda: launch: ") + cudaGetErrorString(e));
}

}  // namespace
}  // namespace vqm_b200

extern "C" int vqm_cu_ss2_compute_noalloc(const vqm_cu_image* original,
                                          const vqm_cu_image* distorted, float background,
                                          uint32_t chroma_filter, void* stream,
                                          double* result_device) {
    try {
        vqm_b200::Run(original, distorted, background, chroma_filter, stream, result_device);
        vqm_b200::SetLastErrorMessage("");
        return VQM_CU_OK;
    } catch (const std::invalid_argument& e) {
        vqm_b200::SetLastErrorMessage(e.what());
        return VQM_CU_INVALID_ARGUMENT;
    } catch (const std::logic_error& e) {
        vqm_b200::SetLastErrorMessage(e.what());
        return VQM_CU_LOGIC_ERROR;
    } catch (const std::exception& e) {
        vqm_b200::SetLastErrorMessage(e.what());
        return VQM_CU_RUNTIME_ERROR;
    }
}
