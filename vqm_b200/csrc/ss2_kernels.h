// Launchers of the SSIMULACRA 2.1 kernels (ss2_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>
#include <vector>

#include "ss2_device.cuh"

namespace vqm_b200 {

// Gaussian taps (13 floats) and score weights (18 x 6 doubles) into the
// current device's constant banks; once per device.
cudaError_t SetConstants(const double* weights108);

cudaError_t LaunchPrepare(const DevBatch& batch, cudaStream_t stream);
// `variant` indexes the blur kernels compiled in (BlurTileShape gives each
// one's output tile); the batch's segments must have been tiled with it.
// The blur also finishes every pair: its last CTA per segment sums the
// segment, its last per pair writes the pair's norms and score, so the
// batch's pair_done and seg_done counters must be zero when it starts (the
// kernel leaves them zero).
cudaError_t LaunchBlur(const DevBatch& batch, int variant, cudaStream_t stream);
// Load every kernel of each stage on the current device (and set the blur
// kernels' shared-memory limits), so that no first launch pays for it.
cudaError_t PreloadPrepare();
cudaError_t PreloadBlur();
// Checks the prepare kernels' cube root against ss2dm::cbrt, bit for bit, on
// every float whose bit pattern lies in [first_bits, last_bits], on the
// current device; synchronous.
cudaError_t CheckCbrt(uint32_t first_bits, uint32_t last_bits, uint64_t* mismatches,
                      uint32_t* first_bad);
// The blur maps' division against ss2dm::divf for every divisor whose bit
// pattern lies in [first_bits, last_bits], at sixteen quotient values each.
cudaError_t CheckDivision(uint32_t first_bits, uint32_t last_bits, uint64_t* mismatches,
                          uint32_t* first_bad);

// The blur variants compiled into the library and their output tiles.
int BlurTileCount();
void BlurTileShape(int index, int* w, int* h);
int BlurTileThreads(int index);
// Tiles one CTA computes down a column (1: one tile per CTA).
int BlurTileStrip(int index);
bool BlurTilePersistent(int index);
// Blocks of variant `index` for a segment of tiles_x x tiles_y tiles: the
// prefix sums of these are a batch's blur_start.
uint32_t BlurBlocks(int index, uint32_t tiles_x, uint32_t tiles_y);
// The variant used when a caller does not choose one, for a launch over
// segments with these tile grids of the default tile (columns, rows, in
// launch order) on a device with `sms` SMs: the strip length with the least
// estimated time (ss2_blur.cu). A strip regroups the compensated partial
// sums, so the choice moves a result by rounding only (~1e-7 relative).
int AutoBlurVariant(const std::vector<std::pair<uint32_t, uint32_t>>& grids, int sms);
// The one-tile-per-CTA variant with variant's tile shape (the variant
// itself when it is one), which half planes run; -1 when there is none.
int HalfPlaneVariant(int variant);
// The variant used when a caller does not choose one.
constexpr int kDefaultBlurVariant = 0;

}  // namespace vqm_b200
