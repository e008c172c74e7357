// Launchers of the SSIMULACRA 2.1 kernels (ss2_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "ss2_device.cuh"

namespace vqm_b200 {

// Gaussian taps (13 floats) and score weights (18 x 6 doubles) into the
// current device's constant banks; once per device.
cudaError_t SetConstants(const float* taps13, const double* weights108);

cudaError_t LaunchPrepare(const DevBatch& batch, cudaStream_t stream);
cudaError_t LaunchBlur(const DevBatch& batch, int tile_w, int tile_h,
                       cudaStream_t stream);
cudaError_t LaunchFinalize(const DevBatch& batch, cudaStream_t stream);

// Blur tile shapes compiled into the library, as (w, h) pairs.
int BlurTileCount();
void BlurTileShape(int index, int* w, int* h);

}  // namespace vqm_b200
