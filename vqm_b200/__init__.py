"""vqm_b200: SSIMULACRA 2.1 image-quality scoring on NVIDIA B200 (sm_100a).

A drop-in for VQM's SSIMULACRA 2 path (GreatValueCreamSoda/vqm): hand-written
CUDA kernels behind a C ABI (include/vqm_cu_ss2.h), with the reference's
C++ API restored in include/vqm_cuda.hpp and mirrored in Python here.

    from vqm_b200 import ss2
    pipe = ss2.Ssimulacra2Pipeline(1920, 1080)
    print(pipe.compute(original, distorted).score())

Importing ``vqm_b200.ss2`` loads the compiled extension and fails if it is
missing; nothing falls back to the CPU.
"""

__all__ = ["ss2", "build"]
