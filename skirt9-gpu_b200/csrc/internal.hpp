// Declarations shared between the C-ABI translation unit and the kernel translation units.
#pragma once

#include <cuda_runtime.h>
#include "lifecycle.cuh"

namespace skg {

// life-cycle launchers, one per precision (separate translation units so the FP64 one can be
// compiled without FMA contraction)
cudaError_t launchLifecycleFP64(int gridKind, const LCParams& p, int blocks, int threads, cudaStream_t s);
int lifecycleBlocksPerSMFP64(int gridKind, int threads);
cudaError_t launchLifecycleFP32(int gridKind, const LCParams& p, int blocks, int threads, cudaStream_t s);
int lifecycleBlocksPerSMFP32(int gridKind, int threads);

// path-segment and optical-depth kernels (reference generators, FP64 exact or FP32)
cudaError_t launchTracePaths(int precision, const GridDev& g, int n, const double* rays, int maxSeg, int* count,
                             int* m, double* ds, int* err, cudaStream_t s);
cudaError_t launchOpticalDepths(int precision, const GridDev& g, const double* dens, double section, int n,
                                const double* rays, double* tau, int* err, cudaStream_t s);

}  // namespace skg
