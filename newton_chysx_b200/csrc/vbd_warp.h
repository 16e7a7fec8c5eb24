// Launchers of the warp-per-instance persistent kernel (compiled in vbd_warp.cu).
#pragma once
#include "vbd_kernels.cuh"

namespace vbd {

// L in {1, 2, 4, 8}; slice = floats of shared memory per warp (SMEM only).
template <typename R, int MODE, bool SMEM>
void launch_persistent_warp(bool soft, int L, const StepCtx<R>& c, const PersistentPlan& p, int slice, int grid,
                            int block, size_t smem, cudaStream_t st);

template <typename R, int MODE, bool SMEM>
const void* persistent_warp_fn(bool soft, int L);

}  // namespace vbd
