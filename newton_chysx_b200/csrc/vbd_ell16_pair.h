// Launchers of the ELL16 persistent kernel whose threads solve two vertices each with paired FP32 instructions
// (compiled in vbd_ell16_pair.cu).
#pragma once
#include "vbd_ell.cuh"

namespace vbd {

template <bool SMEM>
void launch_persistent_ell16_pair(int occ, const StepCtx<float>& c, const PersistentPlan& p, const Ell16View& e,
                                  int grid, int block, size_t smem, cudaStream_t st);

template <bool SMEM>
const void* persistent_ell16_pair_fn(int occ);

}  // namespace vbd
