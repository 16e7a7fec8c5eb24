// Launchers of the ELL16 persistent kernel for models with damped hinges (compiled in vbd_ell16_damped.cu).
#pragma once
#include "vbd_ell.cuh"

namespace vbd {

template <typename R, int MODE, bool SMEM>
void launch_persistent_ell16_damped(int occ, const StepCtx<R>& c, const PersistentPlan& p, const Ell16View& e,
                                    int grid, int block, size_t smem, cudaStream_t st);

template <typename R, int MODE, bool SMEM>
const void* persistent_ell16_damped_fn(int occ);

}  // namespace vbd
