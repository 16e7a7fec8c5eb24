// Launchers for models with springs or tetrahedra (compiled in vbd_soft.cu).
#pragma once
#include "vbd_kernels.cuh"

namespace vbd {

// One color of the per-color sweep: the same-color spring pre-pass (when the model has such springs) and
// the solve, with (sc = true) or without self-contact.
template <typename R, int MODE>
void launch_color_soft(bool sc, int L, const StepCtx<R>& c, const int* verts, int n, int it, int block,
                       cudaStream_t st);

template <typename R, int MODE, bool SMEM>
const void* persistent_soft_fn(int L);

template <typename R, int MODE, bool SMEM>
void launch_persistent_soft(int L, const StepCtx<R>& c, const PersistentPlan& p, int grid, int block, size_t smem,
                            cudaStream_t st);

}  // namespace vbd
