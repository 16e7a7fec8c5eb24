// Launchers of the ELL16 persistent kernel with staged record fetch (compiled in vbd_ell16_staged.cu).
#pragma once
#include "vbd_ell.cuh"

namespace vbd {

// Record stages of the staged variant (cp.async ring depth per thread).
constexpr int kEll16Stages = 4;

// Dynamic shared memory of the staged kernel for `block` threads, on top of `pos_bytes` of instance positions.
inline size_t ell16_staged_smem(size_t pos_bytes, int block) {
  return ((pos_bytes + 15) & ~size_t(15)) + 16 + size_t(2) * kEll16Stages * block * 16;
}

template <typename R, int MODE, bool SMEM>
void launch_persistent_ell16_staged(int occ, const StepCtx<R>& c, const PersistentPlan& p, const Ell16View& e, int grid,
                                    int block, size_t smem, cudaStream_t st);

template <typename R, int MODE, bool SMEM>
const void* persistent_ell16_staged_fn(int occ);

}  // namespace vbd
