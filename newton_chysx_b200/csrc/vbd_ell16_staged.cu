// The ELL16 persistent kernel with stencil records staged through shared memory by cp.async
// (k_persistent_ell16<..., STAGES = kEll16Stages>), in its own translation unit so that it compiles beside
// vbd_b200.cu.
#include "vbd_ell16_staged.h"

namespace vbd {

template <typename R, int MODE, bool SMEM>
void launch_persistent_ell16_staged(int occ, const StepCtx<R>& c, const PersistentPlan& p, const Ell16View& e, int grid,
                                    int block, size_t smem, cudaStream_t st) {
  constexpr int S = kEll16Stages;
  switch (occ) {
    case 2: k_persistent_ell16<R, MODE, SMEM, 2, S><<<grid, block, smem, st>>>(c, p, e); break;
    case 3: k_persistent_ell16<R, MODE, SMEM, 3, S><<<grid, block, smem, st>>>(c, p, e); break;
    case 4: k_persistent_ell16<R, MODE, SMEM, 4, S><<<grid, block, smem, st>>>(c, p, e); break;
    default: k_persistent_ell16<R, MODE, SMEM, 0, S><<<grid, block, smem, st>>>(c, p, e); break;
  }
}

template <typename R, int MODE, bool SMEM>
const void* persistent_ell16_staged_fn(int occ) {
  constexpr int S = kEll16Stages;
  switch (occ) {
    case 2: return (const void*)k_persistent_ell16<R, MODE, SMEM, 2, S>;
    case 3: return (const void*)k_persistent_ell16<R, MODE, SMEM, 3, S>;
    case 4: return (const void*)k_persistent_ell16<R, MODE, SMEM, 4, S>;
    default: return (const void*)k_persistent_ell16<R, MODE, SMEM, 0, S>;
  }
}

#define VBD_STAGED(MODE, SMEM)                                                                                      \
  template void launch_persistent_ell16_staged<float, MODE, SMEM>(int, const StepCtx<float>&, const PersistentPlan&, \
                                                                  const Ell16View&, int, int, size_t, cudaStream_t); \
  template const void* persistent_ell16_staged_fn<float, MODE, SMEM>(int);
VBD_STAGED(MODE_FP32, false)
VBD_STAGED(MODE_FP32, true)
VBD_STAGED(MODE_MIXED, false)
VBD_STAGED(MODE_MIXED, true)
#undef VBD_STAGED

}  // namespace vbd
