// The ELL16 persistent kernel for models with damped hinges (k_persistent_ell16<..., HD = true>): the bending
// term adds the reference's Rayleigh damping (particle_vbd_kernels.py:1057-1190), reading each damped hinge's
// kd from a side array. In its own translation unit so that it compiles beside vbd_b200.cu.
#include "vbd_ell16_damped.h"

namespace vbd {

template <typename R, int MODE, bool SMEM>
void launch_persistent_ell16_damped(int occ, const StepCtx<R>& c, const PersistentPlan& p, const Ell16View& e,
                                    int grid, int block, size_t smem, cudaStream_t st) {
  switch (occ) {
    case 2: k_persistent_ell16<R, MODE, SMEM, 2, false, true><<<grid, block, smem, st>>>(c, p, e); break;
    case 3: k_persistent_ell16<R, MODE, SMEM, 3, false, true><<<grid, block, smem, st>>>(c, p, e); break;
    case 4: k_persistent_ell16<R, MODE, SMEM, 4, false, true><<<grid, block, smem, st>>>(c, p, e); break;
    default: k_persistent_ell16<R, MODE, SMEM, 0, false, true><<<grid, block, smem, st>>>(c, p, e); break;
  }
}

template <typename R, int MODE, bool SMEM>
const void* persistent_ell16_damped_fn(int occ) {
  switch (occ) {
    case 2: return (const void*)k_persistent_ell16<R, MODE, SMEM, 2, false, true>;
    case 3: return (const void*)k_persistent_ell16<R, MODE, SMEM, 3, false, true>;
    case 4: return (const void*)k_persistent_ell16<R, MODE, SMEM, 4, false, true>;
    default: return (const void*)k_persistent_ell16<R, MODE, SMEM, 0, false, true>;
  }
}

#define VBD_ELL16_DAMPED(R, MODE, SMEM)                                                                      \
  template void launch_persistent_ell16_damped<R, MODE, SMEM>(int, const StepCtx<R>&, const PersistentPlan&, \
                                                              const Ell16View&, int, int, size_t, cudaStream_t); \
  template const void* persistent_ell16_damped_fn<R, MODE, SMEM>(int);

VBD_ELL16_DAMPED(float, MODE_FP32, false)
VBD_ELL16_DAMPED(float, MODE_FP32, true)
VBD_ELL16_DAMPED(float, MODE_MIXED, false)
VBD_ELL16_DAMPED(float, MODE_MIXED, true)
VBD_ELL16_DAMPED(double, MODE_FP64, false)

}  // namespace vbd
