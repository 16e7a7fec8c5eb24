// The warp-per-instance persistent kernel (k_persistent_warp), in its own translation unit so that it compiles
// beside vbd_b200.cu.
#include "vbd_warp.h"

namespace vbd {

template <typename R, int MODE, bool SMEM, bool SOFT>
static const void* warp_fn(int L) {
  switch (L) {
    case 1: return (const void*)k_persistent_warp<R, 1, MODE, SMEM, SOFT>;
    case 2: return (const void*)k_persistent_warp<R, 2, MODE, SMEM, SOFT>;
    case 4: return (const void*)k_persistent_warp<R, 4, MODE, SMEM, SOFT>;
    default: return (const void*)k_persistent_warp<R, 8, MODE, SMEM, SOFT>;
  }
}

template <typename R, int MODE, bool SMEM>
const void* persistent_warp_fn(bool soft, int L) {
  return soft ? warp_fn<R, MODE, SMEM, true>(L) : warp_fn<R, MODE, SMEM, false>(L);
}

template <typename R, int MODE, bool SMEM, bool SOFT>
static void launch_l(int L, const StepCtx<R>& c, const PersistentPlan& p, int slice, int grid, int block, size_t smem,
                     cudaStream_t st) {
  switch (L) {
    case 1: k_persistent_warp<R, 1, MODE, SMEM, SOFT><<<grid, block, smem, st>>>(c, p, slice); break;
    case 2: k_persistent_warp<R, 2, MODE, SMEM, SOFT><<<grid, block, smem, st>>>(c, p, slice); break;
    case 4: k_persistent_warp<R, 4, MODE, SMEM, SOFT><<<grid, block, smem, st>>>(c, p, slice); break;
    default: k_persistent_warp<R, 8, MODE, SMEM, SOFT><<<grid, block, smem, st>>>(c, p, slice); break;
  }
}

template <typename R, int MODE, bool SMEM>
void launch_persistent_warp(bool soft, int L, const StepCtx<R>& c, const PersistentPlan& p, int slice, int grid,
                            int block, size_t smem, cudaStream_t st) {
  if (soft)
    launch_l<R, MODE, SMEM, true>(L, c, p, slice, grid, block, smem, st);
  else
    launch_l<R, MODE, SMEM, false>(L, c, p, slice, grid, block, smem, st);
}

#define VBD_WARP(R, MODE, SMEM)                                                                                    \
  template void launch_persistent_warp<R, MODE, SMEM>(bool, int, const StepCtx<R>&, const PersistentPlan&, int, int, \
                                                      int, size_t, cudaStream_t);                                  \
  template const void* persistent_warp_fn<R, MODE, SMEM>(bool, int);
VBD_WARP(float, MODE_FP32, true)
VBD_WARP(float, MODE_FP32, false)
VBD_WARP(float, MODE_MIXED, true)
VBD_WARP(float, MODE_MIXED, false)
VBD_WARP(double, MODE_FP64, false)
#undef VBD_WARP

}  // namespace vbd
