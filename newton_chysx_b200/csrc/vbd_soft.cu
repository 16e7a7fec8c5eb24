// Launchers of the sweep kernels for models with springs or tetrahedra (solve_group<..., SOFT = true>).
//
// They live in their own translation unit so that nvcc compiles them beside vbd_b200.cu; the cloth-only
// kernels keep their register budget because the extra element classes are compiled only here.
#include "vbd_soft.h"

namespace vbd {

template <typename R, int MODE, int L, bool SC>
static void launch_color_soft_l(const StepCtx<R>& c, const int* verts, int n, int it, int block, cudaStream_t st) {
  const long threads = long(n) * L;
  const int grid = int((threads + block - 1) / block);
  if (grid > 0) k_color<R, L, MODE, SC, true><<<grid, block, 0, st>>>(c, verts, n, it);
}

template <typename R, int MODE, bool SC>
static void launch_color_soft_sc(int L, const StepCtx<R>& c, const int* verts, int n, int it, int block,
                                 cudaStream_t st) {
  switch (L) {
    case 1: launch_color_soft_l<R, MODE, 1, SC>(c, verts, n, it, block, st); break;
    case 2: launch_color_soft_l<R, MODE, 2, SC>(c, verts, n, it, block, st); break;
    case 4: launch_color_soft_l<R, MODE, 4, SC>(c, verts, n, it, block, st); break;
    case 8: launch_color_soft_l<R, MODE, 8, SC>(c, verts, n, it, block, st); break;
    case 16: launch_color_soft_l<R, MODE, 16, SC>(c, verts, n, it, block, st); break;
    default: launch_color_soft_l<R, MODE, 32, SC>(c, verts, n, it, block, st); break;
  }
}

template <typename R, int MODE>
void launch_color_soft(bool sc, int L, const StepCtx<R>& c, const int* verts, int n, int it, int block,
                       cudaStream_t st) {
  if (c.n_same_springs && n > 0) k_spring_prepass<R><<<(n + 127) / 128, 128, 0, st>>>(c, verts, n);
  if (sc)
    launch_color_soft_sc<R, MODE, true>(L, c, verts, n, it, block, st);
  else
    launch_color_soft_sc<R, MODE, false>(L, c, verts, n, it, block, st);
}

template <typename R, int MODE, bool SMEM>
const void* persistent_soft_fn(int L) {
  switch (L) {
    case 1: return (const void*)k_persistent<R, 1, MODE, SMEM, true>;
    case 2: return (const void*)k_persistent<R, 2, MODE, SMEM, true>;
    case 4: return (const void*)k_persistent<R, 4, MODE, SMEM, true>;
    case 8: return (const void*)k_persistent<R, 8, MODE, SMEM, true>;
    case 16: return (const void*)k_persistent<R, 16, MODE, SMEM, true>;
    default: return (const void*)k_persistent<R, 32, MODE, SMEM, true>;
  }
}

template <typename R, int MODE, bool SMEM>
void launch_persistent_soft(int L, const StepCtx<R>& c, const PersistentPlan& p, int grid, int block, size_t smem,
                            cudaStream_t st) {
  switch (L) {
    case 1: k_persistent<R, 1, MODE, SMEM, true><<<grid, block, smem, st>>>(c, p); break;
    case 2: k_persistent<R, 2, MODE, SMEM, true><<<grid, block, smem, st>>>(c, p); break;
    case 4: k_persistent<R, 4, MODE, SMEM, true><<<grid, block, smem, st>>>(c, p); break;
    case 8: k_persistent<R, 8, MODE, SMEM, true><<<grid, block, smem, st>>>(c, p); break;
    case 16: k_persistent<R, 16, MODE, SMEM, true><<<grid, block, smem, st>>>(c, p); break;
    default: k_persistent<R, 32, MODE, SMEM, true><<<grid, block, smem, st>>>(c, p); break;
  }
}

template void launch_color_soft<float, MODE_FP32>(bool, int, const StepCtx<float>&, const int*, int, int, int,
                                                  cudaStream_t);
template void launch_color_soft<float, MODE_MIXED>(bool, int, const StepCtx<float>&, const int*, int, int, int,
                                                   cudaStream_t);
template void launch_color_soft<double, MODE_FP64>(bool, int, const StepCtx<double>&, const int*, int, int, int,
                                                   cudaStream_t);
template const void* persistent_soft_fn<float, MODE_FP32, true>(int);
template const void* persistent_soft_fn<float, MODE_FP32, false>(int);
template const void* persistent_soft_fn<float, MODE_MIXED, true>(int);
template const void* persistent_soft_fn<float, MODE_MIXED, false>(int);
template const void* persistent_soft_fn<double, MODE_FP64, false>(int);
template void launch_persistent_soft<float, MODE_FP32, true>(int, const StepCtx<float>&, const PersistentPlan&, int,
                                                             int, size_t, cudaStream_t);
template void launch_persistent_soft<float, MODE_FP32, false>(int, const StepCtx<float>&, const PersistentPlan&, int,
                                                              int, size_t, cudaStream_t);
template void launch_persistent_soft<float, MODE_MIXED, true>(int, const StepCtx<float>&, const PersistentPlan&, int,
                                                              int, size_t, cudaStream_t);
template void launch_persistent_soft<float, MODE_MIXED, false>(int, const StepCtx<float>&, const PersistentPlan&, int,
                                                               int, size_t, cudaStream_t);
template void launch_persistent_soft<double, MODE_FP64, false>(int, const StepCtx<double>&, const PersistentPlan&, int,
                                                               int, size_t, cudaStream_t);

}  // namespace vbd
