// The ELL16 persistent kernel with two vertices per thread in paired FP32 arithmetic
// (k_persistent_ell16<float, MODE_FP32, SMEM, OCC, PAIR = true>), in its own translation unit so that it
// compiles beside vbd_b200.cu.
#include "vbd_ell16_pair.h"

namespace vbd {

template <bool SMEM>
void launch_persistent_ell16_pair(int occ, const StepCtx<float>& c, const PersistentPlan& p, const Ell16View& e,
                                  int grid, int block, size_t smem, cudaStream_t st) {
  switch (occ) {
    case 2: k_persistent_ell16<float, MODE_FP32, SMEM, 2, true><<<grid, block, smem, st>>>(c, p, e); break;
    case 3: k_persistent_ell16<float, MODE_FP32, SMEM, 3, true><<<grid, block, smem, st>>>(c, p, e); break;
    case 4: k_persistent_ell16<float, MODE_FP32, SMEM, 4, true><<<grid, block, smem, st>>>(c, p, e); break;
    default: k_persistent_ell16<float, MODE_FP32, SMEM, 0, true><<<grid, block, smem, st>>>(c, p, e); break;
  }
}

template <bool SMEM>
const void* persistent_ell16_pair_fn(int occ) {
  switch (occ) {
    case 2: return (const void*)k_persistent_ell16<float, MODE_FP32, SMEM, 2, true>;
    case 3: return (const void*)k_persistent_ell16<float, MODE_FP32, SMEM, 3, true>;
    case 4: return (const void*)k_persistent_ell16<float, MODE_FP32, SMEM, 4, true>;
    default: return (const void*)k_persistent_ell16<float, MODE_FP32, SMEM, 0, true>;
  }
}

template void launch_persistent_ell16_pair<false>(int, const StepCtx<float>&, const PersistentPlan&, const Ell16View&,
                                                  int, int, size_t, cudaStream_t);
template void launch_persistent_ell16_pair<true>(int, const StepCtx<float>&, const PersistentPlan&, const Ell16View&,
                                                 int, int, size_t, cudaStream_t);
template const void* persistent_ell16_pair_fn<false>(int);
template const void* persistent_ell16_pair_fn<true>(int);

}  // namespace vbd
