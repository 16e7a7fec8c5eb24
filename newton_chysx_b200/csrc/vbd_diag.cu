// Diagnostics: the device math routines of the step evaluated on caller arrays, so that tests can hold them to
// the CUDA library functions they stand in for.
#include "vbd_b200.h"
#include "vbd_math.cuh"

namespace {

__global__ void k_eval_atan2(int n, const float* __restrict__ y, const float* __restrict__ x, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = vbd::vatan2(y[i], x[i]);
}

}  // namespace

extern "C" int vbd_eval_atan2(int32_t n, const float* y, const float* x, float* out, void* stream) {
  if (n < 0 || (n > 0 && (!y || !x || !out))) return VBD_ERR_INVALID_ARGUMENT;
  if (n == 0) return VBD_OK;
  k_eval_atan2<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, y, x, out);
  return cudaGetLastError() == cudaSuccess ? VBD_OK : VBD_ERR_CUDA;
}
