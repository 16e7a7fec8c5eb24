// The persistent schedule with particle self-contact: one CTA takes a whole instance (world) from the work queue
// and runs the reference's self-contact sequence on it (solver_vbd.py:1731-1766, 2151-2337) with CTA barriers
// instead of kernel boundaries: phase 0 is the forward step and its truncation, phase 1 the iterations, each color
// followed by the division-plane truncation of the instance's own pairs (apply_planar_truncation_parallel_by_
// collision, particle_vbd_kernels.py:2744-2874; apply_truncation_ts, :2877-2897). The detections between the
// phases stay grid-wide launches over all instances, keeping only pairs within an instance. In its own
// translation unit so that it compiles beside vbd_b200.cu.
#include "vbd_sc_persistent.h"

namespace vbd {

namespace {

// Truncation of one instance: the division planes of its pairs, then every vertex moved to q_cd + t d.
template <typename R>
__device__ __forceinline__ void truncate_instance(const StepCtx<R>& c, const ScPersistentPlan& s, int vs, int ve,
                                                  int es, int ee) {
  const int p0 = __ldg(s.vt_off + vs), p1 = __ldg(s.vt_off + ve);
  const int q0 = __ldg(s.ee_off + es), q1 = __ldg(s.ee_off + ee);
  const int nv = p1 - p0, n = nv + (q1 - q0);
  R* ts = static_cast<R*>(s.ts);
  const R eps = R(s.eps), gamma = R(s.gamma);
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    trunc_pair<R>(i < nv, i < nv ? s.vt_pairs[p0 + i] : s.ee_pairs[q0 + i - nv], c.pos_cd, c.disp, eps, gamma, ts);
  __syncthreads();
  const R max_d = R(s.max_d);
  for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) trunc_vertex<R>(i, ts, max_d, c.pos_cd, c.disp, c.pos);
  __syncthreads();
}

template <typename R, int L, int MODE>
__global__ void k_persistent_sc(StepCtx<R> c, PersistentPlan p, ScPersistentPlan s) {
  __shared__ int s_item;
  const GlobalPos<R> pos{c.pos};
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(p.queue, 1);
    __syncthreads();
    const int q = s_item;
    if (q >= p.W) return;
    const int w = __ldg(p.inst_order + q);
    const int vs = __ldg(p.inst_vstart + w), ve = __ldg(p.inst_vstart + w + 1);
    const int es = __ldg(s.inst_estart + w), ee = __ldg(s.inst_estart + w + 1);
    if (s.phase == 0) {
      for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) forward_particle(c, pos, i);
      __syncthreads();
      truncate_instance<R>(c, s, vs, ve, es, ee);
      continue;
    }
    const int cb = __ldg(p.inst_cptr + w), ce = __ldg(p.inst_cptr + w + 1);
    const int per_round = blockDim.x / L;
    const int grp_local = threadIdx.x / L, sub = threadIdx.x % L;
    for (int it = s.it0; it < s.it1; ++it) {
      for (int col = cb; col + 1 < ce; ++col) {
        const int a = __ldg(p.color_ranges + col), b = __ldg(p.color_ranges + col + 1);
        for (int base = a; base < b; base += per_round) {
          const int g = base + grp_local;
          const bool valid = g < b;
          const int v = valid ? __ldg(p.color_verts + g) : 0;
          solve_group<R, L, MODE, GlobalPos<R>, true, false>(c, pos, v, valid, sub, it);
        }
        __syncthreads();
        truncate_instance<R>(c, s, vs, ve, es, ee);
      }
    }
    if (s.finalize)
      for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) finalize_particle(c, pos, i);
  }
}

}  // namespace

template <typename R, int MODE>
void launch_persistent_sc(int L, const StepCtx<R>& c, const PersistentPlan& p, const ScPersistentPlan& s, int grid,
                          int block, cudaStream_t st) {
  switch (L) {
    case 1: k_persistent_sc<R, 1, MODE><<<grid, block, 0, st>>>(c, p, s); break;
    case 2: k_persistent_sc<R, 2, MODE><<<grid, block, 0, st>>>(c, p, s); break;
    case 4: k_persistent_sc<R, 4, MODE><<<grid, block, 0, st>>>(c, p, s); break;
    case 8: k_persistent_sc<R, 8, MODE><<<grid, block, 0, st>>>(c, p, s); break;
    case 16: k_persistent_sc<R, 16, MODE><<<grid, block, 0, st>>>(c, p, s); break;
    default: k_persistent_sc<R, 32, MODE><<<grid, block, 0, st>>>(c, p, s); break;
  }
}

template <typename R, int MODE>
const void* persistent_sc_fn(int L) {
  switch (L) {
    case 1: return (const void*)k_persistent_sc<R, 1, MODE>;
    case 2: return (const void*)k_persistent_sc<R, 2, MODE>;
    case 4: return (const void*)k_persistent_sc<R, 4, MODE>;
    case 8: return (const void*)k_persistent_sc<R, 8, MODE>;
    case 16: return (const void*)k_persistent_sc<R, 16, MODE>;
    default: return (const void*)k_persistent_sc<R, 32, MODE>;
  }
}

#define VBD_SC_PERSISTENT(R, MODE)                                                                              \
  template void launch_persistent_sc<R, MODE>(int, const StepCtx<R>&, const PersistentPlan&,                  \
                                              const ScPersistentPlan&, int, int, cudaStream_t);               \
  template const void* persistent_sc_fn<R, MODE>(int);

VBD_SC_PERSISTENT(float, MODE_FP32)
VBD_SC_PERSISTENT(float, MODE_MIXED)
VBD_SC_PERSISTENT(double, MODE_FP64)

}  // namespace vbd
