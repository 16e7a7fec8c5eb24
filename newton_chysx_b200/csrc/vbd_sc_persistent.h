// Persistent schedule with particle self-contact (compiled in vbd_sc_persistent.cu).
#pragma once
#include "vbd_collide.cuh"
#include "vbd_kernels.cuh"

namespace vbd {

// One instance's self-contact data for the persistent kernel: its pairs are the VT pairs of its vertices and the
// EE pairs of its edges, found by a detection that keeps pairs within an instance (ScBuffers::world).
struct ScPersistentPlan {
  const int* inst_estart;  // [W+1] the edges of instance w are [inst_estart[w], inst_estart[w+1])
  const int* vt_off;       // [V+1] VT pairs of vertex v: vt_pairs[vt_off[v] .. vt_off[v+1])
  const int* ee_off;       // [E+1] EE pairs of edge e: ee_pairs[ee_off[e] .. ee_off[e+1])
  const int4* vt_pairs;    // per pair its four vertices (ScBuffers::vt_pairs, ee_pairs)
  const int4* ee_pairs;
  void* ts;                // [V] R: per-vertex step fractions of the truncation, 1 between passes
  double eps, gamma, max_d;
  int phase;               // 0: forward step and truncation; 1: iterations [it0, it1)
  int it0, it1;
  int finalize;            // phase 1: velocity update and write-back after the last iteration
};

template <typename R, int MODE>
void launch_persistent_sc(int L, const StepCtx<R>& c, const PersistentPlan& p, const ScPersistentPlan& s, int grid,
                          int block, cudaStream_t st);

template <typename R, int MODE>
const void* persistent_sc_fn(int L);

}  // namespace vbd
