// Host side of libvbd_b200.so: the C ABI declared in include/vbd_b200.h.
//
// Replaces the particle part of SolverVBD (newton/_src/solvers/vbd/solver_vbd.py): the constructor's
// adjacency build and scratch allocation (:442-541, :1177-1337), step() (:1575-1622) and the
// collision pipeline's particle-shape contact generation for planes and spheres
// (geometry/kernels.py:1001-1140). See vbd_kernels.cuh for the device side.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <queue>
#include <type_traits>
#include <vector>

#include "vbd_b200.h"
#include "vbd_adjoint.cuh"
#include "vbd_contactgen.cuh"
#include "vbd_collide.cuh"
#include "vbd_ell.cuh"
#include "vbd_ring.cuh"
#include "vbd_soft.h"
#include "vbd_ell16_damped.h"
#include "vbd_ell16_pair.h"
#include "vbd_sc_persistent.h"
#include "vbd_shapes.cuh"
#include "vbd_warp.h"

using namespace vbd;

namespace {

#define CK(x)                                   \
  do {                                          \
    cudaError_t e_ = (x);                       \
    if (e_ != cudaSuccess) return VBD_ERR_CUDA; \
  } while (0)

template <typename T>
int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? VBD_ERR_OUT_OF_MEMORY : VBD_ERR_CUDA;
  }
  return VBD_OK;
}

// ------------------------------------------------------------------------------ packing kernels
__global__ void k_pack_tris(int T, const int* __restrict__ idx, const float* __restrict__ pose,
                            const float* __restrict__ mat, const float* __restrict__ area, int4* o_idx, float4* o_pose,
                            float4* o_mat) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  o_idx[t] = make_int4(idx[3 * t], idx[3 * t + 1], idx[3 * t + 2], 0);
  o_pose[t] = make_float4(pose[4 * t], pose[4 * t + 1], pose[4 * t + 2], pose[4 * t + 3]);
  o_mat[t] = make_float4(mat[5 * t], mat[5 * t + 1], mat[5 * t + 2], area[t]);
}

__global__ void k_pack_edges(int E, const int* __restrict__ idx, const float* __restrict__ ra,
                             const float* __restrict__ rl, const float* __restrict__ bp, int4* o_idx, float4* o_prop) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  o_idx[e] = make_int4(idx[4 * e], idx[4 * e + 1], idx[4 * e + 2], idx[4 * e + 3]);
  o_prop[e] = make_float4(ra[e], rl[e], bp[2 * e], bp[2 * e + 1]);
}

__global__ void k_pack_springs(int N, const int* __restrict__ idx, const float* __restrict__ rest,
                               const float* __restrict__ ke, const float* __restrict__ kd, int2* o_idx, float4* o_prop) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  o_idx[i] = make_int2(idx[2 * i], idx[2 * i + 1]);
  o_prop[i] = make_float4(rest[i], ke[i], kd[i], 0.f);
}

__global__ void k_pack_tets(int N, const int* __restrict__ idx, const float* __restrict__ pose,
                            const float* __restrict__ mat, int4* o_idx, float4* o_pose) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  o_idx[t] = make_int4(idx[4 * t], idx[4 * t + 1], idx[4 * t + 2], idx[4 * t + 3]);
  const float* d = pose + 9 * size_t(t);
  const float* m = mat + 3 * size_t(t);
  o_pose[3 * t] = make_float4(d[0], d[1], d[2], m[0]);
  o_pose[3 * t + 1] = make_float4(d[3], d[4], d[5], m[1]);
  o_pose[3 * t + 2] = make_float4(d[6], d[7], d[8], m[2]);
}

// ------------------------------------------------------------------------------ soft contacts
constexpr int kMaxContactShapes = 16;
struct ShapeTable {
  int type[kMaxContactShapes];
  float4 pos_radius[kMaxContactShapes];
  float4 normal[kMaxContactShapes];  // plane normal (unit)
};

__global__ void k_soft_contacts(int n, const float* __restrict__ q, const float* __restrict__ radius,
                                const int* __restrict__ flags, int S, const ShapeTable shapes, float margin, int cmax,
                                int* count, int* particle, int* shape, float* body_pos, float* body_vel,
                                float* normal) {
  const long tid = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= long(n) * S) return;
  const int i = int(tid / S), s = int(tid % S);
  if (!(flags[i] & 1)) return;
  const float4 sf = shapes.pos_radius[s];  // pos.xyz, radius
  const float xl[3] = {q[3 * i] - sf.x, q[3 * i + 1] - sf.y, q[3 * i + 2] - sf.z};
  float d, nn[3];
  if (shapes.type[s] == 0) {
    const float4 pn = shapes.normal[s];
    d = xl[0] * pn.x + xl[1] * pn.y + xl[2] * pn.z;
    nn[0] = pn.x, nn[1] = pn.y, nn[2] = pn.z;
  } else {
    const float L = sqrtf(xl[0] * xl[0] + xl[1] * xl[1] + xl[2] * xl[2]);
    d = L - sf.w;
    if (L > 1.0e-8f) {
      nn[0] = xl[0] / L, nn[1] = xl[1] / L, nn[2] = xl[2] / L;
    } else {
      nn[0] = 0.f, nn[1] = 0.f, nn[2] = 1.f;
    }
  }
  if (d < margin + radius[i]) {
    const int k = atomicAdd(count, 1);
    if (k < cmax) {
      particle[k] = i;
      shape[k] = s;
      for (int j = 0; j < 3; ++j) {
        body_pos[3 * k + j] = (j == 0 ? sf.x : j == 1 ? sf.y : sf.z) + xl[j] - nn[j] * d;
        body_vel[3 * k + j] = 0.f;
        normal[3 * k + j] = nn[j];
      }
    }
  }
}

// The shapes of one vbd_soft_contacts_table call, passed by value as a kernel parameter.
static_assert(kMaxContactShapes == kParamTableShapes, "one parameter-table size");

}  // namespace

namespace {
void sc_release(ScBuffers& b) {
  void* ps[] = {b.bcount, b.bstart, b.ekey, b.eprim, b.blo, b.bhi, b.stats, b.vt_tri, b.vt_count, b.vt_min,
                b.ee_edge, b.ee_count, b.ee_min, b.flags, b.tmp, b.vt_off, b.vt_pairs, b.ee_off, b.ee_pairs,
                b.ent_cnt, b.ent_off, b.ent, b.vt_foff, b.vt_f, b.ee_foff, b.ee_f, b.scan_tmp};
  for (void* p : ps)
    if (p) cudaFree(p);
  b = ScBuffers();
}
}  // namespace

struct VbdSolver {
  VbdModelDesc md;
  VbdSolverParams prm;
  int V = 0, T = 0, E = 0, S = 0;
  int precision = VBD_PRECISION_FP32;
  int schedule = VBD_SCHEDULE_PER_COLOR;
  int L = 1;
  int block = 256;
  int grid_persistent = 0;
  size_t smem_bytes = 0;  // > 0: persistent kernel keeps instance positions in shared memory
  int max_inst_v = 0;
  int occ = 0;  // ELL persistent kernel: compiled occupancy target (CTAs of 256 per SM), 0 = none
  bool pair = false;  // ELL16 persistent kernel, FP32: two vertices per thread in paired FP32 arithmetic
  bool warp_inst = false;  // persistent CSR kernel: one warp per instance (k_persistent_warp)
  int slice = 0;           // its shared-memory floats per warp (positions), 0 = positions in global memory
  int K = 1;
  // packed model
  int4* tri_idx = nullptr;
  float4* tri_pose = nullptr;
  float4* tri_mat = nullptr;
  int4* edge_idx = nullptr;
  float4* edge_prop = nullptr;
  int *face_off = nullptr, *face_adj = nullptr, *edge_off = nullptr, *edge_adj = nullptr;
  // springs and tetrahedra
  int NS = 0, NT = 0;
  bool soft = false;
  int n_same_springs = 0;
  int2* spr_idx = nullptr;
  float4* spr_prop = nullptr;
  int *spr_off = nullptr, *spr_adj = nullptr, *sspr_off = nullptr, *sspr_adj = nullptr;
  void* spr_acc = nullptr;
  int4* tet_idx = nullptr;
  float4* tet_pose = nullptr;
  int *tet_off = nullptr, *tet_adj = nullptr;
  // colors
  std::vector<int> color_offsets;
  // persistent plan
  int W = 1;
  int *inst_order = nullptr, *inst_vstart = nullptr, *inst_cptr = nullptr, *color_ranges = nullptr,
      *color_verts = nullptr, *queue = nullptr;
  // scratch
  void *pos = nullptr, *qprev = nullptr, *inertia = nullptr;
  int *slot_cnt = nullptr, *slots = nullptr;
  float *c_k = nullptr, *c_ke = nullptr, *c_kd = nullptr, *c_mu = nullptr;
  int c_cap = 0;
  int* err = nullptr;
  double* residual = nullptr;
  // stencil (ELL) layout
  int layout = VBD_LAYOUT_CSR;
  std::vector<int> ranges_host;     // per range: first index into range_verts_host (+ end)
  std::vector<int> range_verts_host;  // processing order of the ELL records
  int *range_nf = nullptr, *range_ne = nullptr;
  long long *range_fbase = nullptr, *range_ebase = nullptr;
  int2* face_nb = nullptr;
  float4* face_dm = nullptr;
  float2* face_mat = nullptr;
  float* face_kd = nullptr;
  int4* hinge_idx = nullptr;
  float2* hinge_prop = nullptr;
  float* hinge_kd = nullptr;
  uint4 *ell16_faceA = nullptr, *ell16_faceB = nullptr, *ell16_hinge = nullptr;
  // one-ring layout (vbd_ring.cuh)
  int* ring_nslot = nullptr;
  long long *ring_base = nullptr, *ring_vbase = nullptr;
  uint4 *ring_A = nullptr, *ring_B = nullptr;
  float4* ring_H = nullptr;
  unsigned* ring_hdr = nullptr;
  float2* ring_kd = nullptr;
  std::vector<int> ell_nf, ell_ne;
  std::vector<long long> ell_fbase, ell_ebase;
  long long ell_faces = 0, ell_hinges = 0;
  bool ell_face_damping = false, ell_hinge_damping = false;
  std::vector<int> inst_start_of_vertex;  // first particle of each particle's instance
  // adjoint work buffers (allocated by the first vbd_adjoint_step)
  void* adj_work = nullptr;
  size_t adj_work_bytes = 0;
  // host copies of the topology (for re-packing the ELL records)
  std::vector<int> h_tri, h_edges, h_foff, h_fadj, h_eoff, h_eadj;
  // particle self-contact (vbd_set_self_contact)
  bool sc_on = false;
  ScBuffers sc;
  double sc_radius = 0, sc_margin = 0, sc_relax = 0.85, sc_ee_eps = 1e-5, sc_rest_excl = 0;
  int sc_interval = 0;
  const float* sc_rest_q = nullptr;
  void *sc_pos_cd = nullptr, *sc_disp = nullptr, *sc_ts = nullptr;
  // self-contact on the persistent schedule: per-instance edge ranges and the instance key of every vertex
  int *sc_estart = nullptr, *sc_world = nullptr;
  int grid_sc = 0;

  ~VbdSolver() {
    void* ps[] = {tri_idx, tri_pose, tri_mat, edge_idx, edge_prop, face_off, face_adj, edge_off, edge_adj,
                  inst_order, inst_vstart, inst_cptr, color_ranges, color_verts, queue, pos, qprev, inertia,
                  slot_cnt, slots, c_k, c_ke, c_kd, c_mu, err, residual, range_nf, range_ne, range_fbase,
                  range_ebase, face_nb, face_dm, face_mat, face_kd, hinge_idx, hinge_prop, hinge_kd, adj_work,
                  ell16_faceA, ell16_faceB, ell16_hinge, sc_pos_cd, sc_disp, sc_ts, ring_nslot, ring_base,
                  ring_vbase, ring_A, ring_B, ring_H, ring_hdr, ring_kd, spr_idx, spr_prop, spr_off, spr_adj, sspr_off,
                  sspr_adj, spr_acc, tet_idx, tet_pose, tet_off, tet_adj, sc_estart, sc_world};
    for (void* p : ps)
      if (p) cudaFree(p);
    sc_release(sc);
  }
};

namespace {

inline unsigned __float_as_uint_host(float f) {
  unsigned u;
  std::memcpy(&u, &f, 4);
  return u;
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <typename T>
int upload_into(T** d, const std::vector<T>& h) {
  dfree(*d);
  int rc = dalloc(d, h.size());
  if (rc) return rc;
  if (!h.empty() && cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return VBD_ERR_CUDA;
  return VBD_OK;
}

template <typename T>
int download(std::vector<T>& h, const T* d, size_t n) {
  h.resize(n);
  if (n && cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) return VBD_ERR_CUDA;
  return VBD_OK;
}

// The stencil records carry mu and lambda pre-multiplied by the triangle's area, so the kernels cannot apply
// the reference's floor of 1e-6 on |lambda + mu| (particle_vbd_kernels.py:919-921) to the material values; it
// is applied here instead: a model with an active triangle (mu > 0 or lambda > 0) whose |lambda + mu| is
// below the floor uses the CSR layout.
bool needs_lnh_floor(const std::vector<float>& mat, int T) {
  for (int t = 0; t < T; ++t) {
    const float mu = mat[5 * t], lm = mat[5 * t + 1];
    if ((mu > 0.f || lm > 0.f) && !(std::fabs(lm + mu) >= 1.0e-6f)) return true;
  }
  return false;
}

// Builds the stencil records (vbd_ell.cuh) for the ranges in h->ranges_host / h->range_verts_host from
// the caller's model arrays. Runs on the host at creation and on refresh.
int build_ell(VbdSolver* h) {
  const VbdModelDesc& m = h->md;
  std::vector<float> pose, mat, area, ra, rl, bp;
  int rc;
  if ((rc = download(pose, m.tri_poses_dev, size_t(4) * h->T)) || (rc = download(mat, m.tri_materials_dev, size_t(5) * h->T)) ||
      (rc = download(area, m.tri_areas_dev, size_t(h->T))) || (rc = download(ra, m.edge_rest_angle_dev, size_t(h->E))) ||
      (rc = download(rl, m.edge_rest_length_dev, size_t(h->E))) ||
      (rc = download(bp, m.edge_bending_properties_dev, size_t(2) * h->E)))
    return rc;
  if (needs_lnh_floor(mat, h->T)) return VBD_ERR_UNSUPPORTED;
  const int R = int(h->ranges_host.size()) - 1;
  h->ell_nf.assign(R, 0);
  h->ell_ne.assign(R, 0);
  h->ell_fbase.assign(R, 0);
  h->ell_ebase.assign(R, 0);
  long long nfaces = 0, nhinges = 0;
  for (int r = 0; r < R; ++r) {
    int nf = 0, ne = 0;
    for (int k = h->ranges_host[r]; k < h->ranges_host[r + 1]; ++k) {
      const int v = h->range_verts_host[k];
      nf = std::max(nf, h->h_foff[v + 1] - h->h_foff[v]);
      ne = std::max(ne, h->h_eoff[v + 1] - h->h_eoff[v]);
    }
    const long long n = h->ranges_host[r + 1] - h->ranges_host[r];
    h->ell_nf[r] = nf;
    h->ell_ne[r] = ne;
    h->ell_fbase[r] = nfaces;
    h->ell_ebase[r] = nhinges;
    nfaces += n * nf;
    nhinges += n * ne;
  }
  h->ell_faces = nfaces;
  h->ell_hinges = nhinges;
  bool fdamp = false, hdamp = false;
  for (int t = 0; t < h->T; ++t) fdamp |= (mat[5 * t] > 0.f || mat[5 * t + 1] > 0.f) && mat[5 * t + 2] > 0.f;
  for (int e = 0; e < h->E; ++e) hdamp |= bp[2 * e] > 0.f && bp[2 * e + 1] > 0.f;
  h->ell_face_damping = fdamp;
  h->ell_hinge_damping = hdamp;
  std::vector<int2> fnb(size_t(nfaces), make_int2(0, 0));
  std::vector<float4> fdm(size_t(nfaces), make_float4(0.f, 0.f, 0.f, 0.f));
  std::vector<float2> fmat(size_t(nfaces), make_float2(0.f, 0.f));
  std::vector<float> fkd(fdamp ? size_t(nfaces) : 0, 0.f);
  std::vector<int4> hidx(size_t(nhinges), make_int4(0, 0, 0, 0));
  std::vector<float2> hprop(size_t(nhinges), make_float2(0.f, 0.f));
  std::vector<float> hkd(hdamp ? size_t(nhinges) : 0, 0.f);
  for (int r = 0; r < R; ++r) {
    const int a = h->ranges_host[r];
    const long long n = h->ranges_host[r + 1] - a;
    for (int j = 0; j < n; ++j) {
      const int v = h->range_verts_host[a + j];
      int s = 0;
      for (int q = h->h_foff[v]; q < h->h_foff[v + 1]; ++q, ++s) {
        const int t = h->h_fadj[q] >> 2, ord = h->h_fadj[q] & 3;
        const long long i = h->ell_fbase[r] + s * n + j;
        const int* ti = &h->h_tri[3 * size_t(t)];
        const double D00 = pose[4 * t], D01 = pose[4 * t + 1], D10 = pose[4 * t + 2], D11 = pose[4 * t + 3];
        double P00 = D00, P01 = D01, P10 = D10, P11 = D11;
        if (ord == 1) {  // [x2 - x1, x0 - x1] = E [[-1,-1],[1,0]]  ->  D' = [[0,1],[-1,-1]] D
          fnb[i] = make_int2(ti[2], ti[0]);
          P00 = D10, P01 = D11, P10 = -D00 - D10, P11 = -D01 - D11;
        } else if (ord == 2) {  // [x0 - x2, x1 - x2] = E [[0,1],[-1,-1]]  ->  D' = [[-1,-1],[1,0]] D
          fnb[i] = make_int2(ti[0], ti[1]);
          P00 = -D00 - D10, P01 = -D01 - D11, P10 = D00, P11 = D01;
        } else {
          fnb[i] = make_int2(ti[1], ti[2]);
        }
        fdm[i] = make_float4(float(P00), float(P01), float(P10), float(P11));
        fmat[i] = make_float2(mat[5 * t] * area[t], mat[5 * t + 1] * area[t]);
        if (fdamp) fkd[i] = mat[5 * t + 2];
      }
      s = 0;
      for (int q = h->h_eoff[v]; q < h->h_eoff[v + 1]; ++q, ++s) {
        const int e = h->h_eadj[q] >> 2, ord = h->h_eadj[q] & 3;
        const long long i = h->ell_ebase[r] + s * n + j;
        const int* ei = &h->h_edges[4 * size_t(e)];
        hidx[i] = make_int4(ei[0], ei[1], ei[2], int(unsigned(ei[3]) | (unsigned(ord) << 30)));
        const float ke = bp[2 * e];
        hprop[i] = make_float2(ra[e], ke > 0.f ? ke * rl[e] : 0.f);
        if (hdamp) hkd[i] = bp[2 * e + 1];
      }
    }
  }
  if ((rc = upload_into(&h->range_nf, h->ell_nf)) || (rc = upload_into(&h->range_ne, h->ell_ne)) ||
      (rc = upload_into(&h->range_fbase, h->ell_fbase)) || (rc = upload_into(&h->range_ebase, h->ell_ebase)))
    return rc;
  if (h->layout == VBD_LAYOUT_ELL16) {
    // instance-local 16-bit ids: world_of each range's vertices is the instance of the range
    std::vector<uint4> fa(static_cast<size_t>(nfaces)), fb(static_cast<size_t>(nfaces)), hr(static_cast<size_t>(nhinges));
    for (int r = 0; r < R; ++r) {
      const int a = h->ranges_host[r];
      if (h->ranges_host[r + 1] == a) continue;
      const int vs = h->inst_start_of_vertex[h->range_verts_host[a]];
      const long long n = h->ranges_host[r + 1] - a;
      for (long long s = 0; s < h->ell_nf[r]; ++s)
        for (long long j = 0; j < n; ++j) {
          const long long i = h->ell_fbase[r] + s * n + j;
          const unsigned la = unsigned(fnb[i].x - vs), lb = unsigned(fnb[i].y - vs);
          const float mk = fmat[i].x > 0.f || fmat[i].y > 0.f ? 1.f : 0.f;
          fa[i] = make_uint4(mk > 0.f ? (la | (lb << 16)) : 0u, __float_as_uint_host(fmat[i].x),
                             __float_as_uint_host(fmat[i].y), __float_as_uint_host(fdm[i].x));
          fb[i] = make_uint4(__float_as_uint_host(fdm[i].y), __float_as_uint_host(fdm[i].z),
                             __float_as_uint_host(fdm[i].w), __float_as_uint_host(fdamp ? fkd[i] : 0.f));
        }
      for (long long s = 0; s < h->ell_ne[r]; ++s)
        for (long long j = 0; j < n; ++j) {
          const long long i = h->ell_ebase[r] + s * n + j;
          const int4 id = hidx[i];
          const unsigned o[4] = {unsigned(id.x - vs), unsigned(id.y - vs), unsigned(id.z - vs),
                                 unsigned((id.w & 0x3fffffff) - vs)};
          const bool live = hprop[i].y > 0.f;
          hr[i] = make_uint4(live ? (o[0] | (o[1] << 16)) : 0u, live ? (o[2] | (o[3] << 16)) : 0u,
                             __float_as_uint_host(hprop[i].x), __float_as_uint_host(hprop[i].y));
        }
    }
    if ((rc = upload_into(&h->ell16_faceA, fa)) || (rc = upload_into(&h->ell16_faceB, fb)) ||
        (rc = upload_into(&h->ell16_hinge, hr)))
      return rc;
    dfree(h->hinge_kd);  // hinge damping: a float per hinge record, in the same slots
    if (hdamp && (rc = upload_into(&h->hinge_kd, hkd))) return rc;
    return VBD_OK;
  }
  if ((rc = upload_into(&h->face_nb, fnb)) || (rc = upload_into(&h->face_dm, fdm)) ||
      (rc = upload_into(&h->face_mat, fmat)) || (rc = upload_into(&h->hinge_idx, hidx)) ||
      (rc = upload_into(&h->hinge_prop, hprop)))
    return rc;
  dfree(h->face_kd);
  dfree(h->hinge_kd);
  if (fdamp && (rc = upload_into(&h->face_kd, fkd))) return rc;
  if (hdamp && (rc = upload_into(&h->hinge_kd, hkd))) return rc;
  return VBD_OK;
}

// One-ring records (vbd_ring.cuh) for the ranges in h->ranges_host / h->range_verts_host. Returns
// VBD_ERR_UNSUPPORTED when a vertex's triangles do not form one fan of at most kRingMax triangles, or
// when a hinge of the model does not sit where the fan walk evaluates it (a spoke between two fan
// triangles, or a rim whose opposite vertices are the vertex and the outer vertex).
int build_ring(VbdSolver* h) {
  const VbdModelDesc& m = h->md;
  std::vector<float> pose, mat, area, ra, rl, bp;
  int rc;
  if ((rc = download(pose, m.tri_poses_dev, size_t(4) * h->T)) || (rc = download(mat, m.tri_materials_dev, size_t(5) * h->T)) ||
      (rc = download(area, m.tri_areas_dev, size_t(h->T))) || (rc = download(ra, m.edge_rest_angle_dev, size_t(h->E))) ||
      (rc = download(rl, m.edge_rest_length_dev, size_t(h->E))) ||
      (rc = download(bp, m.edge_bending_properties_dev, size_t(2) * h->E)))
    return rc;
  if (needs_lnh_floor(mat, h->T)) return VBD_ERR_UNSUPPORTED;
  // interior hinges with stiffness, by their edge
  auto key = [](int a, int b) { return a < b ? (uint64_t(unsigned(a)) << 32) | unsigned(b) : (uint64_t(unsigned(b)) << 32) | unsigned(a); };
  std::vector<std::pair<uint64_t, int>> emap;
  std::vector<int> live_count(h->V, 0);
  for (int e = 0; e < h->E; ++e) {
    const int* ei = &h->h_edges[4 * size_t(e)];
    if (ei[0] < 0 || ei[1] < 0 || !(bp[2 * e] > 0.f)) continue;
    emap.push_back({key(ei[2], ei[3]), e});
    for (int q = 0; q < 4; ++q) live_count[ei[q]]++;
  }
  std::sort(emap.begin(), emap.end());
  for (size_t i = 1; i < emap.size(); ++i)
    if (emap[i].first == emap[i - 1].first) return VBD_ERR_UNSUPPORTED;  // two hinges on one edge
  auto hinge_of = [&](int a, int b) -> int {
    auto it = std::lower_bound(emap.begin(), emap.end(), std::make_pair(key(a, b), -1));
    return (it != emap.end() && it->first == key(a, b)) ? it->second : -1;
  };
  const int R = int(h->ranges_host.size()) - 1;
  std::vector<int> nslot(R, 0);
  std::vector<long long> base(R, 0), vbase(R, 0);
  // per vertex fan: ring ids, face (triangle, order) per slot, closed flag
  struct Fan {
    int k = 0;
    bool closed = false;
    int ring[kRingMax];
    int tri[kRingMax];
    int ord[kRingMax];
  };
  std::vector<Fan> fans(h->V);
  for (int v = 0; v < h->V; ++v) {
    Fan& F = fans[v];
    const int nf = h->h_foff[v + 1] - h->h_foff[v];
    if (nf == 0) continue;
    if (nf > kRingMax) return VBD_ERR_UNSUPPORTED;
    int fa[kRingMax], fb[kRingMax], ft[kRingMax], fo[kRingMax];
    for (int q = 0; q < nf; ++q) {
      const int t = h->h_fadj[h->h_foff[v] + q] >> 2, ord = h->h_fadj[h->h_foff[v] + q] & 3;
      const int* ti = &h->h_tri[3 * size_t(t)];
      fa[q] = ti[(ord + 1) % 3];
      fb[q] = ti[(ord + 2) % 3];
      ft[q] = t;
      fo[q] = ord;
    }
    // start: a first vertex that no face ends in (open fan), else the first face's (closed fan)
    int start = -1, nstart = 0;
    for (int q = 0; q < nf; ++q) {
      bool incoming = false;
      for (int u = 0; u < nf; ++u) incoming |= fb[u] == fa[q];
      if (!incoming) {
        start = q;
        ++nstart;
      }
    }
    if (nstart > 1) return VBD_ERR_UNSUPPORTED;
    F.closed = nstart == 0;
    int q = F.closed ? 0 : start, used = 0;
    std::vector<char> seen(nf, 0);
    F.k = 0;
    while (true) {
      if (seen[q] || F.k >= kRingMax) return VBD_ERR_UNSUPPORTED;
      seen[q] = 1;
      ++used;
      F.ring[F.k] = fa[q];
      F.tri[F.k] = ft[q];
      F.ord[F.k] = fo[q];
      ++F.k;
      int nq = -1;
      for (int u = 0; u < nf; ++u)
        if (fa[u] == fb[q]) {
          if (nq >= 0) return VBD_ERR_UNSUPPORTED;
          nq = u;
        }
      if (nq < 0) {  // open fan ends at fb[q]
        if (F.closed || F.k >= kRingMax) return VBD_ERR_UNSUPPORTED;
        F.ring[F.k] = fb[q];
        F.tri[F.k] = -1;
        ++F.k;
        break;
      }
      if (F.closed && nq == 0) break;
      q = nq;
    }
    if (used != nf) return VBD_ERR_UNSUPPORTED;
  }
  long long nrec = 0, nv = 0;
  for (int r = 0; r < R; ++r) {
    int ns = 0;
    for (int k = h->ranges_host[r]; k < h->ranges_host[r + 1]; ++k) ns = std::max(ns, fans[h->range_verts_host[k]].k);
    nslot[r] = ns;
    base[r] = nrec;
    vbase[r] = nv;
    const long long n = h->ranges_host[r + 1] - h->ranges_host[r];
    nrec += n * ns;
    nv += n;
  }
  std::vector<uint4> A(size_t(std::max(nrec, 1LL)), make_uint4(0u, 0u, 0u, 0u)), B(A.size(), make_uint4(0u, 0u, 0u, 0u));
  std::vector<float4> Hh(A.size(), make_float4(0.f, 0.f, 0.f, 0.f));
  std::vector<float2> KD(A.size(), make_float2(0.f, 0.f));  // (spoke, rim) hinge damping per slot
  bool any_kd = false;
  std::vector<unsigned> hdr(size_t(std::max(nv, 1LL)), 0u);
  for (int r = 0; r < R; ++r) {
    const int a0 = h->ranges_host[r];
    const long long n = h->ranges_host[r + 1] - a0;
    for (long long j = 0; j < n; ++j) {
      const int v = h->range_verts_host[a0 + j];
      const Fan& F = fans[v];
      const int vs = h->inst_start_of_vertex[v];
      hdr[vbase[r] + j] = unsigned(F.k) | (F.closed ? 0x100u : 0u);
      int found = 0;
      for (int i = 0; i < F.k; ++i) {
        const long long idx = base[r] + i * n + j;
        const int inext = i + 1 < F.k ? i + 1 : (F.closed ? 0 : -1);
        const int iprev = i > 0 ? i - 1 : (F.closed ? F.k - 1 : -1);
        unsigned o_loc = 0xffffu;
        float mu = 0.f, lm = 0.f, kd = 0.f;
        double P00 = 0, P01 = 0, P10 = 0, P11 = 0;
        float4 hv = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 hkd = make_float2(0.f, 0.f);
        if (inext >= 0) {  // face i
          const int t = F.tri[i], ord = F.ord[i];
          const double D00 = pose[4 * t], D01 = pose[4 * t + 1], D10 = pose[4 * t + 2], D11 = pose[4 * t + 3];
          P00 = D00, P01 = D01, P10 = D10, P11 = D11;
          if (ord == 1) {
            P00 = D10, P01 = D11, P10 = -D00 - D10, P11 = -D01 - D11;
          } else if (ord == 2) {
            P00 = -D00 - D10, P01 = -D01 - D11, P10 = D00, P11 = D01;
          }
          mu = mat[5 * t] * area[t];
          lm = mat[5 * t + 1] * area[t];
          kd = mat[5 * t + 2];
          // rim hinge (v, o, r_i, r_{i+1})
          const int e = hinge_of(F.ring[i], F.ring[inext]);
          if (e >= 0) {
            const int* ei = &h->h_edges[4 * size_t(e)];
            int o;
            if (ei[0] == v) o = ei[1];
            else if (ei[1] == v) o = ei[0];
            else return VBD_ERR_UNSUPPORTED;
            const float sgn = (ei[0] == v ? 1.f : -1.f) * (ei[2] == F.ring[i] ? 1.f : -1.f);
            hv.z = sgn * ra[e];
            hv.w = bp[2 * e] * rl[e];
            hkd.y = bp[2 * e + 1];
            o_loc = unsigned(o - vs);
            ++found;
          }
        }
        if (inext >= 0 && iprev >= 0) {  // spoke (r_{i+1}, r_{i-1}, v, r_i)
          const int e = hinge_of(v, F.ring[i]);
          if (e >= 0) {
            const int* ei = &h->h_edges[4 * size_t(e)];
            const int rn = F.ring[inext], rp = F.ring[iprev];
            if (!((ei[0] == rn && ei[1] == rp) || (ei[0] == rp && ei[1] == rn))) return VBD_ERR_UNSUPPORTED;
            const float sgn = (ei[0] == rn ? 1.f : -1.f) * (ei[2] == v ? 1.f : -1.f);
            hv.x = sgn * ra[e];
            hv.y = bp[2 * e] * rl[e];
            hkd.x = bp[2 * e + 1];
            ++found;
          }
        }
        const unsigned r_loc = unsigned(F.ring[i] - vs);
        A[idx] = make_uint4(r_loc | (o_loc << 16), __float_as_uint_host(mu), __float_as_uint_host(lm),
                            __float_as_uint_host(float(P00)));
        B[idx] = make_uint4(__float_as_uint_host(float(P01)), __float_as_uint_host(float(P10)),
                            __float_as_uint_host(float(P11)), __float_as_uint_host(kd));
        Hh[idx] = hv;
        KD[idx] = hkd;
        any_kd |= hkd.x > 0.f || hkd.y > 0.f;
      }
      if (found != live_count[v]) return VBD_ERR_UNSUPPORTED;  // a hinge the fan walk would miss
    }
  }
  std::vector<int> ns(nslot);
  if ((rc = upload_into(&h->ring_nslot, ns)) || (rc = upload_into(&h->ring_base, base)) ||
      (rc = upload_into(&h->ring_vbase, vbase)) || (rc = upload_into(&h->ring_A, A)) || (rc = upload_into(&h->ring_B, B)) ||
      (rc = upload_into(&h->ring_H, Hh)) || (rc = upload_into(&h->ring_hdr, hdr)))
    return rc;
  dfree(h->ring_kd);
  if (any_kd && (rc = upload_into(&h->ring_kd, KD))) return rc;
  return VBD_OK;
}

RingView ring_view(const VbdSolver* h) {
  RingView e;
  e.range_nslot = h->ring_nslot;
  e.range_base = h->ring_base;
  e.range_vbase = h->ring_vbase;
  e.A = h->ring_A;
  e.B = h->ring_B;
  e.H = h->ring_H;
  e.hdr = h->ring_hdr;
  e.kd = h->ring_kd;
  return e;
}

Ell16View ell16_view(const VbdSolver* h) {
  Ell16View e;
  e.range_nf = h->range_nf;
  e.range_ne = h->range_ne;
  e.range_fbase = h->range_fbase;
  e.range_ebase = h->range_ebase;
  e.faceA = h->ell16_faceA;
  e.faceB = h->ell16_faceB;
  e.hinge = h->ell16_hinge;
  e.hinge_kd = h->ell_hinge_damping ? h->hinge_kd : nullptr;
  return e;
}

EllView ell_view(const VbdSolver* h) {
  EllView e;
  e.range_nf = h->range_nf;
  e.range_ne = h->range_ne;
  e.range_fbase = h->range_fbase;
  e.range_ebase = h->range_ebase;
  e.face_nb = h->face_nb;
  e.face_dm = h->face_dm;
  e.face_mat = h->face_mat;
  e.face_kd = h->ell_face_damping ? h->face_kd : nullptr;
  e.hinge_idx = h->hinge_idx;
  e.hinge_prop = h->hinge_prop;
  e.hinge_kd = h->ell_hinge_damping ? h->hinge_kd : nullptr;
  return e;
}

int pack_model(VbdSolver* h, cudaStream_t st) {
  const VbdModelDesc& m = h->md;
  if (h->T > 0) {
    k_pack_tris<<<(h->T + 255) / 256, 256, 0, st>>>(h->T, m.tri_indices_dev, m.tri_poses_dev, m.tri_materials_dev,
                                                     m.tri_areas_dev, h->tri_idx, h->tri_pose, h->tri_mat);
    CK(cudaGetLastError());
  }
  if (h->E > 0) {
    k_pack_edges<<<(h->E + 255) / 256, 256, 0, st>>>(h->E, m.edge_indices_dev, m.edge_rest_angle_dev,
                                                      m.edge_rest_length_dev, m.edge_bending_properties_dev,
                                                      h->edge_idx, h->edge_prop);
    CK(cudaGetLastError());
  }
  if (h->NS > 0) {
    k_pack_springs<<<(h->NS + 255) / 256, 256, 0, st>>>(h->NS, m.spring_indices_dev, m.spring_rest_length_dev,
                                                         m.spring_stiffness_dev, m.spring_damping_dev, h->spr_idx,
                                                         h->spr_prop);
    CK(cudaGetLastError());
  }
  if (h->NT > 0) {
    k_pack_tets<<<(h->NT + 255) / 256, 256, 0, st>>>(h->NT, m.tet_indices_dev, m.tet_poses_dev, m.tet_materials_dev,
                                                      h->tet_idx, h->tet_pose);
    CK(cudaGetLastError());
  }
  return VBD_OK;
}

// Vertex -> tetrahedron entries (tet << 2) | order, by tet id (the reference's fill order,
// solver_vbd.py:1261-1297 with _fill_adjacent_tets), and vertex -> spring entries (spring << 1) | end by
// spring id, split into springs whose other end has another color (solved with the vertex's elements) and
// springs whose ends share a color (summed before the color's solve).
void build_soft_adjacency(int V, int NT, const int* tets, int NS, const int* springs, const std::vector<int>& color_of,
                          std::vector<int>& toff, std::vector<int>& tadj, std::vector<int>& soff,
                          std::vector<int>& sadj, std::vector<int>& ssoff, std::vector<int>& ssadj) {
  toff.assign(V + 1, 0);
  for (int t = 0; t < NT; ++t)
    for (int j = 0; j < 4; ++j) toff[tets[4 * t + j] + 1]++;
  for (int i = 0; i < V; ++i) toff[i + 1] += toff[i];
  tadj.assign(std::max(toff[V], 1), 0);
  std::vector<int> fill(toff.begin(), toff.end() - 1);
  for (int t = 0; t < NT; ++t)
    for (int j = 0; j < 4; ++j) tadj[fill[tets[4 * t + j]]++] = (t << 2) | j;
  soff.assign(V + 1, 0);
  ssoff.assign(V + 1, 0);
  for (int k = 0; k < NS; ++k) {
    const int a = springs[2 * k], b = springs[2 * k + 1];
    std::vector<int>& o = color_of[a] == color_of[b] ? ssoff : soff;
    o[a + 1]++;
    o[b + 1]++;
  }
  for (int i = 0; i < V; ++i) soff[i + 1] += soff[i], ssoff[i + 1] += ssoff[i];
  sadj.assign(std::max(soff[V], 1), 0);
  ssadj.assign(std::max(ssoff[V], 1), 0);
  std::vector<int> f1(soff.begin(), soff.end() - 1), f2(ssoff.begin(), ssoff.end() - 1);
  for (int k = 0; k < NS; ++k) {
    const int a = springs[2 * k], b = springs[2 * k + 1];
    const bool same = color_of[a] == color_of[b];
    std::vector<int>& adj = same ? ssadj : sadj;
    std::vector<int>& fl = same ? f2 : f1;
    adj[fl[a]++] = (k << 1);
    adj[fl[b]++] = (k << 1) | 1;
  }
}

// Adjacency in the solver's packed form: one int per entry, (element << 2) | order, in the
// reference's fill order (faces by triangle id; hinges by edge id with v0, v1, o0, o1), with
// boundary hinges (o0 or o1 == -1, which contribute nothing, particle_vbd_kernels.py:1071-1072)
// left out.
void build_packed_adjacency(int V, int T, const int* tri, int E, const int* edges, std::vector<int>& foff,
                            std::vector<int>& fadj, std::vector<int>& eoff, std::vector<int>& eadj) {
  std::vector<int> cnt(V + 1, 0);
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 3; ++j) cnt[tri[3 * t + j] + 1]++;
  foff.assign(V + 1, 0);
  for (int i = 0; i < V; ++i) foff[i + 1] = foff[i] + cnt[i + 1];
  fadj.assign(std::max(foff[V], 1), 0);
  std::vector<int> fill(foff.begin(), foff.end() - 1);
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 3; ++j) {
      const int v = tri[3 * t + j];
      fadj[fill[v]++] = (t << 2) | j;
    }
  std::fill(cnt.begin(), cnt.end(), 0);
  for (int e = 0; e < E; ++e) {
    const int* ei = edges + 4 * e;
    if (ei[0] < 0 || ei[1] < 0) continue;
    for (int j = 0; j < 4; ++j) cnt[ei[j] + 1]++;
  }
  eoff.assign(V + 1, 0);
  for (int i = 0; i < V; ++i) eoff[i + 1] = eoff[i] + cnt[i + 1];
  eadj.assign(std::max(eoff[V], 1), 0);
  fill.assign(eoff.begin(), eoff.end() - 1);
  for (int e = 0; e < E; ++e) {
    const int* ei = edges + 4 * e;
    if (ei[0] < 0 || ei[1] < 0) continue;
    eadj[fill[ei[2]]++] = (e << 2) | 2;
    eadj[fill[ei[3]]++] = (e << 2) | 3;
    eadj[fill[ei[0]]++] = (e << 2) | 0;
    eadj[fill[ei[1]]++] = (e << 2) | 1;
  }
}

template <typename T>
int upload(T** d, const std::vector<T>& h) {
  int rc = dalloc(d, h.size());
  if (rc) return rc;
  CK(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return VBD_OK;
}

template <typename R, int MODE>
StepCtx<R> make_ctx(VbdSolver* h) {
  StepCtx<R> c;
  std::memset(&c, 0, sizeof(c));
  const VbdModelDesc& m = h->md;
  c.tri_idx = h->tri_idx;
  c.tri_pose = h->tri_pose;
  c.tri_mat = h->tri_mat;
  c.edge_idx = h->edge_idx;
  c.edge_prop = h->edge_prop;
  c.face_off = h->face_off;
  c.face_adj = h->face_adj;
  c.edge_off = h->edge_off;
  c.edge_adj = h->edge_adj;
  c.mass = m.particle_mass_dev;
  c.inv_mass = m.particle_inv_mass_dev;
  c.flags = m.particle_flags_dev;
  c.radius = m.particle_radius_dev;
  c.gravity = m.gravity_dev;
  c.pos = (pos4_t<R>*)h->pos;
  c.qprev = (pos4_t<R>*)h->qprev;
  c.inertia = (pos4_t<R>*)h->inertia;
  c.K = h->K;
  c.slot_cnt = h->slot_cnt;
  c.slots = h->slots;
  c.c_k = h->c_k;
  c.c_ke = h->c_ke;
  c.c_kd = h->c_kd;
  c.c_mu = h->c_mu;
  c.soft_ke = m.soft_contact_ke;
  c.soft_kd = m.soft_contact_kd;
  c.soft_mu = m.soft_contact_mu;
  c.shape_ke = m.shape_material_ke_dev;
  c.shape_kd = m.shape_material_kd_dev;
  c.shape_mu = m.shape_material_mu_dev;
  c.shape_body = m.shape_body_dev;
  c.body_com = m.body_com_dev;
  c.k_start = h->prm.avbd_linear_beta == 0.f ? -1.f : h->prm.contact_k_start;
  c.beta = R(h->prm.avbd_linear_beta);
  c.fric_eps = R(h->prm.friction_epsilon);
  c.fp64_thr = h->prm.fp64_solve_threshold;
  c.err = h->err;
  c.residual = MODE == MODE_MIXED ? h->residual : nullptr;
  c.V = h->V;
  c.S = h->S;
  c.dual_in_solve = 1;
  if (h->soft) {
    c.spr_idx = h->spr_idx;
    c.spr_prop = h->spr_prop;
    c.spr_off = h->spr_off;
    c.spr_adj = h->spr_adj;
    c.sspr_off = h->sspr_off;
    c.sspr_adj = h->sspr_adj;
    c.n_same_springs = h->n_same_springs;
    c.spr_acc = (R*)h->spr_acc;
    c.tet_idx = h->tet_idx;
    c.tet_pose = h->tet_pose;
    c.tet_off = h->tet_off;
    c.tet_adj = h->tet_adj;
  }
  return c;
}

template <typename R, int MODE, int L>
void launch_color(const StepCtx<R>& c, const int* verts, int n, int it, int block, cudaStream_t st) {
  const long threads = long(n) * L;
  const int grid = int((threads + block - 1) / block);
  if (grid > 0) k_color<R, L, MODE><<<grid, block, 0, st>>>(c, verts, n, it);
}

template <typename R, int MODE>
void launch_color_any(int L, const StepCtx<R>& c, const int* verts, int n, int it, int block, cudaStream_t st) {
  switch (L) {
    case 1: launch_color<R, MODE, 1>(c, verts, n, it, block, st); break;
    case 2: launch_color<R, MODE, 2>(c, verts, n, it, block, st); break;
    case 4: launch_color<R, MODE, 4>(c, verts, n, it, block, st); break;
    case 8: launch_color<R, MODE, 8>(c, verts, n, it, block, st); break;
    case 16: launch_color<R, MODE, 16>(c, verts, n, it, block, st); break;
    default: launch_color<R, MODE, 32>(c, verts, n, it, block, st); break;
  }
}

template <typename R, int MODE, bool SMEM>
const void* persistent_fn(int L) {
  switch (L) {
    case 1: return (const void*)k_persistent<R, 1, MODE, SMEM>;
    case 2: return (const void*)k_persistent<R, 2, MODE, SMEM>;
    case 4: return (const void*)k_persistent<R, 4, MODE, SMEM>;
    case 8: return (const void*)k_persistent<R, 8, MODE, SMEM>;
    case 16: return (const void*)k_persistent<R, 16, MODE, SMEM>;
    default: return (const void*)k_persistent<R, 32, MODE, SMEM>;
  }
}

template <typename R, int MODE, bool SMEM>
void launch_persistent(int L, const StepCtx<R>& c, const PersistentPlan& p, int grid, int block, size_t smem,
                       cudaStream_t st) {
  switch (L) {
    case 1: k_persistent<R, 1, MODE, SMEM><<<grid, block, smem, st>>>(c, p); break;
    case 2: k_persistent<R, 2, MODE, SMEM><<<grid, block, smem, st>>>(c, p); break;
    case 4: k_persistent<R, 4, MODE, SMEM><<<grid, block, smem, st>>>(c, p); break;
    case 8: k_persistent<R, 8, MODE, SMEM><<<grid, block, smem, st>>>(c, p); break;
    case 16: k_persistent<R, 16, MODE, SMEM><<<grid, block, smem, st>>>(c, p); break;
    default: k_persistent<R, 32, MODE, SMEM><<<grid, block, smem, st>>>(c, p); break;
  }
}

template <typename R, int MODE, bool SMEM>
void launch_persistent_ell16(int occ, const StepCtx<R>& c, const PersistentPlan& p, const Ell16View& e, int grid,
                             int block, size_t smem, cudaStream_t st) {
  switch (occ) {
    case 2: k_persistent_ell16<R, MODE, SMEM, 2><<<grid, block, smem, st>>>(c, p, e); break;
    case 3: k_persistent_ell16<R, MODE, SMEM, 3><<<grid, block, smem, st>>>(c, p, e); break;
    case 4: k_persistent_ell16<R, MODE, SMEM, 4><<<grid, block, smem, st>>>(c, p, e); break;
    default: k_persistent_ell16<R, MODE, SMEM, 0><<<grid, block, smem, st>>>(c, p, e); break;
  }
}

template <typename R, int MODE, bool SMEM>
void launch_persistent_ring(int occ, const StepCtx<R>& c, const PersistentPlan& p, const RingView& e, int grid,
                            int block, size_t smem, cudaStream_t st) {
  switch (occ) {
    case 2: k_persistent_ring<R, MODE, SMEM, 2><<<grid, block, smem, st>>>(c, p, e); break;
    case 3: k_persistent_ring<R, MODE, SMEM, 3><<<grid, block, smem, st>>>(c, p, e); break;
    case 4: k_persistent_ring<R, MODE, SMEM, 4><<<grid, block, smem, st>>>(c, p, e); break;
    default: k_persistent_ring<R, MODE, SMEM, 0><<<grid, block, smem, st>>>(c, p, e); break;
  }
}

template <typename R, int MODE, bool SMEM>
void launch_persistent_ell(int occ, const StepCtx<R>& c, const PersistentPlan& p, const EllView& e, int grid,
                           int block, size_t smem, cudaStream_t st) {
  switch (occ) {
    case 2: k_persistent_ell<R, MODE, SMEM, 2><<<grid, block, smem, st>>>(c, p, e); break;
    case 3: k_persistent_ell<R, MODE, SMEM, 3><<<grid, block, smem, st>>>(c, p, e); break;
    case 4: k_persistent_ell<R, MODE, SMEM, 4><<<grid, block, smem, st>>>(c, p, e); break;
    default: k_persistent_ell<R, MODE, SMEM, 0><<<grid, block, smem, st>>>(c, p, e); break;
  }
}

// ------------------------------------------------------------------------------ self-contact (host)
struct ScSetup {
  double margin, rest_excl, ee_eps;
  const float* rest_q;
  int* err;
};

// Buffers of one detector for V particles, T triangles and E edges (positions of type R).
template <typename R>
int sc_alloc(ScBuffers& b, int V, int T, int E, int vb, int eb) {
  int rc;
  b.V = V, b.T = T, b.E = E, b.vb = vb, b.eb = eb;
  const int P = std::max(T, E);
  int nb = 1024;
  while (nb < 4 * P && nb < (1 << 30)) nb <<= 1;
  b.nbuckets = nb;
  b.gcap = 8LL * std::max(P, 1);
  b.ecap = 4LL * V * vb + 2LL * E * eb;
  if ((rc = dalloc(&b.bcount, size_t(nb) + 1)) || (rc = dalloc(&b.bstart, size_t(nb) + 1)) ||
      (rc = dalloc(&b.ekey, size_t(b.gcap))) || (rc = dalloc(&b.eprim, size_t(b.gcap))) ||
      (rc = dalloc((pos4_t<R>**)&b.blo, size_t(std::max(P, 1)))) ||
      (rc = dalloc((pos4_t<R>**)&b.bhi, size_t(std::max(P, 1)))) || (rc = dalloc(&b.stats, 4)) ||
      (rc = dalloc(&b.vt_tri, size_t(V) * vb)) || (rc = dalloc(&b.vt_count, size_t(V))) ||
      (rc = dalloc((R**)&b.vt_min, size_t(V))) || (rc = dalloc(&b.ee_edge, size_t(E) * eb)) ||
      (rc = dalloc(&b.ee_count, size_t(E))) || (rc = dalloc((R**)&b.ee_min, size_t(E))) ||
      (rc = dalloc(&b.flags, 4)) || (rc = dalloc(&b.tmp, size_t(std::max(V, E)) + 1)) ||
      (rc = dalloc(&b.vt_off, size_t(V) + 1)) || (rc = dalloc(&b.vt_pairs, size_t(V) * vb)) ||
      (rc = dalloc(&b.ee_off, size_t(E) + 1)) || (rc = dalloc(&b.ee_pairs, size_t(E) * eb)) ||
      (rc = dalloc(&b.ent_cnt, size_t(V) + 1)) || (rc = dalloc(&b.ent_off, size_t(V) + 1)) ||
      (rc = dalloc(&b.ent, size_t(b.ecap))))
    return rc;
  size_t b1 = 0, b2 = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, b1, b.bcount, b.bstart, nb + 1));
  CK(cub::DeviceScan::ExclusiveSum(nullptr, b2, b.tmp, b.vt_off, std::max(V, E) + 1));
  b.scan_bytes = std::max(b1, b2);
  if ((rc = dalloc((char**)&b.scan_tmp, b.scan_bytes))) return rc;
  CK(cudaMemset(b.flags, 0, 4 * sizeof(int)));
  return VBD_OK;
}

template <typename T>
int scan(ScBuffers& b, const T* in, T* out, int n, cudaStream_t st) {
  size_t bytes = b.scan_bytes;
  CK(cub::DeviceScan::ExclusiveSum(b.scan_tmp, bytes, in, out, n, st));
  return VBD_OK;
}

// One detection at positions pos (grid build + narrow phase for triangles, then edges).
template <typename R>
int sc_detect(ScBuffers& b, const ScSetup& p, const int4* tri_idx, const int4* edge_idx, const pos4_t<R>* pos,
              int what, cudaStream_t st) {
  ScQuery q;
  q.V = b.V, q.T = b.T, q.E = b.E, q.vb = b.vb, q.eb = b.eb, q.nb = b.nbuckets;
  q.margin = float(p.margin), q.rest_excl = float(p.rest_excl), q.ee_eps = float(p.ee_eps);
  q.tri_idx = tri_idx, q.edge_idx = edge_idx, q.rest_q = p.rest_q;
  q.vt_foff = b.vt_foff, q.vt_f = b.vt_f, q.ee_foff = b.ee_foff, q.ee_f = b.ee_f;
  q.bstart = b.bstart, q.ekey = b.ekey, q.eprim = b.eprim, q.stats = b.stats, q.flags = b.flags;
  q.gcap = (unsigned)std::min<long long>(b.gcap, 0xFFFFFFFFLL);
  q.tv = b.tb > 0 ? b.tv : nullptr, q.tv_count = b.tv_count, q.tv_min = b.tv_min, q.tb = b.tb;
  q.world = b.world;
  pos4_t<R>* lo = (pos4_t<R>*)b.blo;
  pos4_t<R>* hi = (pos4_t<R>*)b.bhi;
  for (int kind = 0; kind < 2; ++kind) {
    if (!(what & (1 << kind))) continue;
    const int P = kind == 0 ? b.T : b.E;
    const int Q = kind == 0 ? b.V : b.E;
    if (Q == 0) continue;
    if (P == 0) {  // nothing to collide with
      CK(cudaMemsetAsync(kind == 0 ? b.vt_count : b.ee_count, 0, sizeof(int) * Q, st));
      k_sc_fill<R><<<(Q + 255) / 256, 256, 0, st>>>(Q, (R*)(kind == 0 ? b.vt_min : b.ee_min), R(p.margin));
      continue;
    }
    CK(cudaMemsetAsync(b.stats, 0, 2 * sizeof(double), st));
    k_sc_boxes<R><<<(P + 255) / 256, 256, 0, st>>>(kind, P, pos, tri_idx, edge_idx, lo, hi, b.stats);
    k_sc_cell<<<1, 1, 0, st>>>(b.stats, P, p.margin);
    CK(cudaMemsetAsync(b.bcount, 0, sizeof(unsigned) * (size_t(b.nbuckets) + 1), st));
    k_sc_grid<R, false><<<(P + 255) / 256, 256, 0, st>>>(P, lo, hi, b.stats, b.nbuckets, b.bcount, nullptr, nullptr,
                                                          nullptr, 0, b.flags);
    int rc = scan<unsigned>(b, b.bcount, b.bstart, b.nbuckets + 1, st);
    if (rc) return rc;
    CK(cudaMemsetAsync(b.bcount, 0, sizeof(unsigned) * (size_t(b.nbuckets) + 1), st));
    k_sc_grid<R, true><<<(P + 255) / 256, 256, 0, st>>>(P, lo, hi, b.stats, b.nbuckets, b.bcount, b.bstart, b.ekey,
                                                         b.eprim, b.gcap, b.flags);
    if (kind == 0)
      k_sc_query_vt<R><<<(Q + 127) / 128, 128, 0, st>>>(q, pos, lo, hi, b.vt_tri, b.vt_count, (R*)b.vt_min);
    else
      k_sc_query_ee<R><<<(Q + 127) / 128, 128, 0, st>>>(q, pos, lo, hi, b.ee_edge, b.ee_count, (R*)b.ee_min);
  }
  CK(cudaGetLastError());
  return VBD_OK;
}

// Dense pair lists and per-vertex entry lists of the last detection.
int sc_compact(ScBuffers& b, const int4* tri_idx, const int4* edge_idx, cudaStream_t st) {
  int rc;
  k_sc_stored<<<(b.V + 256) / 256, 256, 0, st>>>(b.V, b.vb, b.vt_count, b.tmp);
  if ((rc = scan<int>(b, b.tmp, b.vt_off, b.V + 1, st))) return rc;
  if (b.V)
    k_sc_pairs<false><<<(b.V + 255) / 256, 256, 0, st>>>(b.V, b.vb, b.vt_count, b.vt_tri, b.vt_off, tri_idx, edge_idx,
                                                          b.vt_pairs);
  k_sc_stored<<<(b.E + 256) / 256, 256, 0, st>>>(b.E, b.eb, b.ee_count, b.tmp);
  if ((rc = scan<int>(b, b.tmp, b.ee_off, b.E + 1, st))) return rc;
  if (b.E)
    k_sc_pairs<true><<<(b.E + 255) / 256, 256, 0, st>>>(b.E, b.eb, b.ee_count, b.ee_edge, b.ee_off, tri_idx, edge_idx,
                                                         b.ee_pairs);
  CK(cudaMemsetAsync(b.ent_cnt, 0, sizeof(int) * (size_t(b.V) + 1), st));
  k_sc_entries<false><<<kScGridBlocks, 256, 0, st>>>(b.vt_off + b.V, b.ee_off + b.E, b.vt_pairs, b.ee_pairs,
                                                      b.ent_cnt, nullptr, nullptr, 0, b.flags);
  if ((rc = scan<int>(b, b.ent_cnt, b.ent_off, b.V + 1, st))) return rc;
  CK(cudaMemsetAsync(b.ent_cnt, 0, sizeof(int) * (size_t(b.V) + 1), st));
  k_sc_entries<true><<<kScGridBlocks, 256, 0, st>>>(b.vt_off + b.V, b.ee_off + b.E, b.vt_pairs, b.ee_pairs,
                                                     b.ent_cnt, b.ent_off, b.ent, b.ecap, b.flags);
  k_sc_sort_entries<<<(b.V + 127) / 128, 128, 0, st>>>(b.V, b.ent_off, b.ent);
  CK(cudaGetLastError());
  return VBD_OK;
}

// Copies a host CSR filter (rows sorted here) to the device; rows = number of rows, ids < limit.
int sc_upload_filter(const int32_t* off_h, const int32_t* list_h, int rows, int limit, int** off_d, int** list_d) {
  *off_d = nullptr, *list_d = nullptr;
  if (!off_h) return VBD_OK;
  if (off_h[0] != 0) return VBD_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < rows; ++i)
    if (off_h[i + 1] < off_h[i]) return VBD_ERR_INVALID_ARGUMENT;
  const int n = off_h[rows];
  if (n > 0 && !list_h) return VBD_ERR_INVALID_ARGUMENT;
  std::vector<int> off(off_h, off_h + rows + 1), list(list_h, list_h + n);
  for (int v : list)
    if (v < 0 || v >= limit) return VBD_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < rows; ++i) std::sort(list.begin() + off[i], list.begin() + off[i + 1]);
  int rc = upload(off_d, off);
  if (rc) return rc;
  if (list.empty()) list.push_back(0);
  return upload(list_d, list);
}

ScSetup sc_setup(VbdSolver* h) { return {h->sc_margin, h->sc_rest_excl, h->sc_ee_eps, h->sc_rest_q, h->err}; }

// _collision_detection_penetration_free: positions at detection, zero displacements, detect, compact.
template <typename R>
int sc_collide(VbdSolver* h, const R* q_state, cudaStream_t st) {
  pos4_t<R>* pcd = (pos4_t<R>*)h->sc_pos_cd;
  pos4_t<R>* dsp = (pos4_t<R>*)h->sc_disp;
  if (q_state)
    k_sc_begin_from_state<R><<<(h->V + 255) / 256, 256, 0, st>>>(h->V, q_state, pcd, dsp);
  else
    k_sc_begin_from_pos<R><<<(h->V + 255) / 256, 256, 0, st>>>(h->V, (const pos4_t<R>*)h->pos, pcd, dsp);
  int rc = sc_detect<R>(h->sc, sc_setup(h), h->tri_idx, h->edge_idx, pcd, 3, st);
  if (rc) return rc;
  return sc_compact(h->sc, h->tri_idx, h->edge_idx, st);
}

// _penetration_free_truncation with self-contact on.
template <typename R>
void sc_truncate(VbdSolver* h, cudaStream_t st) {
  ScBuffers& b = h->sc;
  k_sc_trunc_pairs<R><<<kScGridBlocks, 256, 0, st>>>(b.vt_off + b.V, b.ee_off + b.E, b.vt_pairs, b.ee_pairs,
                                                      (const pos4_t<R>*)h->sc_pos_cd,
                                                      (const pos4_t<R>*)h->sc_disp, R(h->sc_ee_eps), R(h->sc_relax),
                                                      (R*)h->sc_ts);
  k_sc_trunc_apply<R><<<(h->V + 255) / 256, 256, 0, st>>>(h->V, (R*)h->sc_ts, R(h->sc_margin * h->sc_relax * 0.5),
                                                           (const pos4_t<R>*)h->sc_pos_cd, (pos4_t<R>*)h->sc_disp,
                                                           (pos4_t<R>*)h->pos);
}

template <typename R, int MODE, int L>
void launch_color_sc(const StepCtx<R>& c, const int* verts, int n, int it, int block, cudaStream_t st) {
  const long threads = long(n) * L;
  const int grid = int((threads + block - 1) / block);
  if (grid > 0) k_color<R, L, MODE, true><<<grid, block, 0, st>>>(c, verts, n, it);
}

template <typename R, int MODE>
void launch_color_sc_any(int L, const StepCtx<R>& c, const int* verts, int n, int it, int block, cudaStream_t st) {
  switch (L) {
    case 1: launch_color_sc<R, MODE, 1>(c, verts, n, it, block, st); break;
    case 2: launch_color_sc<R, MODE, 2>(c, verts, n, it, block, st); break;
    case 4: launch_color_sc<R, MODE, 4>(c, verts, n, it, block, st); break;
    case 8: launch_color_sc<R, MODE, 8>(c, verts, n, it, block, st); break;
    case 16: launch_color_sc<R, MODE, 16>(c, verts, n, it, block, st); break;
    default: launch_color_sc<R, MODE, 32>(c, verts, n, it, block, st); break;
  }
}

int ensure_contact_capacity(VbdSolver* h, int cmax, cudaStream_t st) {
  if (cmax <= h->c_cap) return VBD_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return VBD_ERR_UNSUPPORTED;  // growing buffers during capture
  for (float** p : {&h->c_k, &h->c_ke, &h->c_kd, &h->c_mu}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    int rc = dalloc(p, size_t(cmax));
    if (rc) return rc;
  }
  h->c_cap = cmax;
  return VBD_OK;
}

template <typename R, int MODE>
int step_impl(VbdSolver* h, R* q_in, R* q_out, const R* qd_in, R* qd_out, const R* f_ext,
              const VbdContactsDesc* contacts, const VbdBodyState* bodies, R dt, cudaStream_t st) {
  if (!q_in || !q_out || !qd_in || !qd_out || !(dt > R(0))) return VBD_ERR_INVALID_ARGUMENT;
  StepCtx<R> c = make_ctx<R, MODE>(h);
  c.q_in = q_in;
  c.q_out = q_out;
  c.qd_in = qd_in;
  c.qd_out = qd_out;
  c.f_ext = f_ext;
  c.dt = dt;
  c.dt2r = R(1) / (dt * dt);
  const bool has_c = contacts && contacts->soft_contact_max > 0 && contacts->soft_contact_count_dev;
  if (has_c) {
    int rc = ensure_contact_capacity(h, contacts->soft_contact_max, st);
    if (rc) return rc;
    c = make_ctx<R, MODE>(h);
    c.q_in = q_in;
    c.q_out = q_out;
    c.qd_in = qd_in;
    c.qd_out = qd_out;
    c.f_ext = f_ext;
    c.dt = dt;
    c.dt2r = R(1) / (dt * dt);
    c.has_contacts = 1;
    c.c_count = contacts->soft_contact_count_dev;
    c.c_max = contacts->soft_contact_max;
    c.c_particle = contacts->soft_contact_particle_dev;
    c.c_shape = contacts->soft_contact_shape_dev;
    c.c_body_pos = contacts->soft_contact_body_pos_dev;
    c.c_body_vel = contacts->soft_contact_body_vel_dev;
    c.c_normal = contacts->soft_contact_normal_dev;
    if (bodies) {
      c.body_q = bodies->body_q_dev;
      c.body_q_prev = bodies->body_q_prev_dev;
      c.body_qd = bodies->body_qd_dev;
    }
  }
  const int iters = h->prm.iterations;
  if (MODE == MODE_MIXED) CK(cudaMemsetAsync(h->residual, 0, sizeof(double) * 32 * std::max(iters, 1), st));
  if (h->sc_on && h->schedule == VBD_SCHEDULE_PERSISTENT) {
    // self-contact, one instance per CTA: the detections stay grid-wide launches over all instances (pairs within
    // an instance only); between them one persistent launch runs the forward step and its truncation, then one per
    // detection interval runs the iterations, each color followed by the truncation of the instance's own pairs
    c.disp = (pos4_t<R>*)h->sc_disp;
    c.pos_cd = (pos4_t<R>*)h->sc_pos_cd;
    c.ent_off = h->sc.ent_off;
    c.ent = h->sc.ent;
    c.vt_pairs = h->sc.vt_pairs;
    c.ee_pairs = h->sc.ee_pairs;
    c.sc_radius = h->sc_radius;
    c.sc_ee_eps = h->sc_ee_eps;
    c.dual_in_solve = 1;
    int rc = sc_collide<R>(h, q_in, st);
    if (rc) return rc;
    if (has_c) {
      CK(cudaMemsetAsync(h->slot_cnt, 0, sizeof(int) * h->V, st));
      k_contact_prepare<R><<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
    }
    PersistentPlan p{h->W, h->inst_order, h->inst_vstart, h->inst_cptr, h->color_ranges, h->color_verts, h->queue,
                     iters};
    ScPersistentPlan s{h->sc_estart, h->sc.vt_off, h->sc.ee_off, h->sc.vt_pairs, h->sc.ee_pairs, h->sc_ts,
                       h->sc_ee_eps, h->sc_relax, h->sc_margin * h->sc_relax * 0.5, 0, 0, 0, 0};
    CK(cudaMemsetAsync(h->queue, 0, sizeof(int), st));
    launch_persistent_sc<R, MODE>(h->L, c, p, s, h->grid_sc, h->block, st);
    s.phase = 1;
    int it = 0;
    do {
      // a detection at iteration `it` (interval 0: iteration 0 only; a negative interval: none)
      if (iters > 0 && h->sc_interval >= 0 && (rc = sc_collide<R>(h, nullptr, st))) return rc;
      const int it1 = h->sc_interval >= 1 ? std::min(iters, it + h->sc_interval) : iters;
      s.it0 = it, s.it1 = it1, s.finalize = it1 == iters;
      CK(cudaMemsetAsync(h->queue, 0, sizeof(int), st));
      launch_persistent_sc<R, MODE>(h->L, c, p, s, h->grid_sc, h->block, st);
      it = it1;
    } while (it < iters);
    CK(cudaGetLastError());
  } else if (h->schedule == VBD_SCHEDULE_PERSISTENT) {
    CK(cudaMemsetAsync(h->queue, 0, sizeof(int), st));
    if (has_c) {
      CK(cudaMemsetAsync(h->slot_cnt, 0, sizeof(int) * h->V, st));
      k_contact_prepare<R><<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
    }
    PersistentPlan p{h->W, h->inst_order, h->inst_vstart, h->inst_cptr, h->color_ranges, h->color_verts, h->queue,
                     iters};
    if (h->layout == VBD_LAYOUT_RING) {
      const RingView e = ring_view(h);
      if constexpr (std::is_same<R, float>::value) {
        if (h->smem_bytes > 0)
          launch_persistent_ring<R, MODE, true>(h->occ, c, p, e, h->grid_persistent, h->block, h->smem_bytes, st);
        else
          launch_persistent_ring<R, MODE, false>(h->occ, c, p, e, h->grid_persistent, h->block, 0, st);
      } else {
        launch_persistent_ring<R, MODE, false>(0, c, p, e, h->grid_persistent, h->block, 0, st);
      }
    } else if (h->layout == VBD_LAYOUT_ELL16) {
      const Ell16View e = ell16_view(h);
      if constexpr (std::is_same<R, float>::value) {
        if (MODE == MODE_FP32 && h->pair && h->smem_bytes > 0)
          launch_persistent_ell16_pair<true>(h->occ, c, p, e, h->grid_persistent, h->block, h->smem_bytes, st);
        else if (MODE == MODE_FP32 && h->pair)
          launch_persistent_ell16_pair<false>(h->occ, c, p, e, h->grid_persistent, h->block, 0, st);
        else if (h->ell_hinge_damping && h->smem_bytes > 0)
          launch_persistent_ell16_damped<R, MODE, true>(h->occ, c, p, e, h->grid_persistent, h->block, h->smem_bytes,
                                                        st);
        else if (h->ell_hinge_damping)
          launch_persistent_ell16_damped<R, MODE, false>(h->occ, c, p, e, h->grid_persistent, h->block, 0, st);
        else if (h->smem_bytes > 0)
          launch_persistent_ell16<R, MODE, true>(h->occ, c, p, e, h->grid_persistent, h->block, h->smem_bytes, st);
        else
          launch_persistent_ell16<R, MODE, false>(h->occ, c, p, e, h->grid_persistent, h->block, 0, st);
      } else if (h->ell_hinge_damping) {
        launch_persistent_ell16_damped<R, MODE, false>(0, c, p, e, h->grid_persistent, h->block, 0, st);
      } else {
        launch_persistent_ell16<R, MODE, false>(0, c, p, e, h->grid_persistent, h->block, 0, st);
      }
    } else if (h->layout == VBD_LAYOUT_ELL) {
      const EllView e = ell_view(h);
      if constexpr (std::is_same<R, float>::value) {
        if (h->smem_bytes > 0)
          launch_persistent_ell<R, MODE, true>(h->occ, c, p, e, h->grid_persistent, h->block, h->smem_bytes, st);
        else
          launch_persistent_ell<R, MODE, false>(h->occ, c, p, e, h->grid_persistent, h->block, 0, st);
      } else {
        launch_persistent_ell<R, MODE, false>(0, c, p, e, h->grid_persistent, h->block, 0, st);
      }
    } else if (h->warp_inst) {
      if constexpr (std::is_same<R, float>::value) {
        if (h->smem_bytes > 0)
          launch_persistent_warp<R, MODE, true>(h->soft, h->L, c, p, h->slice, h->grid_persistent, h->block,
                                               h->smem_bytes, st);
        else
          launch_persistent_warp<R, MODE, false>(h->soft, h->L, c, p, 0, h->grid_persistent, h->block, 0, st);
      } else {
        launch_persistent_warp<R, MODE, false>(h->soft, h->L, c, p, 0, h->grid_persistent, h->block, 0, st);
      }
    } else if (h->soft) {
      if constexpr (std::is_same<R, float>::value) {
        if (h->smem_bytes > 0)
          launch_persistent_soft<R, MODE, true>(h->L, c, p, h->grid_persistent, h->block, h->smem_bytes, st);
        else
          launch_persistent_soft<R, MODE, false>(h->L, c, p, h->grid_persistent, h->block, 0, st);
      } else {
        launch_persistent_soft<R, MODE, false>(h->L, c, p, h->grid_persistent, h->block, 0, st);
      }
    } else if constexpr (std::is_same<R, float>::value) {
      if (h->smem_bytes > 0)
        launch_persistent<R, MODE, true>(h->L, c, p, h->grid_persistent, h->block, h->smem_bytes, st);
      else
        launch_persistent<R, MODE, false>(h->L, c, p, h->grid_persistent, h->block, 0, st);
    } else {
      launch_persistent<R, MODE, false>(h->L, c, p, h->grid_persistent, h->block, 0, st);
    }
  } else if (h->sc_on) {
    // self-contact (solver_vbd.py:1731-1766, 2151-2337): detection at the step's start positions, forward
    // step, truncation; per iteration an optional re-detection, then per color the solve and a truncation
    c.disp = (pos4_t<R>*)h->sc_disp;
    c.pos_cd = (pos4_t<R>*)h->sc_pos_cd;
    c.ent_off = h->sc.ent_off;
    c.ent = h->sc.ent;
    c.vt_pairs = h->sc.vt_pairs;
    c.ee_pairs = h->sc.ee_pairs;
    c.sc_radius = h->sc_radius;
    c.sc_ee_eps = h->sc_ee_eps;
    const bool sep_duals = has_c && c.beta != R(0);
    c.dual_in_solve = sep_duals ? 0 : 1;
    int rc = sc_collide<R>(h, q_in, st);
    if (rc) return rc;
    k_forward<R><<<(h->V + 255) / 256, 256, 0, st>>>(c);
    if (has_c) k_contact_prepare<R><<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
    sc_truncate<R>(h, st);
    const int* cp = h->md.color_particles_dev;
    for (int it = 0; it < iters; ++it) {
      if (sep_duals) k_contact_duals<R><<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
      if ((h->sc_interval == 0 && it == 0) || (h->sc_interval >= 1 && it % h->sc_interval == 0)) {
        if ((rc = sc_collide<R>(h, nullptr, st))) return rc;
      }
      for (size_t col = 0; col + 1 < h->color_offsets.size(); ++col) {
        const int a = h->color_offsets[col], b = h->color_offsets[col + 1];
        if (h->soft)
          launch_color_soft<R, MODE>(true, h->L, c, cp + a, b - a, it, h->block, st);
        else
          launch_color_sc_any<R, MODE>(h->L, c, cp + a, b - a, it, h->block, st);
        sc_truncate<R>(h, st);
      }
    }
    k_finalize<R><<<(h->V + 255) / 256, 256, 0, st>>>(c);
  } else {
    k_forward<R><<<(h->V + 255) / 256, 256, 0, st>>>(c);
    if (has_c) k_contact_prepare<R><<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
    const int* cp = h->md.color_particles_dev;
    const EllView e = ell_view(h);
    for (int it = 0; it < iters; ++it)
      for (size_t col = 0; col + 1 < h->color_offsets.size(); ++col) {
        const int a = h->color_offsets[col], b = h->color_offsets[col + 1];
        if (h->layout == VBD_LAYOUT_ELL) {
          if (b > a) k_color_ell<R, MODE><<<(b - a + h->block - 1) / h->block, h->block, 0, st>>>(c, e, cp + a, int(col), b - a, it);
        } else if (h->soft) {
          launch_color_soft<R, MODE>(false, h->L, c, cp + a, b - a, it, h->block, st);
        } else {
          launch_color_any<R, MODE>(h->L, c, cp + a, b - a, it, h->block, st);
        }
      }
    k_finalize<R><<<(h->V + 255) / 256, 256, 0, st>>>(c);
  }
  CK(cudaGetLastError());
  return VBD_OK;
}

template <typename R, int MODE, bool SMEM>
const void* persistent_ring_fn(int occ) {
  switch (occ) {
    case 2: return (const void*)k_persistent_ring<R, MODE, SMEM, 2>;
    case 3: return (const void*)k_persistent_ring<R, MODE, SMEM, 3>;
    case 4: return (const void*)k_persistent_ring<R, MODE, SMEM, 4>;
    default: return (const void*)k_persistent_ring<R, MODE, SMEM, 0>;
  }
}

template <typename R, int MODE, bool SMEM>
const void* persistent_ell16_fn(int occ) {
  switch (occ) {
    case 2: return (const void*)k_persistent_ell16<R, MODE, SMEM, 2>;
    case 3: return (const void*)k_persistent_ell16<R, MODE, SMEM, 3>;
    case 4: return (const void*)k_persistent_ell16<R, MODE, SMEM, 4>;
    default: return (const void*)k_persistent_ell16<R, MODE, SMEM, 0>;
  }
}

template <typename R, int MODE, bool SMEM>
const void* persistent_ell_fn(int occ) {
  switch (occ) {
    case 2: return (const void*)k_persistent_ell<R, MODE, SMEM, 2>;
    case 3: return (const void*)k_persistent_ell<R, MODE, SMEM, 3>;
    case 4: return (const void*)k_persistent_ell<R, MODE, SMEM, 4>;
    default: return (const void*)k_persistent_ell<R, MODE, SMEM, 0>;
  }
}


const void* persistent_kernel(VbdSolver* h) {
  const bool sm = h->smem_bytes > 0;
  if (h->layout == VBD_LAYOUT_RING) {
    if (h->precision == VBD_PRECISION_FP64) return persistent_ring_fn<double, MODE_FP64, false>(0);
    if (h->precision == VBD_PRECISION_MIXED)
      return sm ? persistent_ring_fn<float, MODE_MIXED, true>(h->occ) : persistent_ring_fn<float, MODE_MIXED, false>(h->occ);
    return sm ? persistent_ring_fn<float, MODE_FP32, true>(h->occ) : persistent_ring_fn<float, MODE_FP32, false>(h->occ);
  }
  if (h->layout == VBD_LAYOUT_ELL16 && h->pair)
    return sm ? persistent_ell16_pair_fn<true>(h->occ) : persistent_ell16_pair_fn<false>(h->occ);
  if (h->layout == VBD_LAYOUT_ELL16 && h->ell_hinge_damping) {
    if (h->precision == VBD_PRECISION_FP64) return persistent_ell16_damped_fn<double, MODE_FP64, false>(0);
    if (h->precision == VBD_PRECISION_MIXED)
      return sm ? persistent_ell16_damped_fn<float, MODE_MIXED, true>(h->occ)
                : persistent_ell16_damped_fn<float, MODE_MIXED, false>(h->occ);
    return sm ? persistent_ell16_damped_fn<float, MODE_FP32, true>(h->occ)
              : persistent_ell16_damped_fn<float, MODE_FP32, false>(h->occ);
  }
  if (h->layout == VBD_LAYOUT_ELL16) {
    if (h->precision == VBD_PRECISION_FP64) return persistent_ell16_fn<double, MODE_FP64, false>(0);
    if (h->precision == VBD_PRECISION_MIXED)
      return sm ? persistent_ell16_fn<float, MODE_MIXED, true>(h->occ) : persistent_ell16_fn<float, MODE_MIXED, false>(h->occ);
    return sm ? persistent_ell16_fn<float, MODE_FP32, true>(h->occ) : persistent_ell16_fn<float, MODE_FP32, false>(h->occ);
  }
  if (h->layout == VBD_LAYOUT_ELL) {
    if (h->precision == VBD_PRECISION_FP64) return persistent_ell_fn<double, MODE_FP64, false>(0);
    if (h->precision == VBD_PRECISION_MIXED)
      return sm ? persistent_ell_fn<float, MODE_MIXED, true>(h->occ) : persistent_ell_fn<float, MODE_MIXED, false>(h->occ);
    return sm ? persistent_ell_fn<float, MODE_FP32, true>(h->occ) : persistent_ell_fn<float, MODE_FP32, false>(h->occ);
  }
  if (h->warp_inst) {
    if (h->precision == VBD_PRECISION_FP64) return persistent_warp_fn<double, MODE_FP64, false>(h->soft, h->L);
    if (h->precision == VBD_PRECISION_MIXED)
      return sm ? persistent_warp_fn<float, MODE_MIXED, true>(h->soft, h->L)
                : persistent_warp_fn<float, MODE_MIXED, false>(h->soft, h->L);
    return sm ? persistent_warp_fn<float, MODE_FP32, true>(h->soft, h->L)
              : persistent_warp_fn<float, MODE_FP32, false>(h->soft, h->L);
  }
  if (h->soft) {
    if (h->precision == VBD_PRECISION_FP64) return persistent_soft_fn<double, MODE_FP64, false>(h->L);
    if (h->precision == VBD_PRECISION_MIXED)
      return sm ? persistent_soft_fn<float, MODE_MIXED, true>(h->L) : persistent_soft_fn<float, MODE_MIXED, false>(h->L);
    return sm ? persistent_soft_fn<float, MODE_FP32, true>(h->L) : persistent_soft_fn<float, MODE_FP32, false>(h->L);
  }
  if (h->precision == VBD_PRECISION_FP64) return persistent_fn<double, MODE_FP64, false>(h->L);
  if (h->precision == VBD_PRECISION_MIXED)
    return sm ? persistent_fn<float, MODE_MIXED, true>(h->L) : persistent_fn<float, MODE_MIXED, false>(h->L);
  return sm ? persistent_fn<float, MODE_FP32, true>(h->L) : persistent_fn<float, MODE_FP32, false>(h->L);
}

int occupancy_grid(VbdSolver* h) {
  const void* fn = persistent_kernel(h);
  int dev = 0, sms = 0, per_sm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t dyn = h->smem_bytes;
  if (dyn > 0) CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, h->block, dyn));
  if (per_sm < 1) return VBD_ERR_INVALID_ARGUMENT;
  const int per_cta = h->warp_inst ? h->block / 32 : 1;  // instances a CTA works on at once
  h->grid_persistent = std::min((h->W + per_cta - 1) / per_cta, sms * per_sm);
  return VBD_OK;
}

// The particle-shape contacts of a differentiated substep on the step context (static shapes: no body poses).
template <typename R>
void set_contacts(StepCtx<R>& c, const VbdContactsDesc* contacts) {
  c.has_contacts = 1;
  c.c_count = contacts->soft_contact_count_dev;
  c.c_max = contacts->soft_contact_max;
  c.c_particle = contacts->soft_contact_particle_dev;
  c.c_shape = contacts->soft_contact_shape_dev;
  c.c_body_pos = contacts->soft_contact_body_pos_dev;
  c.c_body_vel = contacts->soft_contact_body_vel_dev;
  c.c_normal = contacts->soft_contact_normal_dev;
}

template <typename R>
int record_impl(VbdSolver* h, const R* q_in, const R* qd_in, const R* f_ext, const VbdContactsDesc* contacts, R dt,
                R* y, R* ck, R* q_out, R* qd_out, cudaStream_t st) {
  const bool has_c = contacts && contacts->soft_contact_max > 0 && contacts->soft_contact_count_dev;
  if (has_c) {
    if (h->prm.avbd_linear_beta != 0.f) return VBD_ERR_UNSUPPORTED;  // the penalty ramp is not differentiated
    int rc = ensure_contact_capacity(h, contacts->soft_contact_max, st);
    if (rc) return rc;
  }
  StepCtx<R> c = make_ctx<R, MODE_FP32>(h);
  if (has_c) set_contacts(c, contacts);
  c.q_in = const_cast<R*>(q_in);
  c.qd_in = qd_in;
  c.f_ext = f_ext;
  c.q_out = q_out;
  c.qd_out = qd_out;
  c.dt = dt;
  c.dt2r = R(1) / (dt * dt);
  const int V = h->V, I = h->prm.iterations;
  const size_t n3 = size_t(3) * V;
  k_record_forward<R><<<(V + 255) / 256, 256, 0, st>>>(c, y);
  if (has_c) {
    CK(cudaMemsetAsync(h->slot_cnt, 0, sizeof(int) * V, st));
    k_contact_prepare<R><<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
  }
  CK(cudaMemcpyAsync(ck, y, n3 * sizeof(R), cudaMemcpyDeviceToDevice, st));
  const int* cp = h->md.color_particles_dev;
  for (int it = 0; it < I; ++it) {
    R* cur = ck + size_t(it + 1) * n3;
    CK(cudaMemcpyAsync(cur, ck + size_t(it) * n3, n3 * sizeof(R), cudaMemcpyDeviceToDevice, st));
    for (size_t col = 0; col + 1 < h->color_offsets.size(); ++col) {
      const int a = h->color_offsets[col], b = h->color_offsets[col + 1];
      if (b > a) k_record_color<R><<<(b - a + 127) / 128, 128, 0, st>>>(c, cur, y, cur, cp + a, b - a);
    }
  }
  k_record_finish<R><<<int((n3 + 255) / 256), 256, 0, st>>>(c, ck + size_t(I) * n3);
  CK(cudaGetLastError());
  return VBD_OK;
}

template <typename R>
int adjoint_impl(VbdSolver* h, const R* q_in, const R* y, const R* ck, const VbdContactsDesc* contacts, R dt,
                 const R* aq_out, const R* aqd_out, R* aq_in, R* aqd_in, R* adj_mu, R* adj_lambda, cudaStream_t st) {
  const int V = h->V, I = h->prm.iterations, C = int(h->color_offsets.size()) - 1;
  const size_t n3 = size_t(3) * V;
  const bool has_c = contacts && contacts->soft_contact_max > 0 && contacts->soft_contact_count_dev;
  if (has_c) {
    if (h->prm.avbd_linear_beta != 0.f) return VBD_ERR_UNSUPPORTED;
    int rc = ensure_contact_capacity(h, contacts->soft_contact_max, st);
    if (rc) return rc;
  }
  const size_t need = (size_t(std::max(C, 1)) + 3) * n3 * sizeof(R);
  if (h->adj_work_bytes < need) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return VBD_ERR_UNSUPPORTED;
    if (h->adj_work) cudaFree(h->adj_work);
    h->adj_work = nullptr;
    h->adj_work_bytes = 0;
    int rc = dalloc((char**)&h->adj_work, need);
    if (rc) return rc;
    h->adj_work_bytes = need;
  }
  R* S = (R*)h->adj_work;  // C color-start states
  R* ax = S + size_t(std::max(C, 1)) * n3;
  R* ay = ax + n3;
  R* axp = ay + n3;
  StepCtx<R> c = make_ctx<R, MODE_FP32>(h);
  if (has_c) set_contacts(c, contacts);
  c.q_in = const_cast<R*>(q_in);
  c.dt = dt;
  c.dt2r = R(1) / (dt * dt);
  k_adjoint_begin<R><<<int((n3 + 255) / 256), 256, 0, st>>>(int(n3), aq_out, aqd_out, R(1) / dt, ax, ay);
  // this substep's start positions (damping and contact terms) and contact table, as its forward pass had them
  k_adjoint_qprev<R><<<(V + 255) / 256, 256, 0, st>>>(c);
  CK(cudaMemsetAsync(axp, 0, n3 * sizeof(R), st));
  if (has_c) {
    CK(cudaMemsetAsync(h->slot_cnt, 0, sizeof(int) * V, st));
    k_contact_prepare<R><<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
  }
  AdjCtx<R> A{c, nullptr, y, ax, ay, adj_mu, adj_lambda, axp};
  const int* cp = h->md.color_particles_dev;
  for (int it = I - 1; it >= 0; --it) {
    CK(cudaMemcpyAsync(S, ck + size_t(it) * n3, n3 * sizeof(R), cudaMemcpyDeviceToDevice, st));
    for (int col = 0; col + 1 < C; ++col) {
      R* nxt = S + size_t(col + 1) * n3;
      CK(cudaMemcpyAsync(nxt, S + size_t(col) * n3, n3 * sizeof(R), cudaMemcpyDeviceToDevice, st));
      const int a = h->color_offsets[col], b = h->color_offsets[col + 1];
      if (b > a) k_record_color<R><<<(b - a + 127) / 128, 128, 0, st>>>(c, nxt, y, nxt, cp + a, b - a);
    }
    for (int col = C - 1; col >= 0; --col) {
      A.x = S + size_t(col) * n3;
      const int a = h->color_offsets[col], b = h->color_offsets[col + 1];
      if (b > a) k_adjoint_color<R><<<(b - a + 63) / 64, 64, 0, st>>>(A, cp + a, b - a);
    }
  }
  k_adjoint_end<R><<<(V + 255) / 256, 256, 0, st>>>(c, ax, ay, axp, aqd_out, aq_in, aqd_in);
  CK(cudaGetLastError());
  return VBD_OK;
}

// Greedy coloring of a graph given as (min, max) pairs (deduplicated here), then the balancing pass.
// algorithm 1 (ordered greedy, Ton-That et al. 2023): vertices by decreasing degree, ties by index.
// algorithm 0 (MCS, Pereira & Palsberg 2005): the maximum cardinality search order, each step taking the
// unvisited vertex with the most visited neighbours (ties: lowest index); optimal on chordal graphs and
// typically fewer colors on meshes. Either way each vertex takes the lowest color its colored neighbours leave.
int color_pairs(int V, std::vector<uint64_t>& pairs, float target_ratio, int32_t* colors, int algorithm = 1) {
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  std::vector<int> off(V + 1, 0);
  for (uint64_t p : pairs) {
    off[int(p >> 32) + 1]++;
    off[int(p & 0xffffffffu) + 1]++;
  }
  for (int i = 0; i < V; ++i) off[i + 1] += off[i];
  std::vector<int> nb(off[V]), fill(off.begin(), off.end() - 1);
  for (uint64_t p : pairs) {
    const int a = int(p >> 32), b = int(p & 0xffffffffu);
    nb[fill[a]++] = b;
    nb[fill[b]++] = a;
  }
  std::vector<int> order(V);
  if (algorithm == 0) {
    // maximum cardinality search with a lazy max-heap of (weight, -vertex)
    std::vector<int> weight(V, 0);
    std::vector<char> seen(V, 0);
    std::priority_queue<std::pair<int, int>> heap;
    for (int v = 0; v < V; ++v) heap.push({0, -v});
    int k = 0;
    while (!heap.empty()) {
      const auto top = heap.top();
      heap.pop();
      const int v = -top.second;
      if (seen[v] || top.first != weight[v]) continue;
      seen[v] = 1;
      order[k++] = v;
      for (int j = off[v]; j < off[v + 1]; ++j)
        if (!seen[nb[j]]) heap.push({++weight[nb[j]], -nb[j]});
    }
  } else {
    // degree-ordered greedy (largest degree first, ties by index)
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return off[a + 1] - off[a] > off[b + 1] - off[b]; });
  }
  std::fill(colors, colors + V, -1);
  std::vector<int> mark;
  int ncol = 0;
  for (int v : order) {
    for (int k = off[v]; k < off[v + 1]; ++k) {
      const int c = colors[nb[k]];
      if (c >= 0) {
        if (c >= int(mark.size())) mark.resize(c + 1, -1);
        mark[c] = v;
      }
    }
    int c = 0;
    while (c < int(mark.size()) && mark[c] == v) ++c;
    colors[v] = c;
    ncol = std::max(ncol, c + 1);
  }
  // balancing: move vertices from the largest color to the smallest admissible one
  if (ncol > 1 && target_ratio > 1.f) {
    std::vector<int> size(ncol, 0);
    for (int v = 0; v < V; ++v) size[colors[v]]++;
    for (int round = 0; round < 4 * ncol; ++round) {
      const int cmax = int(std::max_element(size.begin(), size.end()) - size.begin());
      const int cmin = int(std::min_element(size.begin(), size.end()) - size.begin());
      if (size[cmin] > 0 && float(size[cmax]) / float(size[cmin]) <= target_ratio) break;
      bool moved = false;
      for (int v = 0; v < V && size[cmax] - size[cmin] > 1; ++v) {
        if (colors[v] != cmax) continue;
        bool ok = true;
        for (int k = off[v]; k < off[v + 1] && ok; ++k) ok = colors[nb[k]] != cmin;
        if (ok) {
          colors[v] = cmin;
          size[cmax]--;
          size[cmin]++;
          moved = true;
        }
      }
      if (!moved) break;
    }
  }
  return ncol;
}

}  // namespace

extern "C" {

int vbd_create(const VbdModelDesc* model, const VbdSolverParams* params, VbdHandle* out) {
  if (!model || !params || !out) return VBD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const VbdModelDesc& m = *model;
  if (m.particle_count <= 0 || m.tri_count < 0 || m.edge_count < 0 || m.shape_count < 0)
    return VBD_ERR_INVALID_ARGUMENT;
  if (m.color_count <= 0 || !m.color_offsets_host || !m.color_particles_dev) return VBD_ERR_EMPTY_COLORING;
  if (params->iterations < 0) return VBD_ERR_INVALID_ARGUMENT;
  if (params->precision < 0 || params->precision > 2) return VBD_ERR_INVALID_ARGUMENT;
  const int lpv = params->lanes_per_vertex;
  if (lpv != 0 && lpv != 1 && lpv != 2 && lpv != 4 && lpv != 8 && lpv != 16 && lpv != 32)
    return VBD_ERR_INVALID_ARGUMENT;
  if (params->block_size != 0 && (params->block_size < 32 || params->block_size > 1024 || params->block_size % 32))
    return VBD_ERR_INVALID_ARGUMENT;
  if (params->contact_slots < 0 || params->contact_slots > 8) return VBD_ERR_INVALID_ARGUMENT;
  if (m.color_offsets_host[0] != 0 || m.color_offsets_host[m.color_count] != m.particle_count)
    return VBD_ERR_INVALID_ARGUMENT;
  for (int c = 0; c < m.color_count; ++c)
    if (m.color_offsets_host[c + 1] < m.color_offsets_host[c]) return VBD_ERR_INVALID_ARGUMENT;
  if (!m.particle_mass_dev || !m.particle_inv_mass_dev || !m.particle_flags_dev || !m.particle_radius_dev ||
      !m.gravity_dev)
    return VBD_ERR_INVALID_ARGUMENT;
  if (m.tri_count > 0 && (!m.tri_indices_dev || !m.tri_poses_dev || !m.tri_materials_dev || !m.tri_areas_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  if (m.edge_count > 0 && (!m.edge_indices_dev || !m.edge_rest_angle_dev || !m.edge_rest_length_dev ||
                           !m.edge_bending_properties_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  if (m.shape_count > 0 &&
      (!m.shape_material_ke_dev || !m.shape_material_kd_dev || !m.shape_material_mu_dev || !m.shape_body_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  if (m.spring_count < 0 || m.tet_count < 0) return VBD_ERR_INVALID_ARGUMENT;
  if (m.spring_count > 0 && (!m.spring_indices_dev || !m.spring_rest_length_dev || !m.spring_stiffness_dev ||
                             !m.spring_damping_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  if (m.tet_count > 0 && (!m.tet_indices_dev || !m.tet_poses_dev || !m.tet_materials_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  if (m.tri_count >= (1 << 29) || m.edge_count >= (1 << 29) || m.tet_count >= (1 << 29) ||
      m.spring_count >= (1 << 30))
    return VBD_ERR_UNSUPPORTED;
  const bool soft = m.spring_count > 0 || m.tet_count > 0;
  if (soft && (params->layout == VBD_LAYOUT_ELL || params->layout == VBD_LAYOUT_ELL16 ||
               params->layout == VBD_LAYOUT_RING))
    return VBD_ERR_UNSUPPORTED;

  VbdSolver* h = new (std::nothrow) VbdSolver();
  if (!h) return VBD_ERR_OUT_OF_MEMORY;
  h->md = m;
  h->prm = *params;
  h->V = m.particle_count;
  h->T = m.tri_count;
  h->E = m.edge_count;
  h->S = m.shape_count;
  h->NS = m.spring_count;
  h->NT = m.tet_count;
  h->soft = soft;
  h->precision = params->precision;
  h->K = params->contact_slots > 0 ? params->contact_slots : std::max(1, std::min(8, m.shape_count));
  h->color_offsets.assign(m.color_offsets_host, m.color_offsets_host + m.color_count + 1);
  int rc = VBD_OK;
  auto fail = [&](int code) {
    delete h;
    return code;
  };

  // host copies of the topology for the adjacency and the instance plan (one-time)
  std::vector<int> tri(3 * size_t(h->T)), edges(4 * size_t(h->E)), colp(h->V);
  if (h->T && cudaMemcpy(tri.data(), m.tri_indices_dev, tri.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(VBD_ERR_CUDA);
  if (h->E && cudaMemcpy(edges.data(), m.edge_indices_dev, edges.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(VBD_ERR_CUDA);
  if (cudaMemcpy(colp.data(), m.color_particles_dev, size_t(h->V) * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(VBD_ERR_CUDA);
  for (int t : tri)
    if (t < 0 || t >= h->V) return fail(VBD_ERR_INVALID_ARGUMENT);
  for (size_t i = 0; i < edges.size(); ++i)
    if (edges[i] >= h->V || (edges[i] < 0 && (i % 4) >= 2) || edges[i] < -1) return fail(VBD_ERR_INVALID_ARGUMENT);
  for (int p : colp)
    if (p < 0 || p >= h->V) return fail(VBD_ERR_INVALID_ARGUMENT);
  std::vector<int> springs(2 * size_t(h->NS)), tets(4 * size_t(h->NT));
  if (h->NS && cudaMemcpy(springs.data(), m.spring_indices_dev, springs.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(VBD_ERR_CUDA);
  if (h->NT && cudaMemcpy(tets.data(), m.tet_indices_dev, tets.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(VBD_ERR_CUDA);
  for (int i : springs)
    if (i < 0 || i >= h->V) return fail(VBD_ERR_INVALID_ARGUMENT);
  for (int i : tets)
    if (i < 0 || i >= h->V) return fail(VBD_ERR_INVALID_ARGUMENT);

  std::vector<int> foff, fadj, eoff, eadj;
  build_packed_adjacency(h->V, h->T, tri.data(), h->E, edges.data(), foff, fadj, eoff, eadj);
  h->h_tri = tri;
  h->h_edges = edges;
  h->h_foff = foff;
  h->h_fadj = fadj;
  h->h_eoff = eoff;
  h->h_eadj = eadj;
  if ((rc = upload(&h->face_off, foff)) || (rc = upload(&h->face_adj, fadj)) || (rc = upload(&h->edge_off, eoff)) ||
      (rc = upload(&h->edge_adj, eadj)))
    return fail(rc);
  if ((rc = dalloc(&h->tri_idx, h->T)) || (rc = dalloc(&h->tri_pose, h->T)) || (rc = dalloc(&h->tri_mat, h->T)) ||
      (rc = dalloc(&h->edge_idx, h->E)) || (rc = dalloc(&h->edge_prop, h->E)))
    return fail(rc);
  if (soft) {
    std::vector<int> color_of(h->V, -1);
    for (size_t col = 0; col + 1 < h->color_offsets.size(); ++col)
      for (int k = h->color_offsets[col]; k < h->color_offsets[col + 1]; ++k) color_of[colp[k]] = int(col);
    std::vector<int> toff, tadj, soff, sadj, ssoff, ssadj;
    build_soft_adjacency(h->V, h->NT, tets.data(), h->NS, springs.data(), color_of, toff, tadj, soff, sadj, ssoff,
                         ssadj);
    h->n_same_springs = ssoff[h->V];
    const size_t racc = h->precision == VBD_PRECISION_FP64 ? sizeof(double) : sizeof(float);
    if ((rc = upload(&h->tet_off, toff)) || (rc = upload(&h->tet_adj, tadj)) || (rc = upload(&h->spr_off, soff)) ||
        (rc = upload(&h->spr_adj, sadj)) || (rc = upload(&h->sspr_off, ssoff)) || (rc = upload(&h->sspr_adj, ssadj)) ||
        (rc = dalloc(&h->spr_idx, std::max(h->NS, 1))) || (rc = dalloc(&h->spr_prop, std::max(h->NS, 1))) ||
        (rc = dalloc(&h->tet_idx, std::max(h->NT, 1))) || (rc = dalloc(&h->tet_pose, 3 * size_t(std::max(h->NT, 1)))))
      return fail(rc);
    if (h->n_same_springs && (rc = dalloc((char**)&h->spr_acc, racc * 9 * size_t(h->V)))) return fail(rc);
  }
  if ((rc = pack_model(h, 0))) return fail(rc);

  // instances (worlds)
  std::vector<int> wstart;
  if (m.world_count > 1 && m.world_particle_start_host) {
    wstart.assign(m.world_particle_start_host, m.world_particle_start_host + m.world_count + 1);
    if (wstart[0] != 0 || wstart.back() != h->V) return fail(VBD_ERR_INVALID_ARGUMENT);
    for (int w = 0; w < m.world_count; ++w)
      if (wstart[w + 1] < wstart[w]) return fail(VBD_ERR_INVALID_ARGUMENT);
  } else {
    wstart = {0, h->V};
  }
  h->W = int(wstart.size()) - 1;
  std::vector<int> world_of(h->V);
  for (int w = 0; w < h->W; ++w)
    for (int i = wstart[w]; i < wstart[w + 1]; ++i) world_of[i] = w;
  for (int t = 0; t < h->T; ++t)
    if (world_of[tri[3 * t]] != world_of[tri[3 * t + 1]] || world_of[tri[3 * t]] != world_of[tri[3 * t + 2]])
      return fail(VBD_ERR_INVALID_ARGUMENT);
  for (int e = 0; e < h->E; ++e)
    for (int j = 0; j < 4; ++j)
      if (edges[4 * e + j] >= 0 && world_of[edges[4 * e + j]] != world_of[edges[4 * e + 2]])
        return fail(VBD_ERR_INVALID_ARGUMENT);
  for (int k = 0; k < h->NS; ++k)
    if (world_of[springs[2 * k]] != world_of[springs[2 * k + 1]]) return fail(VBD_ERR_INVALID_ARGUMENT);
  for (int t = 0; t < h->NT; ++t)
    for (int j = 1; j < 4; ++j)
      if (world_of[tets[4 * t + j]] != world_of[tets[4 * t]]) return fail(VBD_ERR_INVALID_ARGUMENT);
  // per instance, per global color (in sweep order), the instance's particles of that color
  std::vector<std::vector<std::vector<int>>> per(h->W);
  for (size_t col = 0; col + 1 < h->color_offsets.size(); ++col) {
    for (int w = 0; w < h->W; ++w) per[w].emplace_back();
    for (int k = h->color_offsets[col]; k < h->color_offsets[col + 1]; ++k) per[world_of[colp[k]]][col].push_back(colp[k]);
  }
  std::vector<int> cptr(h->W + 1, 0), ranges, verts;
  for (int w = 0; w < h->W; ++w) {
    cptr[w] = int(ranges.size());
    for (auto& g : per[w]) {
      if (g.empty()) continue;
      ranges.push_back(int(verts.size()));
      verts.insert(verts.end(), g.begin(), g.end());
    }
    ranges.push_back(int(verts.size()));
  }
  cptr[h->W] = int(ranges.size());
  // instance w's ranges are ranges[cptr[w] .. cptr[w+1]-1]; the kernel walks col in [cb, ce-1)
  std::vector<int> order(h->W);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return wstart[a + 1] - wstart[a] > wstart[b + 1] - wstart[b]; });
  if ((rc = upload(&h->inst_order, order)) || (rc = upload(&h->inst_vstart, wstart)) ||
      (rc = upload(&h->inst_cptr, cptr)) || (rc = upload(&h->color_ranges, ranges)) ||
      (rc = upload(&h->color_verts, verts)) || (rc = dalloc(&h->queue, 1)))
    return fail(rc);

  // scratch
  const size_t p4 = h->precision == VBD_PRECISION_FP64 ? sizeof(double4) : sizeof(float4);
  if ((rc = dalloc((char**)&h->pos, p4 * h->V)) || (rc = dalloc((char**)&h->qprev, p4 * h->V)) ||
      (rc = dalloc((char**)&h->inertia, p4 * h->V)) || (rc = dalloc(&h->slot_cnt, h->V)) ||
      (rc = dalloc(&h->slots, size_t(h->V) * h->K)) || (rc = dalloc(&h->err, 1)) ||
      (rc = dalloc(&h->residual, size_t(std::max(params->iterations, 1)) * 32)))
    return fail(rc);
  if (cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess || cudaMemset(h->slot_cnt, 0, sizeof(int) * h->V) != cudaSuccess)
    return fail(VBD_ERR_CUDA);

  // scheduling
  h->schedule = params->schedule;
  if (h->schedule == VBD_SCHEDULE_AUTO) h->schedule = (h->W > 1 || h->V <= 4096) ? VBD_SCHEDULE_PERSISTENT : VBD_SCHEDULE_PER_COLOR;
  // default lanes per vertex: 8 for one persistent instance and for models with tetrahedra or springs (a
  // vertex of a tet mesh has ~11 incident tets; 8 lanes measured fastest on 4,096 blocks of 640 tets: 5.3 ms
  // per substep against 19.1 / 10.0 / 6.1 / 6.8 ms with 1 / 2 / 4 / 16), else 1 (one lane per stencil row)
  const bool stencil_asked = params->layout == VBD_LAYOUT_ELL || params->layout == VBD_LAYOUT_ELL16 ||
                             params->layout == VBD_LAYOUT_RING;
  h->L = lpv ? lpv : (((h->schedule == VBD_SCHEDULE_PERSISTENT && h->W == 1 && !stencil_asked) || soft) ? 8 : 1);
  for (int w = 0; w < h->W; ++w) h->max_inst_v = std::max(h->max_inst_v, wstart[w + 1] - wstart[w]);
  if (h->schedule == VBD_SCHEDULE_PERSISTENT && h->precision != VBD_PRECISION_FP64 &&
      params->positions_in_shared != 1) {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      return fail(VBD_ERR_CUDA);
    const size_t need = size_t(12) * h->max_inst_v;
    if (need + 64 <= size_t(optin)) h->smem_bytes = need;
    else if (params->positions_in_shared == 2) return fail(VBD_ERR_UNSUPPORTED);
  } else if (params->positions_in_shared == 2) {
    return fail(VBD_ERR_UNSUPPORTED);
  }
  h->block = params->block_size ? params->block_size
                                : (h->schedule == VBD_SCHEDULE_PERSISTENT ? (h->smem_bytes > 96 * 1024 ? 512 : 256) : 128);
  // element data layout: stencil records (one thread per vertex) unless lanes per vertex > 1 asks for CSR;
  // the compact 16-bit records when the persistent schedule runs instances below 65536 particles and no
  // hinge carries damping
  if ((params->layout == VBD_LAYOUT_ELL || params->layout == VBD_LAYOUT_ELL16 || params->layout == VBD_LAYOUT_RING) &&
      h->L != 1)
    return fail(VBD_ERR_INVALID_ARGUMENT);
  bool any_hinge_damping = false, lnh_floor = false;
  {
    std::vector<float> bp, tm;
    if (h->E && (rc = download(bp, m.edge_bending_properties_dev, size_t(2) * h->E))) return fail(rc);
    for (int e = 0; e < h->E; ++e) any_hinge_damping |= bp[2 * e] > 0.f && bp[2 * e + 1] > 0.f;
    if (h->T && (rc = download(tm, m.tri_materials_dev, size_t(5) * h->T))) return fail(rc);
    lnh_floor = needs_lnh_floor(tm, h->T);
  }
  if (lnh_floor && (params->layout == VBD_LAYOUT_ELL || params->layout == VBD_LAYOUT_ELL16 ||
                    params->layout == VBD_LAYOUT_RING))
    return fail(VBD_ERR_UNSUPPORTED);
  const bool ell16_ok = h->schedule == VBD_SCHEDULE_PERSISTENT && h->max_inst_v < 65536;
  if (params->layout == VBD_LAYOUT_ELL16 && !ell16_ok) return fail(VBD_ERR_UNSUPPORTED);
  if (params->layout == VBD_LAYOUT_RING && !ell16_ok) return fail(VBD_ERR_UNSUPPORTED);
  if (params->layout == VBD_LAYOUT_CSR || h->L != 1 || h->soft || lnh_floor)
    h->layout = VBD_LAYOUT_CSR;
  else if (params->layout == VBD_LAYOUT_RING)
    h->layout = VBD_LAYOUT_RING;
  else if (params->layout == VBD_LAYOUT_ELL16 || (params->layout == VBD_LAYOUT_AUTO && ell16_ok))
    h->layout = VBD_LAYOUT_ELL16;
  else
    h->layout = VBD_LAYOUT_ELL;
  h->inst_start_of_vertex.assign(h->V, 0);
  for (int w = 0; w < h->W; ++w)
    for (int i = wstart[w]; i < wstart[w + 1]; ++i) h->inst_start_of_vertex[i] = wstart[w];
  if ((h->layout == VBD_LAYOUT_ELL || h->layout == VBD_LAYOUT_ELL16 || h->layout == VBD_LAYOUT_RING) &&
      h->schedule == VBD_SCHEDULE_PERSISTENT && h->block > 512)
    return fail(VBD_ERR_INVALID_ARGUMENT);
  if (params->min_blocks_per_sm != 0) {
    // the kernel is compiled for min_blocks_per_sm CTAs of 256 threads (its register budget); CTAs of 128 threads
    // run twice as many instances side by side on an SM under the same budget
    if (params->min_blocks_per_sm < 2 || params->min_blocks_per_sm > 4 ||
        (h->layout != VBD_LAYOUT_ELL && h->layout != VBD_LAYOUT_ELL16 && h->layout != VBD_LAYOUT_RING) ||
        h->schedule != VBD_SCHEDULE_PERSISTENT || h->precision == VBD_PRECISION_FP64 ||
        (params->block_size != 0 && params->block_size != 256 && params->block_size != 128))
      return fail(VBD_ERR_INVALID_ARGUMENT);
    h->occ = params->min_blocks_per_sm;
    h->block = params->block_size ? params->block_size : 256;
  }
  if (h->layout == VBD_LAYOUT_ELL || h->layout == VBD_LAYOUT_ELL16 || h->layout == VBD_LAYOUT_RING) {
    if (h->schedule == VBD_SCHEDULE_PERSISTENT) {
      h->range_verts_host = verts;
      h->ranges_host.clear();
      for (int w = 0; w < h->W; ++w)
        for (int k = cptr[w]; k + 1 < cptr[w + 1]; ++k) h->ranges_host.push_back(ranges[k]);
      h->ranges_host.push_back(int(verts.size()));
    } else {
      h->range_verts_host = colp;
      h->ranges_host = h->color_offsets;
    }
    if ((rc = h->layout == VBD_LAYOUT_RING ? build_ring(h) : build_ell(h))) return fail(rc);
  }
  if (params->instance_per_warp != 0) {
    // one warp per instance: CSR layout, persistent schedule, lanes per vertex 1..8, whole warps per block
    if (params->instance_per_warp != 1 || h->schedule != VBD_SCHEDULE_PERSISTENT || h->layout != VBD_LAYOUT_CSR ||
        (h->L != 1 && h->L != 2 && h->L != 4 && h->L != 8) || h->occ != 0 || params->pair_vertices != 0)
      return fail(VBD_ERR_INVALID_ARGUMENT);
    h->warp_inst = true;
    h->block = params->block_size ? params->block_size : 256;
    h->smem_bytes = 0;
    h->slice = 0;
    if (h->precision != VBD_PRECISION_FP64 && params->positions_in_shared != 1) {
      int dev = 0, optin = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return fail(VBD_ERR_CUDA);
      const size_t need = size_t(h->block / 32) * 12 * size_t(h->max_inst_v);
      if (need > 0 && need + 64 <= size_t(optin)) {
        h->smem_bytes = need;
        h->slice = 3 * h->max_inst_v;
      } else if (params->positions_in_shared == 2) {
        return fail(VBD_ERR_UNSUPPORTED);
      }
    }
  }
  if (params->pair_vertices != 0) {
    if (params->pair_vertices != 1 || h->layout != VBD_LAYOUT_ELL16 || h->schedule != VBD_SCHEDULE_PERSISTENT ||
        h->precision != VBD_PRECISION_FP32)
      return fail(VBD_ERR_INVALID_ARGUMENT);
    if (any_hinge_damping) return fail(VBD_ERR_UNSUPPORTED);  // the paired bending has no damping term
    h->pair = true;
  }
  if (h->schedule == VBD_SCHEDULE_PERSISTENT && (rc = occupancy_grid(h))) return fail(rc);
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(VBD_ERR_CUDA);
  *out = h;
  return VBD_OK;
}

int vbd_refresh_model(VbdHandle h, void* stream) {
  if (!h) return VBD_ERR_INVALID_ARGUMENT;
  int rc = pack_model(h, (cudaStream_t)stream);
  if (rc) return rc;
  if (h->pair && h->E) {  // the paired kernel has no hinge damping term
    std::vector<float> bp;
    if ((rc = download(bp, h->md.edge_bending_properties_dev, size_t(2) * h->E))) return rc;
    for (int e = 0; e < h->E; ++e)
      if (bp[2 * e] > 0.f && bp[2 * e + 1] > 0.f) return VBD_ERR_UNSUPPORTED;
  }
  if (h->layout == VBD_LAYOUT_ELL || h->layout == VBD_LAYOUT_ELL16 || h->layout == VBD_LAYOUT_RING) {
    if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return VBD_ERR_CUDA;
    if (h->layout == VBD_LAYOUT_RING) {
      for (void** p : {(void**)&h->ring_nslot, (void**)&h->ring_base, (void**)&h->ring_vbase, (void**)&h->ring_A,
                       (void**)&h->ring_B, (void**)&h->ring_H, (void**)&h->ring_hdr}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
      }
      return build_ring(h);
    }
    return build_ell(h);
  }
  return VBD_OK;
}

int vbd_step(VbdHandle h, float* q_in, float* q_out, const float* qd_in, float* qd_out, const float* f_ext,
             const VbdContactsDesc* contacts, const VbdBodyState* bodies, float dt, void* stream) {
  if (!h) return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (h->precision == VBD_PRECISION_FP64) return VBD_ERR_INVALID_ARGUMENT;
  if (h->precision == VBD_PRECISION_MIXED)
    return step_impl<float, MODE_MIXED>(h, q_in, q_out, qd_in, qd_out, f_ext, contacts, bodies, dt, st);
  return step_impl<float, MODE_FP32>(h, q_in, q_out, qd_in, qd_out, f_ext, contacts, bodies, dt, st);
}

int vbd_step_f64(VbdHandle h, double* q_in, double* q_out, const double* qd_in, double* qd_out, const double* f_ext,
                 const VbdContactsDesc* contacts, const VbdBodyState* bodies, double dt, void* stream) {
  if (!h) return VBD_ERR_INVALID_ARGUMENT;
  if (h->precision != VBD_PRECISION_FP64) return VBD_ERR_INVALID_ARGUMENT;
  return step_impl<double, MODE_FP64>(h, q_in, q_out, qd_in, qd_out, f_ext, contacts, bodies, dt,
                                      (cudaStream_t)stream);
}

int vbd_record_step(VbdHandle h, const void* q_in, const void* qd_in, const void* particle_f,
                    const VbdContactsDesc* contacts, double dt, void* y, void* checkpoints, void* q_out, void* qd_out,
                    void* stream) {
  if (!h || !q_in || !qd_in || !y || !checkpoints || !q_out || !qd_out || !(dt > 0.0)) return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (h->precision == VBD_PRECISION_FP64)
    return record_impl<double>(h, (const double*)q_in, (const double*)qd_in, (const double*)particle_f, contacts, dt,
                               (double*)y, (double*)checkpoints, (double*)q_out, (double*)qd_out, st);
  return record_impl<float>(h, (const float*)q_in, (const float*)qd_in, (const float*)particle_f, contacts,
                            float(dt), (float*)y, (float*)checkpoints, (float*)q_out, (float*)qd_out, st);
}

int vbd_adjoint_step(VbdHandle h, const void* q_in, const void* y, const void* checkpoints,
                     const VbdContactsDesc* contacts, double dt, const void* adj_q_out, const void* adj_qd_out,
                     void* adj_q_in, void* adj_qd_in, void* adj_tri_mu, void* adj_tri_lambda, void* stream) {
  if (!h || !q_in || !y || !checkpoints || !adj_q_in || !(dt > 0.0)) return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (h->precision == VBD_PRECISION_FP64)
    return adjoint_impl<double>(h, (const double*)q_in, (const double*)y, (const double*)checkpoints, contacts, dt,
                                (const double*)adj_q_out, (const double*)adj_qd_out, (double*)adj_q_in,
                                (double*)adj_qd_in, (double*)adj_tri_mu, (double*)adj_tri_lambda, st);
  return adjoint_impl<float>(h, (const float*)q_in, (const float*)y, (const float*)checkpoints, contacts, float(dt),
                             (const float*)adj_q_out, (const float*)adj_qd_out, (float*)adj_q_in, (float*)adj_qd_in,
                             (float*)adj_tri_mu, (float*)adj_tri_lambda, st);
}

int vbd_get_error(VbdHandle h, int32_t* bits, void* stream) {
  if (!h || !bits) return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(bits, h->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemsetAsync(h->err, 0, sizeof(int), st));
  CK(cudaStreamSynchronize(st));
  return VBD_OK;
}

int vbd_get_residuals(VbdHandle h, double* out, int32_t n, void* stream) {
  if (!h || !out || n < 0 || n > std::max(h->prm.iterations, 1)) return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) return VBD_OK;
  double buf[32];
  for (int i = 0; i < n; ++i) {
    CK(cudaMemcpyAsync(buf, h->residual + size_t(i) * 32, sizeof(buf), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double acc = 0.0;
    for (double b : buf) acc += b;
    out[i] = acc;
  }
  return VBD_OK;
}

int vbd_launches_per_step(VbdHandle h, int32_t* out) {
  if (!h || !out) return VBD_ERR_INVALID_ARGUMENT;
  const int C = int(h->color_offsets.size()) - 1, I = h->prm.iterations;
  if (h->schedule == VBD_SCHEDULE_PERSISTENT) {
    *out = 1 + (h->S > 0 ? 1 : 0);
  } else if (h->sc_on) {
    // kernels of this library per detection: 1 copy + per primitive kind (boxes, cell, count, fill, query)
    // + compaction (2 x (stored, pairs) + entry count, fill, sort); the six cub scans are not counted
    const int detect = 1 + 2 * 5 + 4 + 3;
    int n_det = 1;
    for (int it = 0; it < I; ++it)
      if ((h->sc_interval == 0 && it == 0) || (h->sc_interval >= 1 && it % h->sc_interval == 0)) ++n_det;
    const bool duals = h->S > 0 && h->prm.avbd_linear_beta != 0.f;
    *out = 2 + (h->S > 0 ? 1 : 0) + n_det * detect + 2 + I * (C * (h->n_same_springs ? 4 : 3) + (duals ? 1 : 0));
  } else {
    *out = 2 + (h->S > 0 ? 1 : 0) + I * C * (h->n_same_springs ? 2 : 1);
  }
  return VBD_OK;
}

int vbd_get_config(VbdHandle h, int32_t* schedule, int32_t* lanes, int32_t* block, int32_t* shared_bytes,
                   int32_t* layout) {
  if (!h) return VBD_ERR_INVALID_ARGUMENT;
  if (layout) *layout = h->layout;
  if (schedule) *schedule = h->schedule;
  if (lanes) *lanes = h->L;
  if (block) *block = h->block;
  if (shared_bytes) *shared_bytes = int32_t(h->smem_bytes);
  return VBD_OK;
}

int vbd_destroy(VbdHandle h) {
  if (!h) return VBD_ERR_INVALID_ARGUMENT;
  cudaDeviceSynchronize();
  delete h;
  return VBD_OK;
}

int vbd_build_adjacency(int32_t V, int32_t T, const int32_t* tri, int32_t E, const int32_t* edges, int32_t* foff,
                        int32_t* faces, int32_t* eoff, int32_t* eadj) {
  if (V < 0 || T < 0 || E < 0 || (T && !tri) || (E && !edges) || !foff || !eoff) return VBD_ERR_INVALID_ARGUMENT;
  std::vector<int> cnt(V, 0), fill(V, 0);
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 3; ++j) {
      if (tri[3 * t + j] < 0 || tri[3 * t + j] >= V) return VBD_ERR_INVALID_ARGUMENT;
      cnt[tri[3 * t + j]]++;
    }
  foff[0] = 0;
  for (int i = 0; i < V; ++i) foff[i + 1] = foff[i] + 2 * cnt[i];
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 3; ++j) {
      const int v = tri[3 * t + j];
      const int o = foff[v] + 2 * fill[v]++;
      faces[o] = t;
      faces[o + 1] = j;
    }
  std::fill(cnt.begin(), cnt.end(), 0);
  std::fill(fill.begin(), fill.end(), 0);
  for (int e = 0; e < E; ++e) {
    const int* ei = edges + 4 * e;
    for (int j = 0; j < 4; ++j)
      if (ei[j] >= V || (ei[j] < 0 && (j >= 2 || ei[j] != -1))) return VBD_ERR_INVALID_ARGUMENT;
    cnt[ei[2]]++;
    cnt[ei[3]]++;
    if (ei[0] != -1) cnt[ei[0]]++;
    if (ei[1] != -1) cnt[ei[1]]++;
  }
  eoff[0] = 0;
  for (int i = 0; i < V; ++i) eoff[i + 1] = eoff[i] + 2 * cnt[i];
  auto put = [&](int v, int e, int order) {
    const int o = eoff[v] + 2 * fill[v]++;
    eadj[o] = e;
    eadj[o + 1] = order;
  };
  for (int e = 0; e < E; ++e) {
    const int* ei = edges + 4 * e;
    put(ei[2], e, 2);
    put(ei[3], e, 3);
    if (ei[0] != -1) put(ei[0], e, 0);
    if (ei[1] != -1) put(ei[1], e, 1);
  }
  return VBD_OK;
}

int vbd_color_graph(int32_t V, int32_t pair_count, const int32_t* pairs_host, int32_t algorithm, float target_ratio,
                    int32_t* colors) {
  if (V < 0 || pair_count < 0 || (pair_count && !pairs_host) || !colors || algorithm < 0 || algorithm > 1)
    return VBD_ERR_INVALID_ARGUMENT;
  if (V == 0) return 0;
  std::vector<uint64_t> pairs;
  pairs.reserve(pair_count);
  for (int k = 0; k < pair_count; ++k) {
    int a = pairs_host[2 * k], b = pairs_host[2 * k + 1];
    if (a < 0 || b < 0 || a >= V || b >= V) return VBD_ERR_INVALID_ARGUMENT;
    if (a == b) continue;
    if (a > b) std::swap(a, b);
    pairs.push_back((uint64_t(uint32_t(a)) << 32) | uint32_t(b));
  }
  return color_pairs(V, pairs, target_ratio, colors, algorithm);
}

int vbd_color_particles(int32_t V, int32_t T, const int32_t* tri, const float* tri_mat, int32_t E,
                        const int32_t* edges, const float* edge_props, int32_t include_bending, float target_ratio,
                        int32_t* colors) {
  if (V < 0 || T < 0 || E < 0 || !colors) return VBD_ERR_INVALID_ARGUMENT;
  if (V == 0) return 0;
  // graph edges as (min, max) pairs, deduplicated (graph_coloring.py:45-51, 99-236)
  std::vector<uint64_t> pairs;
  pairs.reserve(size_t(3) * T + (include_bending ? size_t(6) * E : 0));
  auto add = [&](int a, int b) {
    if (a < 0 || b < 0 || a == b) return;
    if (a > b) std::swap(a, b);
    pairs.push_back((uint64_t(uint32_t(a)) << 32) | uint32_t(b));
  };
  for (int t = 0; t < T; ++t) {
    if (tri_mat && tri_mat[5 * t] * tri_mat[5 * t + 1] == 0.f) continue;  // inactive triangle mask
    add(tri[3 * t], tri[3 * t + 1]);
    add(tri[3 * t], tri[3 * t + 2]);
    add(tri[3 * t + 1], tri[3 * t + 2]);
  }
  if (include_bending)
    for (int e = 0; e < E; ++e) {
      if (edge_props && edge_props[2 * e] == 0.f && edge_props[2 * e + 1] == 0.f) continue;
      const int* ei = edges + 4 * e;
      for (int i = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j) add(ei[i], ei[j]);
    }
  for (uint64_t p : pairs)
    if (int(p >> 32) >= V || int(p & 0xffffffffu) >= V) return VBD_ERR_INVALID_ARGUMENT;
  return color_pairs(V, pairs, target_ratio, colors);
}


int vbd_soft_contacts(int32_t n, const float* q, const float* radius, const int32_t* flags, int32_t S,
                      const int32_t* shape_type, const float* shape_pos, const float* shape_radius,
                      const float* shape_normal, float margin,
                      int32_t cmax, int32_t* count, int32_t* particle, int32_t* shape, float* body_pos,
                      float* body_vel, float* normal, void* stream) {
  if (n < 0 || S < 0 || S > kMaxContactShapes || cmax < 0 || !count || (S && (!shape_type || !shape_pos)))
    return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(count, 0, sizeof(int), st));
  if (n == 0 || S == 0) return VBD_OK;
  ShapeTable tab;
  std::memset(&tab, 0, sizeof(tab));
  for (int s = 0; s < S; ++s) {
    if (shape_type[s] != 0 && shape_type[s] != 1) return VBD_ERR_UNSUPPORTED;
    tab.type[s] = shape_type[s];
    tab.pos_radius[s] = make_float4(shape_pos[3 * s], shape_pos[3 * s + 1], shape_pos[3 * s + 2],
                                    shape_radius ? shape_radius[s] : 0.f);
    float nx = 0.f, ny = 0.f, nz = 1.f;
    if (shape_normal) nx = shape_normal[3 * s], ny = shape_normal[3 * s + 1], nz = shape_normal[3 * s + 2];
    const float nl = sqrtf(nx * nx + ny * ny + nz * nz);
    if (shape_type[s] == 0 && !(nl > 0.f)) return VBD_ERR_INVALID_ARGUMENT;
    tab.normal[s] = nl > 0.f ? make_float4(nx / nl, ny / nl, nz / nl, 0.f) : make_float4(0.f, 0.f, 1.f, 0.f);
  }
  const long total = long(n) * S;
  k_soft_contacts<<<int((total + 255) / 256), 256, 0, st>>>(n, q, radius, flags, S, tab, margin, cmax, count, particle,
                                                            shape, body_pos, body_vel, normal);
  CK(cudaGetLastError());
  return VBD_OK;
}

int vbd_soft_contacts_table(int32_t n, const float* q, const float* radius, const int32_t* flags,
                            const VbdShapeTable* tb, float margin, int32_t cmax, int32_t* count, int32_t* particle,
                            int32_t* shape, float* body_pos, float* body_vel, float* normal, void* stream) {
  if (!tb) return VBD_ERR_INVALID_ARGUMENT;
  const int S = tb->shape_count;
  if (n < 0 || S < 0 || S > kMaxContactShapes || cmax < 0 || !count || tb->heightfield_count < 0 ||
      tb->elevation_count < 0 || (S && (!tb->shape_type_host || !tb->shape_transform_host || !tb->shape_scale_host)))
    return VBD_ERR_INVALID_ARGUMENT;
  if (n > 0 && S > 0 && (!q || !radius || !flags || (cmax > 0 && (!particle || !shape || !body_pos || !body_vel || !normal))))
    return VBD_ERR_INVALID_ARGUMENT;
  ShapeParamTable tab;
  std::memset(&tab, 0, sizeof(tab));
  int m = 0;  // shapes that collide with particles, in model order (COLLIDE_PARTICLES, geometry/kernels.py:1033-1034)
  for (int s0 = 0; s0 < S; ++s0) {
    if (tb->shape_flags_host && !(tb->shape_flags_host[s0] & 4)) continue;
    const int rc = fill_shape_rec(tb, s0, tab.rec[m++]);
    if (rc != VBD_OK) return rc;
  }
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(count, 0, sizeof(int), st));
  if (n == 0 || m == 0) return VBD_OK;
  bool worlds = false, bodies = false;
  for (int s = 0; s < m; ++s) {
    worlds = worlds || tab.rec[s].world != -1;
    bodies = bodies || tab.rec[s].body >= 0;
  }
  if (bodies && !tb->body_q_dev) return VBD_ERR_INVALID_ARGUMENT;
  const bool w = worlds && tb->particle_world_dev;
  auto kern = bodies ? (w ? k_soft_contacts_shapes<true, true> : k_soft_contacts_shapes<false, true>)
                     : (w ? k_soft_contacts_shapes<true, false> : k_soft_contacts_shapes<false, false>);
  kern<<<(n + 255) / 256, 256, 0, st>>>(n, q, radius, flags, m, tab, tb->elevations_dev, tb->particle_world_dev,
                                         tb->body_q_dev, margin, cmax, count, particle, shape, body_pos, body_vel,
                                         normal);
  CK(cudaGetLastError());
  return VBD_OK;
}

int vbd_soft_contacts_shapes(int32_t n, const float* q, const float* radius, const int32_t* flags, int32_t S,
                             const int32_t* shape_type, const float* shape_transform, const float* shape_scale,
                             float margin, int32_t cmax, int32_t* count, int32_t* particle, int32_t* shape,
                             float* body_pos, float* body_vel, float* normal, void* stream) {
  for (int s = 0; s < S && shape_type; ++s)  // grids and meshes come with vbd_soft_contacts_table
    if (shape_type[s] == GEO_HFIELD || shape_type[s] == GEO_MESH || shape_type[s] == GEO_CONVEX_MESH)
      return VBD_ERR_UNSUPPORTED;
  VbdShapeTable tb;
  std::memset(&tb, 0, sizeof(tb));
  tb.shape_count = S;
  tb.shape_type_host = shape_type;
  tb.shape_transform_host = shape_transform;
  tb.shape_scale_host = shape_scale;
  return vbd_soft_contacts_table(n, q, radius, flags, &tb, margin, cmax, count, particle, shape, body_pos, body_vel,
                                 normal, stream);
}

int vbd_set_self_contact(VbdHandle h, const VbdSelfContactDesc* d) {
  if (!h || !d) return VBD_ERR_INVALID_ARGUMENT;
  if (!(d->radius > 0.0) || !(d->margin >= d->radius) || !(d->relaxation > 0.0) || d->vertex_buffer_size < 1 ||
      d->edge_buffer_size < 1 || !(d->edge_parallel_epsilon >= 0.0) || !(d->rest_exclusion_radius >= 0.0))
    return VBD_ERR_INVALID_ARGUMENT;
  if (d->rest_exclusion_radius > 0.0 && !d->rest_q_dev) return VBD_ERR_INVALID_ARGUMENT;
  const bool persistent = h->schedule == VBD_SCHEDULE_PERSISTENT;
  if ((h->schedule != VBD_SCHEDULE_PER_COLOR && !persistent) || h->layout != VBD_LAYOUT_CSR) return VBD_ERR_UNSUPPORTED;
  // persistent: cloth only, the AVBD penalty fixed (its dual update would need a grid-wide pass per iteration)
  if (persistent && (h->soft || h->warp_inst || h->prm.avbd_linear_beta != 0.f)) return VBD_ERR_UNSUPPORTED;
  const long long V = h->V, E = h->E;
  if (V * d->vertex_buffer_size >= (1LL << 29) || E * d->edge_buffer_size >= (1LL << 29) ||
      4 * V * d->vertex_buffer_size + 2 * E * d->edge_buffer_size >= (1LL << 31))
    return VBD_ERR_TOO_LARGE;
  if (cudaDeviceSynchronize() != cudaSuccess) return VBD_ERR_CUDA;
  sc_release(h->sc);
  for (void** p : {&h->sc_pos_cd, &h->sc_disp, &h->sc_ts}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  h->sc_on = false;
  const bool f64 = h->precision == VBD_PRECISION_FP64;
  int rc = f64 ? sc_alloc<double>(h->sc, h->V, h->T, h->E, d->vertex_buffer_size, d->edge_buffer_size)
               : sc_alloc<float>(h->sc, h->V, h->T, h->E, d->vertex_buffer_size, d->edge_buffer_size);
  if (rc) return rc;
  if ((rc = sc_upload_filter(d->vt_filter_offsets_host, d->vt_filter_host, h->V, h->T, &h->sc.vt_foff, &h->sc.vt_f)) ||
      (rc = sc_upload_filter(d->ee_filter_offsets_host, d->ee_filter_host, h->E, h->E, &h->sc.ee_foff, &h->sc.ee_f)))
    return rc;
  const size_t p4 = f64 ? sizeof(double4) : sizeof(float4);
  if ((rc = dalloc((char**)&h->sc_pos_cd, p4 * h->V)) || (rc = dalloc((char**)&h->sc_disp, p4 * h->V)) ||
      (rc = dalloc((char**)&h->sc_ts, (f64 ? 8 : 4) * size_t(h->V))))
    return rc;
  if (f64)
    k_sc_fill<double><<<(h->V + 255) / 256, 256>>>(h->V, (double*)h->sc_ts, 1.0);
  else
    k_sc_fill<float><<<(h->V + 255) / 256, 256>>>(h->V, (float*)h->sc_ts, 1.f);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  h->sc_radius = d->radius;
  h->sc_margin = d->margin;
  h->sc_relax = d->relaxation;
  h->sc_ee_eps = d->edge_parallel_epsilon;
  h->sc_rest_excl = d->rest_exclusion_radius;
  h->sc_interval = d->detection_interval;
  h->sc_rest_q = d->rest_q_dev;
  for (int** p : {&h->sc_estart, &h->sc_world}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (persistent) {
    // the edges of an instance must be one contiguous range (add_world appends them world by world); pairs across
    // instances are skipped by the detection (the instance key of a vertex is its instance's first particle)
    std::vector<int> wstart(size_t(h->W) + 1);
    CK(cudaMemcpy(wstart.data(), h->inst_vstart, sizeof(int) * wstart.size(), cudaMemcpyDeviceToHost));
    std::vector<int> we(h->E), estart(size_t(h->W) + 1);
    for (int e = 0; e < h->E; ++e) {
      const int v0 = h->h_edges[4 * size_t(e) + 2];
      we[e] = int(std::upper_bound(wstart.begin(), wstart.end(), v0) - wstart.begin()) - 1;
      if (e > 0 && we[e] < we[e - 1]) return VBD_ERR_UNSUPPORTED;
    }
    for (int w = 0; w <= h->W; ++w) estart[w] = int(std::lower_bound(we.begin(), we.end(), w) - we.begin());
    if ((rc = upload(&h->sc_estart, estart)) || (rc = upload(&h->sc_world, h->inst_start_of_vertex))) return rc;
    h->sc.world = h->sc_world;
    const void* fn = f64 ? persistent_sc_fn<double, MODE_FP64>(h->L)
                         : (h->precision == VBD_PRECISION_MIXED ? persistent_sc_fn<float, MODE_MIXED>(h->L)
                                                                : persistent_sc_fn<float, MODE_FP32>(h->L));
    int dev = 0, sms = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, h->block, 0));
    if (per_sm < 1) return VBD_ERR_INVALID_ARGUMENT;
    h->grid_sc = std::min(h->W, sms * per_sm);
  }
  h->sc_on = true;
  return VBD_OK;
}

int vbd_get_self_contact_counts(VbdHandle h, int32_t* vt_pairs, int32_t* ee_pairs, int32_t* flags, void* stream) {
  if (!h || !h->sc_on) return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  int nv = 0, ne = 0, fl[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(&nv, h->sc.vt_off + h->V, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&ne, h->sc.ee_off + h->E, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(fl, h->sc.flags, sizeof(fl), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (vt_pairs) *vt_pairs = nv;
  if (ee_pairs) *ee_pairs = ne;
  if (flags) *flags = fl[0] | (fl[2] << 2) | (fl[3] << 3);
  return VBD_OK;
}

int vbd_build_contact_filters(int32_t V, int32_t T, const int32_t* tri, int32_t E, const int32_t* edges, int32_t ring,
                              int32_t* vt_off, int32_t* vt_list, int32_t* ee_off, int32_t* ee_list) {
  if (V < 0 || T < 0 || E < 0 || ring < 2 || (T && !tri) || (E && !edges) || !vt_off || !ee_off)
    return VBD_ERR_INVALID_ARGUMENT;
  for (long long i = 0; i < 3LL * T; ++i)
    if (tri[i] < 0 || tri[i] >= V) return VBD_ERR_INVALID_ARGUMENT;
  for (int e = 0; e < E; ++e)
    for (int j = 0; j < 4; ++j)
      if (edges[4 * e + j] < -1 || edges[4 * e + j] >= V || (j >= 2 && edges[4 * e + j] < 0))
        return VBD_ERR_INVALID_ARGUMENT;
  // vertex -> faces, vertex -> edges in any role, vertex -> edges it is an endpoint of, one-ring neighbours
  std::vector<std::vector<int>> vf(V), ve_any(V), ve_end(V), nbr(V);
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 3; ++j) vf[tri[3 * t + j]].push_back(t);
  for (int e = 0; e < E; ++e) {
    const int* ei = edges + 4 * e;
    for (int j = 0; j < 4; ++j)
      if (ei[j] >= 0) ve_any[ei[j]].push_back(e);
    ve_end[ei[2]].push_back(e);
    ve_end[ei[3]].push_back(e);
    if (ei[2] != ei[3]) {
      nbr[ei[2]].push_back(ei[3]);
      nbr[ei[3]].push_back(ei[2]);
    }
  }
  for (auto& l : nbr) {
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
  }
  // vertices within ring - 1 steps of v (including v), as leq_n_ring_vertices / one_ring_vertices
  std::vector<int> mark(V, -1), ringv;
  auto ring_of = [&](int v, int stamp, std::vector<int>& out) {
    out.clear();
    std::vector<int> frontier{v};
    if (mark[v] != stamp) {
      mark[v] = stamp;
      out.push_back(v);
    }
    for (int k = 0; k < ring - 1 && !frontier.empty(); ++k) {
      std::vector<int> next;
      for (int u : frontier)
        for (int w : nbr[u])
          if (mark[w] != stamp) {
            mark[w] = stamp;
            out.push_back(w);
            next.push_back(w);
          }
      frontier.swap(next);
    }
  };
  // pass over vertices: triangles touching a ring vertex other than v, minus v's own triangles
  std::vector<int> row;
  long long total = 0;
  vt_off[0] = 0;
  int stamp = 0;
  for (int v = 0; v < V; ++v) {
    ring_of(v, stamp++, ringv);
    row.clear();
    for (int w : ringv)
      if (w != v) row.insert(row.end(), vf[w].begin(), vf[w].end());
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    std::vector<int> own = vf[v];
    std::sort(own.begin(), own.end());
    std::vector<int> keep;
    std::set_difference(row.begin(), row.end(), own.begin(), own.end(), std::back_inserter(keep));
    if (vt_list)
      std::copy(keep.begin(), keep.end(), vt_list + total);
    total += keep.size();
    if (total >= (1LL << 31)) return VBD_ERR_TOO_LARGE;
    vt_off[v + 1] = int(total);
  }
  // pass over edges: edges with an endpoint in either endpoint's ring (other than the endpoints),
  // minus edges in which an endpoint takes any role
  total = 0;
  ee_off[0] = 0;
  std::vector<int> r1, r2;
  for (int e = 0; e < E; ++e) {
    const int a = edges[4 * e + 2], b = edges[4 * e + 3];
    ring_of(a, stamp++, r1);
    ring_of(b, stamp++, r2);
    row.clear();
    for (const auto* lst : {&r1, &r2})
      for (int w : *lst)
        if (w != a && w != b) row.insert(row.end(), ve_end[w].begin(), ve_end[w].end());
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    std::vector<int> own = ve_any[a];
    own.insert(own.end(), ve_any[b].begin(), ve_any[b].end());
    std::sort(own.begin(), own.end());
    std::vector<int> keep;
    std::set_difference(row.begin(), row.end(), own.begin(), own.end(), std::back_inserter(keep));
    if (ee_list)
      std::copy(keep.begin(), keep.end(), ee_list + total);
    total += keep.size();
    if (total >= (1LL << 31)) return VBD_ERR_TOO_LARGE;
    ee_off[e + 1] = int(total);
  }
  return VBD_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------ standalone detector
struct VbdCollider {
  int V = 0, T = 0, E = 0;
  int4* tri_idx = nullptr;
  int4* edge_idx = nullptr;
  float4* pos = nullptr;
  double ee_eps = 1e-5;
  ScBuffers b;
  ~VbdCollider() {
    for (void* p : {(void*)tri_idx, (void*)edge_idx, (void*)pos})
      if (p) cudaFree(p);
    sc_release(b);
  }
};

namespace {
__global__ void k_col_pack(int T, const int* __restrict__ tri, int E, const int* __restrict__ edges, int4* ti, int4* ei) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < T) ti[i] = make_int4(tri[3 * i], tri[3 * i + 1], tri[3 * i + 2], 0);
  if (i < E) ei[i] = make_int4(edges[4 * i], edges[4 * i + 1], edges[4 * i + 2], edges[4 * i + 3]);
}
__global__ void k_col_pos(int V, const float* __restrict__ q, float4* p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < V) p[i] = make_float4(q[3 * i], q[3 * i + 1], q[3 * i + 2], 0.f);
}
// reference layout: 2 ints (primitive, partner) per slot, -1 in unused slots
__global__ void k_col_export(int P, int cap, const int* __restrict__ list, const int* __restrict__ cnt,
                             const float* __restrict__ mn, int* out, int* out_cnt, float* out_min) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const int n = min(cnt[i], cap);
  for (int k = 0; k < cap; ++k) {
    out[2 * (size_t(i) * cap + k)] = k < n ? i : -1;
    out[2 * (size_t(i) * cap + k) + 1] = k < n ? list[size_t(i) * cap + k] : -1;
  }
  if (out_cnt) out_cnt[i] = cnt[i];
  if (out_min) out_min[i] = mn[i];
}
__global__ void k_col_flags(const int* __restrict__ f, int* out) {
  if (threadIdx.x < 3 && f[threadIdx.x]) out[threadIdx.x] = 1;
}
}  // namespace

extern "C" {

int vbd_collider_create(int32_t V, int32_t T, const int32_t* tri_dev, int32_t E, const int32_t* edges_dev,
                        int32_t vertex_buffer_size, int32_t edge_buffer_size, float edge_parallel_epsilon,
                        const int32_t* vt_filter_offsets_host, const int32_t* vt_filter_host,
                        const int32_t* ee_filter_offsets_host, const int32_t* ee_filter_host, VbdColliderHandle* out) {
  if (!out || V < 0 || T < 0 || E < 0 || (T && !tri_dev) || (E && !edges_dev) || vertex_buffer_size < 1 ||
      edge_buffer_size < 1)
    return VBD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  VbdCollider* c = new (std::nothrow) VbdCollider();
  if (!c) return VBD_ERR_OUT_OF_MEMORY;
  c->V = V, c->T = T, c->E = E, c->ee_eps = edge_parallel_epsilon;
  int rc;
  if ((rc = dalloc(&c->tri_idx, size_t(T))) || (rc = dalloc(&c->edge_idx, size_t(E))) ||
      (rc = dalloc(&c->pos, size_t(V))) || (rc = sc_alloc<float>(c->b, V, T, E, vertex_buffer_size, edge_buffer_size)) ||
      (rc = sc_upload_filter(vt_filter_offsets_host, vt_filter_host, V, T, &c->b.vt_foff, &c->b.vt_f)) ||
      (rc = sc_upload_filter(ee_filter_offsets_host, ee_filter_host, E, E, &c->b.ee_foff, &c->b.ee_f))) {
    delete c;
    return rc;
  }
  // the indices are checked once here, as vbd_create checks a model's
  std::vector<int> ht(3 * size_t(T)), he(4 * size_t(E));
  if ((T && cudaMemcpy(ht.data(), tri_dev, ht.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (E && cudaMemcpy(he.data(), edges_dev, he.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)) {
    delete c;
    return VBD_ERR_CUDA;
  }
  bool ok = true;
  for (int v : ht) ok = ok && v >= 0 && v < V;
  for (size_t i = 0; i < he.size(); ++i) ok = ok && he[i] < V && he[i] >= ((i % 4) >= 2 ? 0 : -1);
  if (!ok) {
    delete c;
    return VBD_ERR_INVALID_ARGUMENT;
  }
  const int n = std::max(T, E);
  if (n > 0) k_col_pack<<<(n + 255) / 256, 256>>>(T, tri_dev, E, edges_dev, c->tri_idx, c->edge_idx);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
    delete c;
    return VBD_ERR_CUDA;
  }
  *out = c;
  return VBD_OK;
}

int vbd_collider_detect(VbdColliderHandle c, int32_t what, const float* pos_dev, float max_query_radius,
                        float min_query_radius, const float* ref_pos_dev, int32_t* vt_dev, int32_t* vt_count_dev,
                        float* vt_min_dev, int32_t* ee_dev, int32_t* ee_count_dev, float* ee_min_dev,
                        int32_t* resize_flags_dev, void* stream) {
  if (!c || !pos_dev || !(max_query_radius >= 0.f) || (what & ~3) || (min_query_radius > 0.f && !ref_pos_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  if (((what & 1) && !vt_dev) || ((what & 2) && !ee_dev)) return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (c->V) k_col_pos<<<(c->V + 255) / 256, 256, 0, st>>>(c->V, pos_dev, c->pos);
  CK(cudaMemsetAsync(c->b.flags, 0, 4 * sizeof(int), st));
  ScSetup p{double(max_query_radius), double(min_query_radius), c->ee_eps, ref_pos_dev, nullptr};
  const bool tris = (what & 1) && c->b.tb > 0 && c->T > 0;
  const long long nt = (long long)c->T * c->b.tb;
  if (tris)
    k_sc_tri_init<<<unsigned((std::max<long long>(nt, c->T) + 255) / 256), 256, 0, st>>>(
        c->T, c->b.tb, c->b.tv, c->b.tv_count, c->b.tv_min, max_query_radius);
  int rc = sc_detect<float>(c->b, p, c->tri_idx, c->edge_idx, c->pos, what, st);
  if (rc) return rc;
  if (tris) k_sc_tri_finish<<<unsigned((nt + 255) / 256), 256, 0, st>>>(c->T, c->b.tb, c->b.tv);
  if ((what & 1) && c->V)
    k_col_export<<<(c->V + 255) / 256, 256, 0, st>>>(c->V, c->b.vb, c->b.vt_tri, c->b.vt_count, (const float*)c->b.vt_min,
                                                     vt_dev, vt_count_dev, vt_min_dev);
  if ((what & 2) && c->E)
    k_col_export<<<(c->E + 255) / 256, 256, 0, st>>>(c->E, c->b.eb, c->b.ee_edge, c->b.ee_count, (const float*)c->b.ee_min,
                                                     ee_dev, ee_count_dev, ee_min_dev);
  if (resize_flags_dev) k_col_flags<<<1, 32, 0, st>>>(c->b.flags, resize_flags_dev);
  CK(cudaGetLastError());
  return VBD_OK;
}

int vbd_collider_set_triangle_buffers(VbdColliderHandle c, int32_t buffer_size, int32_t* vertices_dev,
                                      int32_t* count_dev, float* min_dist_dev) {
  if (!c || buffer_size < 0 || (buffer_size > 0 && c->T > 0 && (!vertices_dev || !count_dev || !min_dist_dev)))
    return VBD_ERR_INVALID_ARGUMENT;
  c->b.tb = buffer_size;
  c->b.tv = buffer_size > 0 ? vertices_dev : nullptr;
  c->b.tv_count = buffer_size > 0 ? count_dev : nullptr;
  c->b.tv_min = buffer_size > 0 ? min_dist_dev : nullptr;
  return VBD_OK;
}

int vbd_collider_destroy(VbdColliderHandle c) {
  if (!c) return VBD_ERR_INVALID_ARGUMENT;
  cudaDeviceSynchronize();
  delete c;
  return VBD_OK;
}

}  // extern "C"
