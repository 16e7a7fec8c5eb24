// Device-resident shape sets for particle contacts: a model's shapes uploaded once, with the lists that
// give each particle only the shapes it may touch (create_soft_contacts' world filter, geometry/kernels.py:
// 1036-1043): a particle of world w tests the global shapes and the shapes of world w, a global particle tests
// every shape. Any number of shapes and worlds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "vbd_b200.h"
#include "vbd_contactgen.cuh"

using vbd::ShapeRec;

struct VbdShapeSetImpl {
  const ShapeRec* recs;  // the shapes that collide with particles, in model order
  const int* global;     // indices into recs of the global shapes
  const int* world_off;  // [W + 1]: world w's shapes are world_list[world_off[w] .. world_off[w + 1])
  const int* world_list;
  int m, n_global, W;
  const float* elev;
  void* buffer;
  vbd::ShapeParamTable small;  // the records again when m <= kParamTableShapes: launched as a kernel parameter
  bool worlds;                 // some shape belongs to a world
  bool bodies;                 // some shape is on a body: launches need the body transforms
  bool param_table;            // launch small sets with `small` (else the global-memory kernel for every size)
};

namespace {

template <bool BODIES>
__global__ void __launch_bounds__(256, 4)
    k_soft_contacts_set(int n, const float* __restrict__ q, const float* __restrict__ radius,
                        const int* __restrict__ flags, const int* __restrict__ particle_world,
                        const ShapeRec* __restrict__ recs, int m, const int* __restrict__ global, int n_global,
                        const int* __restrict__ world_off, const int* __restrict__ world_list, int W,
                        const float* __restrict__ elev, const float* __restrict__ body_q, float margin, int cmax,
                        int* count, int* particle, int* shape, float* body_pos, float* body_vel, float* normal) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(flags[i] & 1)) return;
  const vbd::vec3<float> x = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};
  const float r = radius[i];
  const int pw = particle_world ? particle_world[i] : -1;
  // one loop over two segments: every shape (a global particle) or the global shapes, then world pw's shapes
  const int na = pw == -1 ? m : n_global;
  const bool own = pw >= 0 && pw < W;
  const int w0 = own ? world_off[pw] : 0, nb = own ? world_off[pw + 1] - w0 : 0;
  for (int k = 0; k < na + nb; ++k) {
    const int s = k < na ? (pw == -1 ? k : global[k]) : world_list[w0 + k - na];
    vbd::soft_contact_shape<BODIES>(recs[s], elev, body_q, x, r, margin, i, cmax, count, particle, shape, body_pos,
                                    body_vel, normal);
  }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int vbd_shape_set_create(const VbdShapeTable* tb, VbdShapeSetHandle* out) {
  if (!out) return VBD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!tb || tb->shape_count < 0 || tb->heightfield_count < 0 || tb->elevation_count < 0 ||
      (tb->shape_count && (!tb->shape_type_host || !tb->shape_transform_host || !tb->shape_scale_host)))
    return VBD_ERR_INVALID_ARGUMENT;
  std::vector<ShapeRec> recs;
  int W = 0;
  for (int s0 = 0; s0 < tb->shape_count; ++s0) {
    if (tb->shape_flags_host && !(tb->shape_flags_host[s0] & 4)) continue;  // not COLLIDE_PARTICLES
    ShapeRec rec;
    const int rc = vbd::fill_shape_rec(tb, s0, rec);
    if (rc != VBD_OK) return rc;
    if (rec.world < -1) return VBD_ERR_INVALID_ARGUMENT;
    if (rec.world + 1 > W) W = rec.world + 1;
    recs.push_back(rec);
  }
  const int m = int(recs.size());
  std::vector<int> global, off(W + 1, 0), list;
  for (int s = 0; s < m; ++s) {
    if (recs[s].world == -1) global.push_back(s);
    else ++off[recs[s].world + 1];
  }
  for (int w = 0; w < W; ++w) off[w + 1] += off[w];
  list.resize(off[W]);
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (int s = 0; s < m; ++s)
    if (recs[s].world >= 0) list[fill[recs[s].world]++] = s;
  const size_t sr = align256(sizeof(ShapeRec) * std::max(m, 1)), sg = align256(sizeof(int) * std::max<size_t>(global.size(), 1));
  const size_t so = align256(sizeof(int) * off.size()), sl = align256(sizeof(int) * std::max<size_t>(list.size(), 1));
  char* buf = nullptr;
  if (cudaMalloc(&buf, sr + sg + so + sl) != cudaSuccess) return VBD_ERR_OUT_OF_MEMORY;
  const bool ok =
      (m == 0 || cudaMemcpy(buf, recs.data(), sizeof(ShapeRec) * m, cudaMemcpyHostToDevice) == cudaSuccess) &&
      (global.empty() ||
       cudaMemcpy(buf + sr, global.data(), sizeof(int) * global.size(), cudaMemcpyHostToDevice) == cudaSuccess) &&
      cudaMemcpy(buf + sr + sg, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
      (list.empty() ||
       cudaMemcpy(buf + sr + sg + so, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice) == cudaSuccess);
  if (!ok) {
    cudaFree(buf);
    return VBD_ERR_CUDA;
  }
  VbdShapeSetImpl* set = new (std::nothrow) VbdShapeSetImpl();
  if (!set) {
    cudaFree(buf);
    return VBD_ERR_OUT_OF_MEMORY;
  }
  set->recs = reinterpret_cast<const ShapeRec*>(buf);
  set->global = reinterpret_cast<const int*>(buf + sr);
  set->world_off = reinterpret_cast<const int*>(buf + sr + sg);
  set->world_list = reinterpret_cast<const int*>(buf + sr + sg + so);
  set->m = m;
  set->n_global = int(global.size());
  set->W = W;
  set->elev = tb->elevations_dev;
  set->buffer = buf;
  set->worlds = W > 0;
  set->bodies = std::any_of(recs.begin(), recs.end(), [](const ShapeRec& r) { return r.body >= 0; });
  set->param_table = true;
  if (m <= vbd::kParamTableShapes) std::copy(recs.begin(), recs.end(), set->small.rec);
  *out = set;
  return VBD_OK;
}

int vbd_shape_set_use_parameter_table(VbdShapeSetHandle set, int32_t enable) {
  if (!set || (enable != 0 && enable != 1)) return VBD_ERR_INVALID_ARGUMENT;
  set->param_table = enable != 0;
  return VBD_OK;
}

int vbd_shape_set_destroy(VbdShapeSetHandle set) {
  if (!set) return VBD_OK;
  const cudaError_t e = cudaFree(set->buffer);
  delete set;
  return e == cudaSuccess ? VBD_OK : VBD_ERR_CUDA;
}

int vbd_soft_contacts_set(VbdShapeSetHandle set, int32_t n, const float* q, const float* radius, const int32_t* flags,
                          const int32_t* particle_world, const float* body_q, float margin, int32_t cmax, int32_t* count,
                          int32_t* particle, int32_t* shape, float* body_pos, float* body_vel, float* normal,
                          void* stream) {
  if (!set || n < 0 || cmax < 0 || !count || (set->bodies && !body_q)) return VBD_ERR_INVALID_ARGUMENT;
  if (n > 0 && set->m > 0 &&
      (!q || !radius || !flags || (cmax > 0 && (!particle || !shape || !body_pos || !body_vel || !normal))))
    return VBD_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(count, 0, sizeof(int), st) != cudaSuccess) return VBD_ERR_CUDA;
  if (n == 0 || set->m == 0) return VBD_OK;
  if (set->param_table && set->m <= vbd::kParamTableShapes) {  // small sets: records in the constant bank measured faster
    const bool w = set->worlds && particle_world;
    auto kern = set->bodies ? (w ? vbd::k_soft_contacts_shapes<true, true> : vbd::k_soft_contacts_shapes<false, true>)
                            : (w ? vbd::k_soft_contacts_shapes<true, false> : vbd::k_soft_contacts_shapes<false, false>);
    kern<<<(n + 255) / 256, 256, 0, st>>>(n, q, radius, flags, set->m, set->small, set->elev, particle_world, body_q,
                                           margin, cmax, count, particle, shape, body_pos, body_vel, normal);
    return cudaGetLastError() == cudaSuccess ? VBD_OK : VBD_ERR_CUDA;
  }
  auto kset = set->bodies ? k_soft_contacts_set<true> : k_soft_contacts_set<false>;
  kset<<<(n + 255) / 256, 256, 0, st>>>(n, q, radius, flags, particle_world, set->recs, set->m, set->global,
                                         set->n_global, set->world_off, set->world_list, set->W, set->elev, body_q,
                                         margin, cmax, count, particle, shape, body_pos, body_vel, normal);
  return cudaGetLastError() == cudaSuccess ? VBD_OK : VBD_ERR_CUDA;
}

}  // extern "C"
