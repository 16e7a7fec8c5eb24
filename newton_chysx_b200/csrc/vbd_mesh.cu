// Static triangle meshes for particle contacts: vbd_mesh_create builds, on the host, the median-split bounding-
// volume hierarchy and the angle-weighted pseudo-normals that mesh_query_point_sign (vbd_mesh.cuh) reads, and
// uploads them in one allocation. The reference builds a Warp mesh (wp.Mesh, geometry/types.py:1436-1453) from
// Mesh.vertices and Mesh.indices with zero velocities.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <utility>
#include <vector>

#include "vbd_b200.h"
#include "vbd_mesh.cuh"

using vbd::MeshBvhNode;

namespace {

struct D3 {
  double x, y, z;
};
D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 cross3(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
D3 unit(D3 a) {
  const double l = std::sqrt(dot3(a, a));
  return l > 0.0 ? mul(a, 1.0 / l) : a;
}

struct Box {
  float lo[3], hi[3];
};

Box merge(const Box& a, const Box& b) {
  Box r;
  for (int k = 0; k < 3; ++k) r.lo[k] = std::min(a.lo[k], b.lo[k]), r.hi[k] = std::max(a.hi[k], b.hi[k]);
  return r;
}

// Median split along the longest axis of the centroids' box; ties in the centroid coordinate go by triangle
// index, so the hierarchy is the same on every run. Returns the node id, or ~triangle for a leaf.
int build_node(std::vector<int>& idx, int b, int e, const std::vector<Box>& tb, const std::vector<float>& cen,
               std::vector<MeshBvhNode>& nodes, Box& out) {
  if (e - b == 1) {
    out = tb[idx[b]];
    return ~idx[b];
  }
  float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = b; i < e; ++i)
    for (int k = 0; k < 3; ++k) clo[k] = std::min(clo[k], cen[3 * idx[i] + k]), chi[k] = std::max(chi[k], cen[3 * idx[i] + k]);
  int axis = 0;
  for (int k = 1; k < 3; ++k)
    if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
  const int m = b + (e - b) / 2;
  std::nth_element(idx.begin() + b, idx.begin() + m, idx.begin() + e, [&](int x, int y) {
    const float cx = cen[3 * x + axis], cy = cen[3 * y + axis];
    return cx < cy || (cx == cy && x < y);
  });
  const int id = int(nodes.size());
  nodes.emplace_back();
  Box l, r;
  const int cl = build_node(idx, b, m, tb, cen, nodes, l);
  const int cr = build_node(idx, m, e, tb, cen, nodes, r);
  MeshBvhNode& nd = nodes[id];
  std::memset(&nd, 0, sizeof(nd));
  nd.lo[0] = make_float4(l.lo[0], l.lo[1], l.lo[2], 0.f), nd.hi[0] = make_float4(l.hi[0], l.hi[1], l.hi[2], 0.f);
  nd.lo[1] = make_float4(r.lo[0], r.lo[1], r.lo[2], 0.f), nd.hi[1] = make_float4(r.hi[0], r.hi[1], r.hi[2], 0.f);
  nd.child[0] = cl, nd.child[1] = cr;
  out = merge(l, r);
  return id;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" {

int vbd_mesh_create(const float* points, int32_t point_count, const int32_t* indices, int32_t tri_count,
                    VbdMeshHandle* out) {
  if (!out) return VBD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (point_count < 1 || tri_count < 1 || !points || !indices || tri_count > (1 << 28) || point_count > (1 << 28))
    return VBD_ERR_INVALID_ARGUMENT;
  const int V = point_count, T = tri_count;
  for (long i = 0; i < 3L * V; ++i)
    if (!std::isfinite(points[i])) return VBD_ERR_INVALID_ARGUMENT;
  for (long i = 0; i < 3L * T; ++i)
    if (indices[i] < 0 || indices[i] >= V) return VBD_ERR_INVALID_ARGUMENT;
  auto P = [&](int v) { return D3{points[3 * v], points[3 * v + 1], points[3 * v + 2]}; };
  // pseudo-normals: unit face normals; per edge the sum over its faces; per vertex the angle-weighted sum
  std::vector<float4> fn(T), en(3 * size_t(T)), vn(V);
  std::vector<D3> vacc(V, D3{0.0, 0.0, 0.0});
  std::map<std::pair<int, int>, D3> eacc;
  std::vector<D3> fu(T);
  for (int t = 0; t < T; ++t) {
    const int a = indices[3 * t], b = indices[3 * t + 1], c = indices[3 * t + 2];
    const D3 pa = P(a), pb = P(b), pc = P(c);
    const D3 n = unit(cross3(sub(pb, pa), sub(pc, pa)));
    fu[t] = n;
    fn[t] = make_float4(float(n.x), float(n.y), float(n.z), 0.f);
    const int vs[3] = {a, b, c};
    const D3 ps[3] = {pa, pb, pc};
    for (int k = 0; k < 3; ++k) {
      const D3 u = sub(ps[(k + 1) % 3], ps[k]), w = sub(ps[(k + 2) % 3], ps[k]);
      const double ang = std::atan2(std::sqrt(dot3(cross3(u, w), cross3(u, w))), dot3(u, w));
      vacc[vs[k]] = add(vacc[vs[k]], mul(n, ang));
    }
    const std::pair<int, int> es[3] = {{std::min(a, b), std::max(a, b)}, {std::min(a, c), std::max(a, c)},
                                       {std::min(b, c), std::max(b, c)}};
    for (const auto& e : es) {
      auto it = eacc.find(e);
      if (it == eacc.end()) eacc.emplace(e, n);
      else it->second = add(it->second, n);
    }
  }
  for (int t = 0; t < T; ++t) {
    const int a = indices[3 * t], b = indices[3 * t + 1], c = indices[3 * t + 2];
    const std::pair<int, int> es[3] = {{std::min(a, b), std::max(a, b)}, {std::min(a, c), std::max(a, c)},
                                       {std::min(b, c), std::max(b, c)}};
    for (int k = 0; k < 3; ++k) {
      const D3 s = eacc[es[k]];
      en[3 * size_t(t) + k] = make_float4(float(s.x), float(s.y), float(s.z), 0.f);
    }
  }
  for (int v = 0; v < V; ++v) vn[v] = make_float4(float(vacc[v].x), float(vacc[v].y), float(vacc[v].z), 0.f);
  std::vector<float4> pts(V);
  for (int v = 0; v < V; ++v) pts[v] = make_float4(points[3 * v], points[3 * v + 1], points[3 * v + 2], 0.f);
  std::vector<int4> tris(T);
  std::vector<Box> tb(T);
  std::vector<float> cen(3 * size_t(T));
  for (int t = 0; t < T; ++t) {
    const int i0 = indices[3 * t], i1 = indices[3 * t + 1], i2 = indices[3 * t + 2];
    tris[t] = make_int4(i0, i1, i2, 0);
    for (int k = 0; k < 3; ++k) {
      const float x0 = points[3 * i0 + k], x1 = points[3 * i1 + k], x2 = points[3 * i2 + k];
      tb[t].lo[k] = std::min(x0, std::min(x1, x2));
      tb[t].hi[k] = std::max(x0, std::max(x1, x2));
      cen[3 * size_t(t) + k] = 0.5f * (tb[t].lo[k] + tb[t].hi[k]);
    }
  }
  std::vector<MeshBvhNode> nodes;
  nodes.reserve(T > 1 ? T - 1 : 1);
  if (T > 1) {
    std::vector<int> idx(T);
    std::iota(idx.begin(), idx.end(), 0);
    Box root;
    build_node(idx, 0, T, tb, cen, nodes, root);
  }
  // one allocation: nodes | pts | tris | fn | en | vn
  const size_t szn = align256(sizeof(MeshBvhNode) * std::max<size_t>(nodes.size(), 1));
  const size_t szp = align256(sizeof(float4) * V), szt = align256(sizeof(int4) * T), szf = align256(sizeof(float4) * T);
  const size_t sze = align256(sizeof(float4) * 3 * size_t(T)), szv = align256(sizeof(float4) * V);
  char* buf = nullptr;
  if (cudaMalloc(&buf, szn + szp + szt + szf + sze + szv) != cudaSuccess) return VBD_ERR_OUT_OF_MEMORY;
  char* o = buf;
  auto put = [&](const void* src, size_t bytes, size_t span) {
    char* at = o;
    o += span;
    return bytes == 0 || cudaMemcpy(at, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  char* const base_n = buf;
  const bool ok = put(nodes.data(), sizeof(MeshBvhNode) * nodes.size(), szn) && put(pts.data(), sizeof(float4) * V, szp) &&
                  put(tris.data(), sizeof(int4) * T, szt) && put(fn.data(), sizeof(float4) * T, szf) &&
                  put(en.data(), sizeof(float4) * 3 * size_t(T), sze) && put(vn.data(), sizeof(float4) * V, szv);
  if (!ok) {
    cudaFree(buf);
    return VBD_ERR_CUDA;
  }
  VbdMeshImpl* m = new (std::nothrow) VbdMeshImpl();
  if (!m) {
    cudaFree(buf);
    return VBD_ERR_OUT_OF_MEMORY;
  }
  m->buffer = buf;
  m->point_count = V;
  m->view.nodes = reinterpret_cast<const MeshBvhNode*>(base_n);
  m->view.pts = reinterpret_cast<const float4*>(base_n + szn);
  m->view.tris = reinterpret_cast<const int4*>(base_n + szn + szp);
  m->view.fn = reinterpret_cast<const float4*>(base_n + szn + szp + szt);
  m->view.en = reinterpret_cast<const float4*>(base_n + szn + szp + szt + szf);
  m->view.vn = reinterpret_cast<const float4*>(base_n + szn + szp + szt + szf + sze);
  m->view.tri_count = T;
  *out = m;
  return VBD_OK;
}

int vbd_mesh_destroy(VbdMeshHandle mesh) {
  if (!mesh) return VBD_OK;
  const cudaError_t e = cudaFree(mesh->buffer);
  delete mesh;
  return e == cudaSuccess ? VBD_OK : VBD_ERR_CUDA;
}

}  // extern "C"
