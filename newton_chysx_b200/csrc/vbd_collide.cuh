// Self-contact collision detection and the penetration-free truncation, device side.
//
// Replaces the reference's TriMeshCollisionDetector (newton/_src/solvers/vbd/tri_mesh_collision.py:91-413:
// wp.Bvh refit + vertex_triangle_collision_detection_kernel / edge_colliding_edges_detection_kernel,
// geometry/kernels.py:1252-1497) and the truncation kernels (particle_vbd_kernels.py:2744-2897).
//
// Broad phase: a uniform grid hashed into a power-of-two bucket table, rebuilt by a counting sort at
// every detection (no tree to refit). The cell size is max(2 margin + mean box size, largest box) x 1.01,
// so a primitive box covers at most 2 cells per axis (<= 8 insertions) and a query box at most 2
// (vertex) or 3 (edge) cells per axis. A primitive inserted in several cells is reported once: only in
// the cell holding the lower corner of the intersection of its box with the query box. The candidate
// set is then the set a BVH returns (all boxes overlapping the query box), and the narrow phase keeps the
// pairs closer than the margin, as the reference does.
//
// Buffers: each vertex keeps up to vertex_buffer triangle ids, each edge up to edge_buffer edge ids, in
// increasing id order (the reference keeps the first ones in BVH traversal order); the count includes the
// pairs past the buffer, and a flag records the overflow, as the reference's resize_flags do.
//
// For the solve, the recorded pairs are compacted into dense lists, and every vertex gets a sorted list of
// (pair, slot) entries naming the pairs it belongs to, so that its solve gathers its contact terms itself.
#pragma once
#include <climits>
#include <cub/cub.cuh>

#include "vbd_selfcontact.cuh"

namespace vbd {

constexpr int kScGridBlocks = 148 * 8;  // grid-stride launches over device-side pair counts

struct ScBuffers {
  int V = 0, T = 0, E = 0, vb = 0, eb = 0;
  int nbuckets = 0;              // power of two
  unsigned* bcount = nullptr;    // [nbuckets + 1] per-bucket counts, then fill cursors
  unsigned* bstart = nullptr;    // [nbuckets + 1] exclusive scan of the counts
  long long* ekey = nullptr;     // [gcap] cell key of each grid entry
  int* eprim = nullptr;          // [gcap] primitive of each grid entry
  long long gcap = 0;
  void* blo = nullptr;           // primitive boxes, pos4_t<R> [max(T, E)]
  void* bhi = nullptr;
  double* stats = nullptr;       // [4]: sum of box sizes, max box size (bits), cell size, 1 / cell size
  int* vt_tri = nullptr;         // [V * vb] colliding triangles of each vertex, ascending
  int* vt_count = nullptr;       // [V]
  void* vt_min = nullptr;        // [V] R: closest recorded distance (margin when none)
  int* ee_edge = nullptr;        // [E * eb]
  int* ee_count = nullptr;       // [E]
  void* ee_min = nullptr;        // [E] R
  int* flags = nullptr;          // [4] overflow flags: 0 vertex, 1 triangle, 2 edge buffers; 3 internal (grid)
  const int* world = nullptr;    // [V] instance key per vertex: pairs across instances are skipped; null = all kept
  int* tv = nullptr;             // caller's triangle -> colliding vertices buffers (stand-alone detector only)
  int* tv_count = nullptr;
  float* tv_min = nullptr;
  int tb = 0;
  int* tmp = nullptr;            // [max(V, E) + 1]
  int* vt_off = nullptr;         // [V + 1]
  int4* vt_pairs = nullptr;      // [V * vb] the pair's vertices: the triangle's three, then the vertex
  int* ee_off = nullptr;         // [E + 1]
  int4* ee_pairs = nullptr;      // [E * eb] the pair's vertices: the edge's two, then the other edge's two
  int* ent_cnt = nullptr;        // [V + 1] entries per vertex, then fill cursors
  int* ent_off = nullptr;        // [V + 1]
  unsigned* ent = nullptr;       // [ecap] (kind << 31) | (slot << 29) | pair
  long long ecap = 0;
  int* vt_foff = nullptr;        // filter lists (CSR, sorted rows), or null
  int* vt_f = nullptr;
  int* ee_foff = nullptr;
  int* ee_f = nullptr;
  void* scan_tmp = nullptr;
  size_t scan_bytes = 0;
};

// ------------------------------------------------------------------------------------ grid helpers
__device__ __forceinline__ int cell_of(double x, double inv) {
  double c = floor(x * inv);
  c = c < -1048576.0 ? -1048576.0 : (c > 1048575.0 ? 1048575.0 : c);
  return int(c);
}
__device__ __forceinline__ long long cell_key(int x, int y, int z) {
  return ((long long)(x & 0x1FFFFF) << 42) | ((long long)(y & 0x1FFFFF) << 21) | (long long)(z & 0x1FFFFF);
}
__device__ __forceinline__ unsigned cell_hash(int x, int y, int z, int nb) {
  return ((unsigned)x * 73856093u ^ (unsigned)y * 19349663u ^ (unsigned)z * 83492791u) & unsigned(nb - 1);
}

// Primitive boxes (kind 0: triangles of tri_idx, kind 1: edges of edge_idx) and their size statistics.
template <typename R>
__global__ void k_sc_boxes(int kind, int P, const pos4_t<R>* __restrict__ pos, const int4* __restrict__ tri_idx,
                           const int4* __restrict__ edge_idx, pos4_t<R>* lo, pos4_t<R>* hi, double* stats) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ext = 0.0;
  if (i < P) {
    vec3<R> a, b;
    if (kind == 0) {
      const int4 t = __ldg(tri_idx + i);
      const vec3<R> x0 = ld3<R>(pos[t.x]), x1 = ld3<R>(pos[t.y]), x2 = ld3<R>(pos[t.z]);
      a = {vmin(vmin(x0.x, x1.x), x2.x), vmin(vmin(x0.y, x1.y), x2.y), vmin(vmin(x0.z, x1.z), x2.z)};
      b = {vmax(vmax(x0.x, x1.x), x2.x), vmax(vmax(x0.y, x1.y), x2.y), vmax(vmax(x0.z, x1.z), x2.z)};
    } else {
      const int4 e = __ldg(edge_idx + i);
      const vec3<R> x0 = ld3<R>(pos[e.z]), x1 = ld3<R>(pos[e.w]);
      a = {vmin(x0.x, x1.x), vmin(x0.y, x1.y), vmin(x0.z, x1.z)};
      b = {vmax(x0.x, x1.x), vmax(x0.y, x1.y), vmax(x0.z, x1.z)};
    }
    lo[i] = pk4(a, R(0));
    hi[i] = pk4(b, R(0));
    ext = double(vmax(vmax(b.x - a.x, b.y - a.y), b.z - a.z));
    if (!(ext >= 0.0)) ext = 0.0;  // a NaN box does not size the grid
  }
  double s = ext, m = ext;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(stats, s);
    atomicMax((unsigned long long*)(stats + 1), (unsigned long long)__double_as_longlong(m));
  }
}

static __global__ void k_sc_cell(double* stats, int P, double margin) {
  const double mean = P > 0 ? stats[0] / P : 0.0;
  const double mx = __longlong_as_double((long long)*(unsigned long long*)(stats + 1));
  double c = fmax(2.0 * margin + mean, mx) * 1.01;
  if (!(c > 1e-9)) c = 1e-9;
  if (!(c < 1e30)) c = 1e30;
  stats[2] = c;
  stats[3] = 1.0 / c;
}

// insert (fill == false: count) every primitive into the cells its box overlaps
template <typename R, bool FILL>
__global__ void k_sc_grid(int P, const pos4_t<R>* __restrict__ lo, const pos4_t<R>* __restrict__ hi,
                          const double* __restrict__ stats, int nb, unsigned* bcount, const unsigned* __restrict__ bstart,
                          long long* ekey, int* eprim, long long gcap, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const double inv = stats[3];
  const pos4_t<R> a = lo[i], b = hi[i];
  const int x0 = cell_of(double(a.x), inv), y0 = cell_of(double(a.y), inv), z0 = cell_of(double(a.z), inv);
  int x1 = cell_of(double(b.x), inv), y1 = cell_of(double(b.y), inv), z1 = cell_of(double(b.z), inv);
  if (x1 > x0 + 1 || y1 > y0 + 1 || z1 > z0 + 1) {  // not reachable with the cell size above
    atomicOr(flags + 3, 1);
    x1 = min(x1, x0 + 1), y1 = min(y1, y0 + 1), z1 = min(z1, z0 + 1);
  }
  for (int x = x0; x <= x1; ++x)
    for (int y = y0; y <= y1; ++y)
      for (int z = z0; z <= z1; ++z) {
        const unsigned h = cell_hash(x, y, z, nb);
        const unsigned k = atomicAdd(bcount + h, 1u);
        if (FILL) {
          const long long slot = (long long)bstart[h] + k;
          if (slot < gcap) {
            ekey[slot] = cell_key(x, y, z);
            eprim[slot] = i;
          } else {
            atomicOr(flags + 3, 1);
          }
        }
      }
}

__device__ __forceinline__ bool sorted_contains(const int* __restrict__ off, const int* __restrict__ list, int row,
                                                int key) {
  if (!off) return false;
  int lo = __ldg(off + row), hi = __ldg(off + row + 1);
  if (hi <= lo || key < __ldg(list + lo) || key > __ldg(list + hi - 1)) return false;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(list + mid) > key)
      hi = mid;
    else
      lo = mid + 1;
  }
  return __ldg(list + hi - 1) == key;
}

// Keeps the `cap` smallest ids in ascending order; n = ids stored before this call (<= cap).
__device__ __forceinline__ void insert_smallest(int* list, int n, int cap, int id) {
  if (n == cap) {
    if (id >= list[cap - 1]) return;
    n = cap - 1;
  }
  int j = n - 1;
  while (j >= 0 && list[j] > id) {
    list[j + 1] = list[j];
    --j;
  }
  list[j + 1] = id;
}

struct ScQuery {
  int V, T, E, vb, eb, nb;
  float margin, rest_excl, ee_eps;
  const int4* tri_idx;
  const int4* edge_idx;
  const float* rest_q;  // model.particle_q (rest shape), V x 3
  const int *vt_foff, *vt_f, *ee_foff, *ee_f;
  const unsigned* bstart;
  const long long* ekey;
  const int* eprim;
  const double* stats;
  int* flags;
  unsigned gcap;  // grid entries written (bucket ranges are clamped to it)
  // triangle -> colliding vertices (the stand-alone detector's record_triangle_contacting_vertices); tv NULL = off
  const int* world;  // [V] instance key per vertex (pairs across instances skipped), or null
  int* tv;         // [T, tb] vertex ids, kept increasing, INT_MAX past the stored ones during the query
  int* tv_count;   // [T] pairs found (may exceed tb)
  float* tv_min;   // [T] minimum distance, as float bits (distances are >= 0, so integer order is value order)
  int tb;
};

// Triangle side of a vertex-triangle pair (vertex_triangle_collision_detection_kernel with its
// triangle_colliding_vertices buffers, geometry/kernels.py:1373-1384): count, minimum distance, and the vertex in
// the triangle's list, which keeps the tb smallest vertex ids in increasing order whatever the thread timing (a
// sorted insertion: slot j keeps the smallest id of those that reach it, the larger one moves on).
__device__ __forceinline__ void record_triangle_vertex(const ScQuery& s, int t, int v, float dist) {
  atomicAdd(s.tv_count + t, 1);
  atomicMin(reinterpret_cast<int*>(s.tv_min) + t, __float_as_int(dist));
  int* slot = s.tv + size_t(t) * s.tb;
  int val = v;
  for (int j = 0; j < s.tb; ++j) {
    const int old = atomicMin(slot + j, val);
    if (old == INT_MAX) return;
    val = max(old, val);
  }
  atomicOr(s.flags + 1, 1);  // TRI_COLLISION_BUFFER_OVERFLOW_INDEX
}

static __global__ void k_sc_tri_init(int T, int tb, int* tv, int* tv_count, float* tv_min, float radius) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < (long long)T * tb) tv[i] = INT_MAX;
  if (i < T) {
    tv_count[i] = 0;
    tv_min[i] = radius;
  }
}

// Slots past the stored vertices read -1.
static __global__ void k_sc_tri_finish(int T, int tb, int* tv) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < (long long)T * tb && tv[i] == INT_MAX) tv[i] = -1;
}

template <typename R>
__device__ __forceinline__ vec3<R> rest_at(const float* q, int i) {
  return {R(q[3 * i]), R(q[3 * i + 1]), R(q[3 * i + 2])};
}

// Narrow phase of one vertex against the triangle grid (vertex_triangle_collision_detection_kernel).
template <typename R>
__global__ void k_sc_query_vt(ScQuery s, const pos4_t<R>* __restrict__ pos, const pos4_t<R>* __restrict__ lo,
                              const pos4_t<R>* __restrict__ hi, int* vt_tri, int* vt_count, R* vt_min) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= s.V) return;
  const vec3<R> p = ld3<R>(pos[v]);
  const R m = R(s.margin);
  const vec3<R> qlo = {p.x - m, p.y - m, p.z - m}, qhi = {p.x + m, p.y + m, p.z + m};
  const double inv = s.stats[3];
  const int x0 = cell_of(double(qlo.x), inv), y0 = cell_of(double(qlo.y), inv), z0 = cell_of(double(qlo.z), inv);
  const int x1 = min(cell_of(double(qhi.x), inv), x0 + 3), y1 = min(cell_of(double(qhi.y), inv), y0 + 3),
            z1 = min(cell_of(double(qhi.z), inv), z0 + 3);
  int* list = vt_tri + size_t(v) * s.vb;
  int cnt = 0;
  R mn = m;
  for (int cx = x0; cx <= x1; ++cx)
    for (int cy = y0; cy <= y1; ++cy)
      for (int cz = z0; cz <= z1; ++cz) {
        const unsigned h = cell_hash(cx, cy, cz, s.nb);
        const long long key = cell_key(cx, cy, cz);
        const unsigned e0 = __ldg(s.bstart + h), e1 = min(__ldg(s.bstart + h + 1), s.gcap);
        for (unsigned e = e0; e < e1; ++e) {
          if (__ldg(s.ekey + e) != key) continue;
          const int t = __ldg(s.eprim + e);
          const pos4_t<R> a = lo[t], b = hi[t];
          if (a.x > qhi.x || a.y > qhi.y || a.z > qhi.z || b.x < qlo.x || b.y < qlo.y || b.z < qlo.z) continue;
          // report the pair from one cell only
          if (cell_of(double(vmax(qlo.x, R(a.x))), inv) != cx || cell_of(double(vmax(qlo.y, R(a.y))), inv) != cy ||
              cell_of(double(vmax(qlo.z, R(a.z))), inv) != cz)
            continue;
          const int4 ti = __ldg(s.tri_idx + t);
          if (v == ti.x || v == ti.y || v == ti.z) continue;
          if (s.world && __ldg(s.world + ti.x) != __ldg(s.world + v)) continue;
          if (sorted_contains(s.vt_foff, s.vt_f, v, t)) continue;
          R bary[3];
          const R dist = length(tri_closest(ld3<R>(pos[ti.x]), ld3<R>(pos[ti.y]), ld3<R>(pos[ti.z]), p, bary) - p);
          if (s.rest_excl > 0.f) {
            const vec3<R> rv = rest_at<R>(s.rest_q, v);
            R rb[3];
            const R dref = length(tri_closest(rest_at<R>(s.rest_q, ti.x), rest_at<R>(s.rest_q, ti.y),
                                              rest_at<R>(s.rest_q, ti.z), rv, rb) - rv);
            if (dref < R(s.rest_excl)) continue;
          }
          if (dist < m) {
            mn = vmin(mn, dist);
            insert_smallest(list, min(cnt, s.vb), s.vb, t);
            ++cnt;
            if (s.tv) record_triangle_vertex(s, t, v, float(dist));
          }
        }
      }
  if (cnt > s.vb) atomicOr(s.flags + 0, 1);
  vt_count[v] = cnt;
  vt_min[v] = mn;
}

// Narrow phase of one edge against the edge grid (edge_colliding_edges_detection_kernel).
template <typename R>
__global__ void k_sc_query_ee(ScQuery s, const pos4_t<R>* __restrict__ pos, const pos4_t<R>* __restrict__ lo,
                              const pos4_t<R>* __restrict__ hi, int* ee_edge, int* ee_count, R* ee_min) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= s.E) return;
  const int4 ei = __ldg(s.edge_idx + e);
  const vec3<R> p0 = ld3<R>(pos[ei.z]), p1 = ld3<R>(pos[ei.w]);
  const R m = R(s.margin);
  const pos4_t<R> ea = lo[e], eb_ = hi[e];
  const vec3<R> qlo = {R(ea.x) - m, R(ea.y) - m, R(ea.z) - m}, qhi = {R(eb_.x) + m, R(eb_.y) + m, R(eb_.z) + m};
  const double inv = s.stats[3];
  const int x0 = cell_of(double(qlo.x), inv), y0 = cell_of(double(qlo.y), inv), z0 = cell_of(double(qlo.z), inv);
  const int x1 = min(cell_of(double(qhi.x), inv), x0 + 3), y1 = min(cell_of(double(qhi.y), inv), y0 + 3),
            z1 = min(cell_of(double(qhi.z), inv), z0 + 3);
  int* list = ee_edge + size_t(e) * s.eb;
  int cnt = 0;
  R mn = m;
  for (int cx = x0; cx <= x1; ++cx)
    for (int cy = y0; cy <= y1; ++cy)
      for (int cz = z0; cz <= z1; ++cz) {
        const unsigned h = cell_hash(cx, cy, cz, s.nb);
        const long long key = cell_key(cx, cy, cz);
        const unsigned g0 = __ldg(s.bstart + h), g1 = min(__ldg(s.bstart + h + 1), s.gcap);
        for (unsigned g = g0; g < g1; ++g) {
          if (__ldg(s.ekey + g) != key) continue;
          const int f = __ldg(s.eprim + g);
          const pos4_t<R> a = lo[f], b = hi[f];
          if (a.x > qhi.x || a.y > qhi.y || a.z > qhi.z || b.x < qlo.x || b.y < qlo.y || b.z < qlo.z) continue;
          if (cell_of(double(vmax(qlo.x, R(a.x))), inv) != cx || cell_of(double(vmax(qlo.y, R(a.y))), inv) != cy ||
              cell_of(double(vmax(qlo.z, R(a.z))), inv) != cz)
            continue;
          const int4 fi = __ldg(s.edge_idx + f);
          if (ei.z == fi.z || ei.z == fi.w || ei.w == fi.z || ei.w == fi.w) continue;
          if (s.world && __ldg(s.world + fi.z) != __ldg(s.world + ei.z)) continue;
          if (sorted_contains(s.ee_foff, s.ee_f, e, f)) continue;
          R ss, tt, dist;
          edge_closest(p0, p1, ld3<R>(pos[fi.z]), ld3<R>(pos[fi.w]), R(s.ee_eps), ss, tt, dist);
          if (s.rest_excl > 0.f) {
            R rs, rt, dref;
            edge_closest(rest_at<R>(s.rest_q, ei.z), rest_at<R>(s.rest_q, ei.w), rest_at<R>(s.rest_q, fi.z),
                         rest_at<R>(s.rest_q, fi.w), R(s.ee_eps), rs, rt, dref);
            if (dref < R(s.rest_excl)) continue;
          }
          if (dist < m) {
            mn = vmin(mn, dist);
            insert_smallest(list, min(cnt, s.eb), s.eb, f);
            ++cnt;
          }
        }
      }
  if (cnt > s.eb) atomicOr(s.flags + 2, 1);
  ee_count[e] = cnt;
  ee_min[e] = mn;
}

// tmp[i] = number of stored pairs of primitive i (tmp[P] = 0 for the scan)
static __global__ void k_sc_stored(int P, int cap, const int* __restrict__ count, int* tmp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P) tmp[i] = min(count[i], cap);
  if (i == P) tmp[i] = 0;
}

// Dense pair lists: each pair stored as its four vertex ids, so that the solve and the truncation read a pair's
// positions one load after its entry. VT (vertex i, triangle t): (t0, t1, t2, i); EE (edge i, edge j): the
// vertices of i, then those of j.
template <bool EE>
__global__ void k_sc_pairs(int P, int cap, const int* __restrict__ count, const int* __restrict__ list,
                           const int* __restrict__ off, const int4* __restrict__ tri_idx,
                           const int4* __restrict__ edge_idx, int4* pairs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const int n = min(count[i], cap), o = off[i];
  const int4 a = EE ? __ldg(edge_idx + i) : make_int4(0, 0, 0, 0);
  for (int k = 0; k < n; ++k) {
    const int j = list[size_t(i) * cap + k];
    if (EE) {
      const int4 b = __ldg(edge_idx + j);
      pairs[o + k] = make_int4(a.z, a.w, b.z, b.w);
    } else {
      const int4 t = __ldg(tri_idx + j);
      pairs[o + k] = make_int4(t.x, t.y, t.z, i);
    }
  }
}

// Per-vertex entry lists. FILL == false counts, FILL == true writes through the cursors.
template <bool FILL>
__global__ void k_sc_entries(const int* __restrict__ n_vt, const int* __restrict__ n_ee, const int4* __restrict__ vt_pairs,
                             const int4* __restrict__ ee_pairs, int* cnt, const int* __restrict__ off, unsigned* ent,
                             long long ecap, int* flags) {
  const int nv = *n_vt, ne = *n_ee;
  auto put = [&](int vert, unsigned code) {
    const int k = atomicAdd(cnt + vert, 1);
    if (FILL) {
      const long long slot = (long long)off[vert] + k;
      if (slot < ecap)
        ent[slot] = code;
      else
        atomicOr(flags + 3, 1);
    }
  };
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv + ne; i += gridDim.x * blockDim.x) {
    if (i < nv) {
      const int4 q = vt_pairs[i];
      put(q.w, (3u << 29) | unsigned(i));
      put(q.x, (0u << 29) | unsigned(i));
      put(q.y, (1u << 29) | unsigned(i));
      put(q.z, (2u << 29) | unsigned(i));
    } else {
      const int j = i - nv;
      const int4 q = ee_pairs[j];
      put(q.x, 0x80000000u | (0u << 29) | unsigned(j));
      put(q.y, 0x80000000u | (1u << 29) | unsigned(j));
    }
  }
}

static __global__ void k_sc_sort_entries(int V, const int* __restrict__ off, unsigned* ent) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const int b = off[v], e = off[v + 1];
  for (int i = b + 1; i < e; ++i) {
    const unsigned key = ent[i];
    int j = i - 1;
    while (j >= b && ent[j] > key) {
      ent[j + 1] = ent[j];
      --j;
    }
    ent[j + 1] = key;
  }
}

// Copies the detection positions (and zeroes the displacements): the start of a detection.
template <typename R>
__global__ void k_sc_begin_from_state(int V, const R* __restrict__ q, pos4_t<R>* pos_cd, pos4_t<R>* disp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  pos_cd[i] = pk4(vec3<R>{q[3 * i], q[3 * i + 1], q[3 * i + 2]}, R(0));
  disp[i] = pk4(zero3<R>(), R(0));
}
template <typename R>
__global__ void k_sc_begin_from_pos(int V, const pos4_t<R>* __restrict__ pos, pos4_t<R>* pos_cd, pos4_t<R>* disp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  pos_cd[i] = pos[i];
  disp[i] = pk4(zero3<R>(), R(0));
}

// ------------------------------------------------------------------------------------ truncation
__device__ __forceinline__ void ts_min(float* ts, int i, float t) { atomicMin((unsigned*)(ts + i), __float_as_uint(t)); }
__device__ __forceinline__ void ts_min(double* ts, int i, double t) {
  atomicMin((unsigned long long*)(ts + i), (unsigned long long)__double_as_longlong(t));
}

// Step fractions of every recorded pair (apply_planar_truncation_parallel_by_collision): per vertex the
// minimum over its pairs. All fractions lie in [0, 1], so the minimum of their bit patterns is theirs.
// Division planes of one vertex-triangle (vt) or edge-edge pair and the step fractions of its vertices
// (apply_planar_truncation_parallel_by_collision, particle_vbd_kernels.py:2744-2874): the per-vertex minimum is
// kept with an integer atomicMin on the fraction's bits (fractions lie in [0, 1]).
template <typename R>
__device__ __forceinline__ void trunc_pair(bool vt, int4 q, const pos4_t<R>* __restrict__ pos_cd,
                                           const pos4_t<R>* __restrict__ disp, R eps, R gamma, R* ts) {
  // the vertex first for a VT pair (the planes' order), the stored order for an EE pair
  const int ids[4] = {vt ? q.w : q.x, vt ? q.x : q.y, vt ? q.y : q.z, vt ? q.z : q.w};
  vec3<R> x[4], dx[4], n, d;
  bool cut[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) x[k] = ld3<R>(pos_cd[ids[k]]), dx[k] = ld3<R>(disp[ids[k]]);
  if (vt)
    vt_plane(x, dx, cut, n, d);
  else
    ee_plane(x, dx, cut, n, d);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (cut[k]) {
      const R t = plane_t(x[k], dx[k], n, d, eps, gamma);
      if (t < R(1)) ts_min(ts, ids[k], t);
    }
}

// disp *= t, |disp| <= max_d, q = q_cd + disp (apply_truncation_ts); resets t to 1 for the next pass.
template <typename R>
__device__ __forceinline__ void trunc_vertex(int i, R* ts, R max_d, const pos4_t<R>* __restrict__ pos_cd,
                                             pos4_t<R>* disp, pos4_t<R>* pos) {
  const R t = ts[i];
  ts[i] = R(1);
  vec3<R> d = ld3<R>(disp[i]) * t;
  const R len = length(d);
  if (len > max_d) d = {d.x * max_d / len, d.y * max_d / len, d.z * max_d / len};
  disp[i] = pk4(d, R(0));
  pos[i] = pk4(ld3<R>(pos_cd[i]) + d, R(0));
}

template <typename R>
__global__ void k_sc_trunc_pairs(const int* __restrict__ n_vt, const int* __restrict__ n_ee,
                                 const int4* __restrict__ vt_pairs, const int4* __restrict__ ee_pairs,
                                 const pos4_t<R>* __restrict__ pos_cd, const pos4_t<R>* __restrict__ disp, R eps, R gamma,
                                 R* ts) {
  const int nv = *n_vt, ne = *n_ee;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv + ne; i += gridDim.x * blockDim.x)
    trunc_pair<R>(i < nv, i < nv ? vt_pairs[i] : ee_pairs[i - nv], pos_cd, disp, eps, gamma, ts);
}

template <typename R>
__global__ void k_sc_trunc_apply(int V, R* ts, R max_d, const pos4_t<R>* __restrict__ pos_cd, pos4_t<R>* disp,
                                 pos4_t<R>* pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < V) trunc_vertex<R>(i, ts, max_d, pos_cd, disp, pos);
}

template <typename R>
__global__ void k_sc_fill(int n, R* a, R v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

}  // namespace vbd
