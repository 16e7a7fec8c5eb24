// One-ring ("RING") layout of the per-vertex element data, and the solve that reads it.
//
// On a manifold triangle mesh the elements a vertex v belongs to are laid out around it: its incident
// triangles form a fan (v, r_0, r_1), (v, r_1, r_2), ... over the ordered ring r_0..r_{k-1} (closed when
// the last triangle comes back to r_0). Its hinges are the "spokes" (v, r_i), shared by the triangles on
// either side of r_i, and the "rims" (r_i, r_{i+1}), shared by triangle i and the outer triangle across
// the rim, whose third vertex is o_i. The ELL layouts store one record per incidence and recompute each
// hinge's two face normals from scratch (24 normals and 48 position gathers per interior vertex of a
// grid); here the walk round the fan computes each incident face normal once and uses it for the
// membrane, the two spokes and the rim of that face (12 normals and 12 position gathers).
//
// Records, slot-major per color range like the ELL layouts (slot i of vertex j of range r at
// base[r] + i * n[r] + j), 16-bit instance-local ids:
//   uint4 A: (r_i | o_i << 16, mu A, lambda A, D'00)      o_i = 0xffff when the rim has no hinge
//   uint4 B: (D'01, D'10, D'11, membrane damping)         D' = rest inverse re-expressed for (v, r_i, r_{i+1})
//   float4 H: (spoke rest angle, spoke ke l0, rim rest angle, rim ke l0)   zero stiffness: no hinge
//   per vertex: k | closed << 8
//   float2 kd: (spoke damping, rim damping), a side array present only when some hinge is damped; a damped
//   hinge is evaluated by the generic bending routine on its four positions (the shared normals carry no
//   velocity), which needs the positions at the start of the step
// Each hinge is evaluated in a fixed orientation: spoke i as (o0, o1, v0, v1) = (r_{i+1}, r_{i-1}, v, r_i)
// and rim i as (v, o_i, r_i, r_{i+1}). Swapping the two opposite vertices or the two edge vertices of a
// hinge negates the reference's dihedral angle (particle_vbd_kernels.py:1057-1190), so the rest angle is
// stored with the sign that makes k (theta - theta0)^2 / 2 the reference's energy.
#pragma once
#include "vbd_kernels.cuh"

namespace vbd {

constexpr int kRingMax = 8;  // triangles per vertex fan

struct RingView {
  const int* range_nslot;         // [ranges] slots of the range
  const long long* range_base;    // [ranges] first slot record of the range
  const long long* range_vbase;   // [ranges] first per-vertex header of the range
  const uint4* A;
  const uint4* B;
  const float4* H;
  const unsigned* hdr;
  const float2* kd;  // [slots] (spoke, rim) hinge damping; NULL when no hinge is damped
};

// A damped hinge in the ring's orientation (o0, o1, v0, v1), the solved vertex in role `role`: positions as
// offsets from the solved vertex x, ids for the positions at the start of the step.
template <typename R>
__device__ __forceinline__ void ring_damped_hinge(const StepCtx<R>& c, int role, vec3<R> x, const vec3<R> a[4],
                                                  const int id[4], R rest_angle, R k, R kd, vec3<R>& f, sym3<R>& H) {
  vec3<R> xs[4], xp[4];
  for (int q = 0; q < 4; ++q) {
    xs[q] = x + a[q];
    xp[q] = ld3<R>(c.qprev[id[q]]);
  }
  bending_add<R>(role, xs, rest_angle, R(1), k, kd, c.dt, xp, f, H);
}

// Dihedral angle of a hinge from its two face normals (unit) and its unit edge, in the reference's
// orientation convention: theta = atan2((n1 x n2) . e, n1 . n2).
template <typename R>
__device__ __forceinline__ R ring_theta(vec3<R> n1, vec3<R> n2, vec3<R> eh) {
  return vatan2(dot(cross(n1, n2), eh), dot(n1, n2));
}

template <typename R, int MODE, typename P>
__device__ __forceinline__ void solve_ring(const StepCtx<R>& c, const P& pos, const RingView& e, int r, int n, int j,
                                           int v, int vs, int iteration) {
  const pos4_t<R> in4 = c.inertia[v];
  const R m = R(in4.w);
  if (m == R(0)) return;
  const vec3<R> x = pos.ld(v);
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  const unsigned hd = __ldg(e.hdr + __ldg(e.range_vbase + r) + j);
  const int k = int(hd & 0xffu);
  const bool closed = (hd >> 8) & 1u;
  if (k > 0) {
    const long long b0 = __ldg(e.range_base + r) + j;
    const R eps2 = R(1.0e-12);
    // slot 0
    uint4 A = __ldg(e.A + b0);
    const int id_first = vs + int(A.x & 0xffffu);
    const vec3<R> a_first = pos.ld(id_first) - x;
    vec3<R> a_cur = a_first, a_prev = zero3<R>(), a_second = zero3<R>();
    int id_cur = id_first, id_prev = v, id_second = v;  // particle ids of r_i, r_{i-1}, r_1
    vec3<R> n_prev = zero3<R>(), n_first = zero3<R>();  // unit normals of faces i - 1 and 0
    R il_prev = R(0), il_first = R(0);                   // their inverse lengths (0: degenerate or absent)
    bool have_prev = false, have_first = false;
    float4 H0 = make_float4(0.f, 0.f, 0.f, 0.f);
    float kd0 = 0.f;  // spoke damping of slot 0
    for (int i = 0; i < k; ++i) {
      const long long bi = b0 + (long long)i * n;
      const uint4 B = __ldg(e.B + bi);
      const float4 Hh = __ldg(e.H + bi);
      const float2 hkd = e.kd ? __ldg(e.kd + bi) : make_float2(0.f, 0.f);
      if (i == 0) {
        H0 = Hh;
        kd0 = hkd.x;
      }
      const int inext = i + 1 < k ? i + 1 : (closed ? 0 : -1);
      uint4 An = A;
      vec3<R> a_next = zero3<R>();
      int id_next = v;
      if (inext > 0) {
        An = __ldg(e.A + b0 + (long long)inext * n);
        id_next = vs + int(An.x & 0xffffu);
        a_next = pos.ld(id_next) - x;
      } else if (inext == 0) {
        a_next = a_first;
        id_next = id_first;
      }
      bool have_face = false;
      vec3<R> n_cur = zero3<R>();
      R il_cur = R(0);
      if (inext >= 0) {
        // face i = (v, r_i, r_{i+1})
        const float muA = __uint_as_float(A.y), lmA = __uint_as_float(A.z);
        if (muA > 0.f || lmA > 0.f) {
          const R pose[4] = {R(__uint_as_float(A.w)), R(__uint_as_float(B.x)), R(__uint_as_float(B.y)),
                             R(__uint_as_float(B.z))};
          const float kd = __uint_as_float(B.w);
          vec3<R> xp[3];
          if (kd > 0.f) {
            xp[0] = ld3<R>(c.qprev[v]);
            xp[1] = ld3<R>(c.qprev[id_cur]);
            xp[2] = ld3<R>(c.qprev[id_next]);  // r_0's on the face that closes a fan
          }
          membrane_add<R>(0, zero3<R>(), a_cur, a_next, pose, R(muA), R(lmA), R(kd), R(1), c.dt, xp, f, H, R(0));
        }
        const vec3<R> N = cross(a_cur, a_next);
        const R s1 = dot(N, N);
        have_face = true;
        if (s1 >= eps2) {
          il_cur = vrsqrt(s1);
          n_cur = N * il_cur;
        }
        // rim hinge i: (v, o_i, r_i, r_{i+1}), the solved vertex is the first opposite vertex
        const float kr = Hh.w;
        const unsigned o = A.x >> 16;
        if (kr > 0.f && o != 0xffffu && hkd.y > 0.f) {
          const vec3<R> ha[4] = {zero3<R>(), pos.ld(vs + int(o)) - x, a_cur, a_next};
          const int hid[4] = {v, vs + int(o), id_cur, id_next};
          ring_damped_hinge<R>(c, 0, x, ha, hid, R(Hh.z), R(kr), R(hkd.y), f, H);
        } else if (kr > 0.f && o != 0xffffu && il_cur > R(0)) {
          const vec3<R> b = pos.ld(vs + int(o)) - x;
          const vec3<R> N2 = cross(a_next - b, a_cur - b);
          const vec3<R> ed = a_next - a_cur;
          const R s2 = dot(N2, N2), se = dot(ed, ed);
          if (s2 >= eps2 && se >= eps2) {
            const R il2 = vrsqrt(s2), ile = vrsqrt(se);
            const R theta = ring_theta(n_cur, N2 * il2, ed * ile);
            const R kk = R(kr);
            const vec3<R> d = n_cur * (-(se * ile) * il_cur);
            f = f + (-kk * (theta - R(Hh.z))) * d;
            souter_add(H, d, kk);
          }
        }
      }
      // spoke hinge i: (r_{i+1}, r_{i-1}, v, r_i) between faces i and i - 1 (slot 0 of a closed fan waits for
      // face k - 1)
      if (i == 0) {
        a_second = a_next;
        id_second = id_next;
        n_first = n_cur;
        il_first = il_cur;
        have_first = have_face;
      } else if (have_face && have_prev && Hh.y > 0.f && hkd.x > 0.f) {
        const vec3<R> ha[4] = {a_next, a_prev, zero3<R>(), a_cur};
        const int hid[4] = {id_next, id_prev, v, id_cur};
        ring_damped_hinge<R>(c, 2, x, ha, hid, R(Hh.x), R(Hh.y), R(hkd.x), f, H);
      } else if (have_face && have_prev && Hh.y > 0.f && il_cur > R(0) && il_prev > R(0)) {
        const R se = dot(a_cur, a_cur);
        if (se >= eps2) {
          const R ile = vrsqrt(se);
          const vec3<R> eh = a_cur * ile;
          const R theta = ring_theta(n_cur, n_prev, eh);
          const R kk = R(Hh.y);
          const vec3<R> d = n_cur * (dot(a_cur - a_next, eh) * il_cur) + n_prev * (dot(a_cur - a_prev, eh) * il_prev);
          f = f + (-kk * (theta - R(Hh.x))) * d;
          souter_add(H, d, kk);
        }
      }
      a_prev = a_cur;
      a_cur = a_next;
      id_prev = id_cur;
      id_cur = id_next;
      n_prev = n_cur;
      il_prev = il_cur;
      have_prev = have_face;
      A = An;
    }
    // spoke 0 of a closed fan: faces 0 and k - 1 (the last face computed, now in n_prev; a_prev and id_prev
    // are r_{k-1}'s)
    if (closed && have_first && have_prev && H0.y > 0.f && kd0 > 0.f) {
      const vec3<R> ha[4] = {a_second, a_prev, zero3<R>(), a_first};
      const int hid[4] = {id_second, id_prev, v, id_first};
      ring_damped_hinge<R>(c, 2, x, ha, hid, R(H0.x), R(H0.y), R(kd0), f, H);
    } else if (closed && have_first && have_prev && H0.y > 0.f && il_first > R(0) && il_prev > R(0)) {
      const R se = dot(a_first, a_first);
      if (se >= eps2) {
        const R ile = vrsqrt(se);
        const vec3<R> eh = a_first * ile;
        const R theta = ring_theta(n_first, n_prev, eh);
        const R kk = R(H0.y);
        // a_{-1} = a_{k-1}: a_prev after the loop is a_{k-1} (the loop's last shift set a_cur = a_first)
        const vec3<R> d =
            n_first * (dot(a_first - a_second, eh) * il_first) + n_prev * (dot(a_first - a_prev, eh) * il_prev);
        f = f + (-kk * (theta - R(H0.x))) * d;
        souter_add(H, d, kk);
      }
    }
  }
  const R md = m * c.dt2r;
  f = f + md * (ld3<R>(in4) - x);
  H.xx += md;
  H.yy += md;
  H.zz += md;
  vec3<R> dlt;
  double r2;
  const int ncont = c.has_contacts ? c.slot_cnt[v] : 0;
  const double det_used = contacts_and_solve<R, MODE>(c, v, ncont, x, f, H, nullptr, dlt, r2);
  if (MODE == MODE_MIXED && c.residual) residual_add(c.residual, iteration, r2);
  if (!isfinite(det_used)) {
    set_err(c.err, 1);
    return;
  }
  if (!(fabs(det_used) > 1e-8)) {
    set_err(c.err, 4);
    return;
  }
  const vec3<R> xn = x + dlt;
  if (!(isfinite(double(xn.x)) && isfinite(double(xn.y)) && isfinite(double(xn.z)))) {
    set_err(c.err, 1);
    return;
  }
  pos.st(v, xn);
}

template <typename R, int MODE, bool SMEM, int OCC>
__global__ void __launch_bounds__(OCC ? 256 : 512, OCC ? OCC : 1) k_persistent_ring(StepCtx<R> c, PersistentPlan p,
                                                                                   RingView e) {
  extern __shared__ float s_pos[];
  __shared__ int s_item;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(p.queue, 1);
    __syncthreads();
    const int q = s_item;
    if (q >= p.W) return;
    const int w = __ldg(p.inst_order + q);
    const int vs = __ldg(p.inst_vstart + w), ve = __ldg(p.inst_vstart + w + 1);
    using Pos = typename std::conditional<SMEM, SmemPos, GlobalPos<R>>::type;
    Pos pos;
    if constexpr (SMEM) {
      pos = SmemPos{s_pos, vs};
    } else {
      pos = GlobalPos<R>{c.pos};
    }
    for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) forward_particle(c, pos, i);
    __syncthreads();
    const int cb = __ldg(p.inst_cptr + w), ce = __ldg(p.inst_cptr + w + 1);
    for (int it = 0; it < p.iterations; ++it) {
      for (int col = cb; col + 1 < ce; ++col) {
        const int a = __ldg(p.color_ranges + col), b = __ldg(p.color_ranges + col + 1);
        const int r = col - w;
        for (int j = threadIdx.x; j < b - a; j += blockDim.x)
          solve_ring<R, MODE>(c, pos, e, r, b - a, j, __ldg(p.color_verts + a + j), vs, it);
        __syncthreads();
      }
    }
    for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) finalize_particle(c, pos, i);
  }
}

}  // namespace vbd
