// Stencil ("ELL") layout of the per-vertex element data, and the solve that reads it.
//
// The CSR path (vbd_kernels.cuh) reaches a triangle or hinge through the vertex adjacency and
// gathers its record by element id, so the 32 lanes of a warp touch 32 unrelated records. Here
// every (vertex, element) incidence gets its own record, prepared once per model, stored in the
// order in which the sweep visits the vertices and slot-major within a color range:
//     record(range r, slot s, vertex j of the range) at  base[r] + s * n[r] + j
// so that lane j of a warp reading slot s of consecutive vertices reads consecutive addresses, and no
// adjacency list sits on the dependent-load chain.
//
// Face record, with the solved vertex renumbered as vertex 0 of the triangle (cyclic order, so the
// orientation is kept):
//   int2   (a, b)            the other two vertices
//   float4 D'^-1             rest inverse re-expressed for that numbering: [x_a - x, x_b - x] D'^-1 = F
//   float2 (mu A, lambda A)  Lame coefficients times the rest area (the energy is homogeneous of degree
//                            one in (mu, lambda), so scaling both by the area scales force and Hessian)
//   float  damping           read only when the model has non-zero membrane damping
// Hinge record:
//   int4   (o0, o1, v0, v1)  with the solved vertex's role (0..3) in the top two bits of v1
//   float2 (rest angle, ke * rest length)
//   float  kd                read only when the model has non-zero bending damping
// Empty slots (vertices with fewer elements than the range's maximum) carry zero stiffness.
#pragma once
#include "vbd_kernels.cuh"
#include "vbd_pair.cuh"

namespace vbd {

// Stencil records are read once per sweep and never again before the next iteration: ask L2 for the
// records a few slots ahead (no registers held), and load them with the streaming hint so that they do
// not push the vertex positions out of L1. Two slots ahead measured best on the batched benchmark (31.2 ms per
// substep against 31.6 ms with three, 32.2 ms with five and 34.3 ms without the prefetch).
constexpr int kRecordPrefetch = 2;
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

struct EllView {
  const int* range_nf;    // [ranges] face slots of the range
  const int* range_ne;    // [ranges] hinge slots
  const long long* range_fbase;  // [ranges] first face record of the range
  const long long* range_ebase;  // [ranges] first hinge record
  const int2* face_nb;
  const float4* face_dm;
  const float2* face_mat;
  const float* face_kd;  // NULL when no membrane damping
  const int4* hinge_idx;
  const float2* hinge_prop;
  const float* hinge_kd;  // NULL when no bending damping
};

// One vertex (thread) of range r at position j (0-based within the range).
template <typename R, int MODE, typename P>
__device__ __forceinline__ void solve_ell(const StepCtx<R>& c, const P& pos, const EllView& e, int r, int n, int j,
                                          int v, int iteration) {
  const pos4_t<R> in4 = c.inertia[v];
  const R m = R(in4.w);
  if (m == R(0)) return;
  const vec3<R> x = pos.ld(v);
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  const int nf = __ldg(e.range_nf + r), ne = __ldg(e.range_ne + r);
  // Faces. The records of slot s + 1 are loaded while slot s is evaluated, so each thread keeps one
  // global load in flight under the element math.
  {
    const long long b0 = __ldg(e.range_fbase + r) + j;
    const float2* pm = e.face_mat + b0;
    const int2* pn = e.face_nb + b0;
    const float4* pd = e.face_dm + b0;
    for (int q = 1; q < kRecordPrefetch && q < nf; ++q) {
      prefetch_l2(pm + (long long)q * n);
      prefetch_l2(pn + (long long)q * n);
      prefetch_l2(pd + (long long)q * n);
    }
    const float* pk = e.face_kd ? e.face_kd + b0 : nullptr;
    float2 mat_n = make_float2(0.f, 0.f);
    int2 nb_n = make_int2(0, 0);
    float4 dm_n = make_float4(0.f, 0.f, 0.f, 0.f);
    if (nf > 0) {
      mat_n = __ldg(pm);
      nb_n = __ldg(pn);
      dm_n = __ldg(pd);
    }
    for (int s = 0; s < nf; ++s) {
      const float2 mat = mat_n;
      const int2 nb = nb_n;
      const float4 dm = dm_n;
      const float kd = pk ? __ldg(pk) : 0.f;
      if (s + kRecordPrefetch < nf) {
        prefetch_l2(pm + (long long)kRecordPrefetch * n);
        prefetch_l2(pn + (long long)kRecordPrefetch * n);
        prefetch_l2(pd + (long long)kRecordPrefetch * n);
      }
      if (s + 1 < nf) {
        pm += n;
        pn += n;
        pd += n;
        if (pk) pk += n;
        mat_n = __ldg(pm);
        nb_n = __ldg(pn);
        dm_n = __ldg(pd);
      }
      if (!(mat.x > 0.f || mat.y > 0.f)) continue;
      const R pose[4] = {R(dm.x), R(dm.y), R(dm.z), R(dm.w)};
      vec3<R> xp[3];
      if (kd > 0.f) {
        xp[0] = ld3<R>(c.qprev[v]);
        xp[1] = ld3<R>(c.qprev[nb.x]);
        xp[2] = ld3<R>(c.qprev[nb.y]);
      }
      membrane_add<R>(0, x, pos.ld(nb.x), pos.ld(nb.y), pose, R(mat.x), R(mat.y), R(kd), R(1), c.dt, xp, f, H, R(0));
    }
  }
  // Hinges, pipelined the same way.
  {
    const long long b0 = __ldg(e.range_ebase + r) + j;
    const float2* pp = e.hinge_prop + b0;
    const int4* pi = e.hinge_idx + b0;
    const float* pk = e.hinge_kd ? e.hinge_kd + b0 : nullptr;
    for (int q = 1; q < kRecordPrefetch && q < ne; ++q) {
      prefetch_l2(pp + (long long)q * n);
      prefetch_l2(pi + (long long)q * n);
    }
    float2 pr_n = make_float2(0.f, 0.f);
    int4 id_n = make_int4(0, 0, 0, 0);
    if (ne > 0) {
      pr_n = __ldg(pp);
      id_n = __ldg(pi);
    }
    for (int s = 0; s < ne; ++s) {
      const float2 pr = pr_n;
      const int4 id = id_n;
      const float kd = pk ? __ldg(pk) : 0.f;
      if (s + kRecordPrefetch < ne) {
        prefetch_l2(pp + (long long)kRecordPrefetch * n);
        prefetch_l2(pi + (long long)kRecordPrefetch * n);
      }
      if (s + 1 < ne) {
        pp += n;
        pi += n;
        if (pk) pk += n;
        pr_n = __ldg(pp);
        id_n = __ldg(pi);
      }
      if (!(pr.y > 0.f)) continue;
      const int ord = int((unsigned)id.w >> 30);
      const int v1 = id.w & 0x3fffffff;
      vec3<R> xs[4];
      xs[0] = pos.ld(id.x);
      xs[1] = pos.ld(id.y);
      xs[2] = pos.ld(id.z);
      xs[3] = pos.ld(v1);
      vec3<R> xp[4];
      if (kd > 0.f) {
        xp[0] = ld3<R>(c.qprev[id.x]);
        xp[1] = ld3<R>(c.qprev[id.y]);
        xp[2] = ld3<R>(c.qprev[id.z]);
        xp[3] = ld3<R>(c.qprev[v1]);
      }
      bending_add<R>(ord, xs, R(pr.x), R(1), R(pr.y), R(kd), c.dt, xp, f, H);
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

// Per-color launch: range r = color r; verts = the color's particles.
template <typename R, int MODE>
__global__ void k_color_ell(StepCtx<R> c, EllView e, const int* __restrict__ verts, int r, int n, int iteration) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  solve_ell<R, MODE>(c, GlobalPos<R>{c.pos}, e, r, n, j, __ldg(verts + j), iteration);
}

// One launch per substep, one CTA per instance at a time (ranges = the instance's colors).
// OCC > 0: compiled for OCC resident CTAs of 256 threads per SM (register budget 65536 / (256 OCC));
// OCC = 0: CTAs of up to 512 threads, up to 128 registers per thread.
template <typename R, int MODE, bool SMEM, int OCC>
__global__ void __launch_bounds__(OCC ? 256 : 512, OCC ? OCC : 1) k_persistent_ell(StepCtx<R> c, PersistentPlan p,
                                                                                  EllView e) {
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
        // range index of (instance, color) = col - w: each instance has one more range offset than ranges
        const int a = __ldg(p.color_ranges + col), b = __ldg(p.color_ranges + col + 1);
        const int r = col - w;
        for (int j = threadIdx.x; j < b - a; j += blockDim.x)
          solve_ell<R, MODE>(c, pos, e, r, b - a, j, __ldg(p.color_verts + a + j), it);
        __syncthreads();
      }
    }
    for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) finalize_particle(c, pos, i);
  }
}

}  // namespace vbd

namespace vbd {

// ---------------------------------------------------------------------------------------------
// Compact stencil records for instances of fewer than 65536 particles (persistent schedule):
// vertex ids are 16-bit offsets from the instance's first particle, so that
//   face  = 32 bytes in two 16-byte halves (two arrays, each read fully coalesced):
//           A = (a | b << 16, mu A, lambda A, D'00)      B = (D'01, D'10, D'11, damping)
//   hinge = 16 bytes: (o0 | o1 << 16, v0 | v1 << 16, rest angle, ke * rest length)
//           the hinge's four vertices in their (o0, o1, v0, v1) order; the solved vertex's role is the
//           place of its own id among them.
//   hinge damping kd: a float per hinge record in a side array, present only when some hinge of the model
//           is damped; the kernel variant that reads it (HD = true) adds the reference's Rayleigh term, which
//           needs the four vertices' positions at the start of the step.


struct Ell16View {
  const int* range_nf;
  const int* range_ne;
  const long long* range_fbase;
  const long long* range_ebase;
  const uint4* faceA;
  const uint4* faceB;
  const uint4* hinge;
  const float* hinge_kd;  // [hinge records]; NULL when no hinge is damped
};

// Membrane term of one 32-byte face record (A, B halves) for the solved vertex v at x.
template <typename R, typename P>
__device__ __forceinline__ void ell16_face(const StepCtx<R>& c, const P& pos, int v, int vs, vec3<R> x, uint4 A, uint4 B,
                                           vec3<R>& f, sym3<R>& H) {
  const float muA = __uint_as_float(A.y), lmA = __uint_as_float(A.z);
  if (!(muA > 0.f || lmA > 0.f)) return;
  const R pose[4] = {R(__uint_as_float(A.w)), R(__uint_as_float(B.x)), R(__uint_as_float(B.y)),
                     R(__uint_as_float(B.z))};
  const float kd = __uint_as_float(B.w);
  const int ia = vs + int(A.x & 0xffffu), ib = vs + int(A.x >> 16);
  vec3<R> xp[3];
  if (kd > 0.f) {
    xp[0] = ld3<R>(c.qprev[v]);
    xp[1] = ld3<R>(c.qprev[ia]);
    xp[2] = ld3<R>(c.qprev[ib]);
  }
  membrane_add<R>(0, x, pos.ld(ia), pos.ld(ib), pose, R(muA), R(lmA), R(kd), R(1), c.dt, xp, f, H, R(0));
}

// Bending term of one 16-byte hinge record for the solved vertex (instance-local id lv): the record lists the
// hinge's four vertices in their (o0, o1, v0, v1) order, so the solved vertex's role is where lv appears and all
// four positions are gathered (the solved vertex's own gather reads its current position).
// HD: the model has damped hinges; kd is this record's damping (0 for an undamped hinge), and a damped hinge
// reads the four vertices' positions at the start of the step (c.qprev).
template <typename R, bool HD, typename P>
__device__ __forceinline__ void ell16_hinge(const StepCtx<R>& c, const P& pos, int vs, int lv, uint4 hh, float kd,
                                            vec3<R>& f, sym3<R>& H) {
  const float k = __uint_as_float(hh.w);
  if (!(k > 0.f)) return;
  const int i0 = int(hh.x & 0xffffu), i1 = int(hh.x >> 16), i2 = int(hh.y & 0xffffu), i3 = int(hh.y >> 16);
  // the solved vertex's role is where its id appears; the role constants of bending_add_coef straight from it
  const bool r0 = i0 == lv, r1 = i1 == lv, r2 = i2 == lv, r3 = !(r0 || r1 || r2);
  const R ca = r0 ? R(-1) : (r2 ? R(1) : R(0));
  const R cb = r1 ? R(-1) : (r3 ? R(1) : R(0));
  const R dd = r2 ? R(1) : (r3 ? R(-1) : R(0));
  vec3<R> xs[4];
  xs[0] = pos.ld(vs + i0);
  xs[1] = pos.ld(vs + i1);
  xs[2] = pos.ld(vs + i2);
  xs[3] = pos.ld(vs + i3);
  if constexpr (HD) {
    if (kd > 0.f) {
      vec3<R> xp[4];
      xp[0] = ld3<R>(c.qprev[vs + i0]);
      xp[1] = ld3<R>(c.qprev[vs + i1]);
      xp[2] = ld3<R>(c.qprev[vs + i2]);
      xp[3] = ld3<R>(c.qprev[vs + i3]);
      bending_add_coef<R>(ca, cb, dd, xs, R(__uint_as_float(hh.z)), R(1), R(k), R(kd), c.dt, xp, f, H);
      return;
    }
  }
  bending_add_coef<R>(ca, cb, dd, xs, R(__uint_as_float(hh.z)), R(1), R(k), R(0), c.dt, nullptr, f, H);
}

template <typename R, int MODE, bool HD, typename P>
__device__ __forceinline__ void solve_ell16(const StepCtx<R>& c, const P& pos, const Ell16View& e, int r, int n, int j,
                                            int v, int vs, int iteration) {
  const pos4_t<R> in4 = c.inertia[v];
  const R m = R(in4.w);
  if (m == R(0)) return;
  // the contact count is read now, so that its load is in flight during the element loops
  const int ncont = c.has_contacts ? c.slot_cnt[v] : 0;
  const vec3<R> x = pos.ld(v);
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  const int nf = __ldg(e.range_nf + r), ne = __ldg(e.range_ne + r);
  const long long fb = __ldg(e.range_fbase + r) + j, eb = __ldg(e.range_ebase + r) + j;
  {
    {
      const uint4* pa = e.faceA + fb;
      const uint4* pb = e.faceB + fb;
      uint4 A_n = make_uint4(0u, 0u, 0u, 0u), B_n = make_uint4(0u, 0u, 0u, 0u);
      if (nf > 0) {
        A_n = __ldcs(pa);
        B_n = __ldcs(pb);
      }
      for (int q = 1; q < kRecordPrefetch && q < nf; ++q) {
        prefetch_l2(pa + (long long)q * n);
        prefetch_l2(pb + (long long)q * n);
      }
      for (int s = 0; s < nf; ++s) {
        const uint4 A = A_n, B = B_n;
        if (s + kRecordPrefetch < nf) {
          prefetch_l2(pa + (long long)kRecordPrefetch * n);
          prefetch_l2(pb + (long long)kRecordPrefetch * n);
        }
        if (s + 1 < nf) {
          pa += n;
          pb += n;
          A_n = __ldcs(pa);
          B_n = __ldcs(pb);
        }
        ell16_face<R>(c, pos, v, vs, x, A, B, f, H);
      }
    }
    {
      const uint4* ph = e.hinge + eb;
      const float* pk = HD ? e.hinge_kd + eb : nullptr;
      uint4 h_n = make_uint4(0u, 0u, 0u, 0u);
      if (ne > 0) h_n = __ldcs(ph);
      for (int q = 1; q < kRecordPrefetch && q < ne; ++q) prefetch_l2(ph + (long long)q * n);
      for (int s = 0; s < ne; ++s) {
        const uint4 hh = h_n;
        float kd = 0.f;
        if constexpr (HD) {
          kd = __ldcs(pk);
          pk += n;
        }
        if (s + kRecordPrefetch < ne) prefetch_l2(ph + (long long)kRecordPrefetch * n);
        if (s + 1 < ne) {
          ph += n;
          h_n = __ldcs(ph);
        }
        ell16_hinge<R, HD>(c, pos, vs, v - vs, hh, kd, f, H);
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

// Two vertices of one color range (records j0 and j1, particles v0 and v1) solved together, one per lane of
// the paired FP32 arithmetic of vbd_pair.cuh: the same terms, order and 3x3 solve as solve_ell16 in FP32. When
// has1 is false lane 1 repeats lane 0 and is discarded. A face with damping falls back to the scalar membrane
// for that slot. Contacts and the checks of the solve run per lane.
template <typename P>
__device__ __forceinline__ void solve_ell16_pair(const StepCtx<float>& c, const P& pos, const Ell16View& e, int r, int n,
                                                 int j0, int j1, int v0, int v1, bool has1, int vs) {
  const float4 in0 = c.inertia[v0], in1 = c.inertia[v1];
  const bool act0 = in0.w != 0.f, act1 = has1 && in1.w != 0.f;
  if (!act0 && !act1) return;
  const vec3<float> xs0 = pos.ld(v0), xs1 = pos.ld(v1);
  const pv3 x = pv3_of(xs0, xs1);
  pv3 f = {pfs(0.f), pfs(0.f), pfs(0.f)};
  psym H = {pfs(0.f), pfs(0.f), pfs(0.f), pfs(0.f), pfs(0.f), pfs(0.f)};
  const int nf = __ldg(e.range_nf + r), ne = __ldg(e.range_ne + r);
  const long long fb = __ldg(e.range_fbase + r);
  {
    const uint4* pa = e.faceA + fb;
    const uint4* pb = e.faceB + fb;
    for (int q = 0; q < kRecordPrefetch && q < nf; ++q) {
      prefetch_l2(pa + (long long)q * n + j0);
      prefetch_l2(pb + (long long)q * n + j0);
      prefetch_l2(pa + (long long)q * n + j1);
      prefetch_l2(pb + (long long)q * n + j1);
    }
    for (int s = 0; s < nf; ++s, pa += n, pb += n) {
      if (s + kRecordPrefetch < nf) {
        prefetch_l2(pa + (long long)kRecordPrefetch * n + j0);
        prefetch_l2(pb + (long long)kRecordPrefetch * n + j0);
        prefetch_l2(pa + (long long)kRecordPrefetch * n + j1);
        prefetch_l2(pb + (long long)kRecordPrefetch * n + j1);
      }
      const uint4 A0 = __ldcs(pa + j0), B0 = __ldcs(pb + j0), A1 = __ldcs(pa + j1), B1 = __ldcs(pb + j1);
      if (__uint_as_float(B0.w) > 0.f || __uint_as_float(B1.w) > 0.f) {
        // damped face: scalar membrane per lane
        vec3<float> fl = zero3<float>();
        sym3<float> hl = szero<float>();
        ell16_face<float>(c, pos, v0, vs, xs0, A0, B0, fl, hl);
        f.x.v.x += fl.x, f.y.v.x += fl.y, f.z.v.x += fl.z;
        H.xx.v.x += hl.xx, H.yy.v.x += hl.yy, H.zz.v.x += hl.zz, H.xy.v.x += hl.xy, H.xz.v.x += hl.xz, H.yz.v.x += hl.yz;
        fl = zero3<float>();
        hl = szero<float>();
        ell16_face<float>(c, pos, v1, vs, xs1, A1, B1, fl, hl);
        f.x.v.y += fl.x, f.y.v.y += fl.y, f.z.v.y += fl.z;
        H.xx.v.y += hl.xx, H.yy.v.y += hl.yy, H.zz.v.y += hl.zz, H.xy.v.y += hl.xy, H.xz.v.y += hl.xz, H.yz.v.y += hl.yz;
        continue;
      }
      float mu0 = __uint_as_float(A0.y), lm0 = __uint_as_float(A0.z);
      float mu1 = __uint_as_float(A1.y), lm1 = __uint_as_float(A1.z);
      const bool on0 = mu0 > 0.f || lm0 > 0.f, on1 = mu1 > 0.f || lm1 > 0.f;
      if (!on0 && !on1) continue;
      if (!on0) mu0 = lm0 = 0.f;  // an inactive face in one lane adds exactly zero
      if (!on1) mu1 = lm1 = 0.f;
      const pv3 xa = pv3_of(pos.ld(vs + int(A0.x & 0xffffu)), pos.ld(vs + int(A1.x & 0xffffu)));
      const pv3 xb = pv3_of(pos.ld(vs + int(A0.x >> 16)), pos.ld(vs + int(A1.x >> 16)));
      pmembrane_add(x, xa, xb, pf2(__uint_as_float(A0.w), __uint_as_float(A1.w)),
                    pf2(__uint_as_float(B0.x), __uint_as_float(B1.x)), pf2(__uint_as_float(B0.y), __uint_as_float(B1.y)),
                    pf2(__uint_as_float(B0.z), __uint_as_float(B1.z)), pf2(mu0, mu1), pf2(lm0, lm1), f, H);
    }
  }
  {
    const uint4* ph = e.hinge + __ldg(e.range_ebase + r);
    for (int q = 0; q < kRecordPrefetch && q < ne; ++q) {
      prefetch_l2(ph + (long long)q * n + j0);
      prefetch_l2(ph + (long long)q * n + j1);
    }
    for (int s = 0; s < ne; ++s, ph += n) {
      if (s + kRecordPrefetch < ne) {
        prefetch_l2(ph + (long long)kRecordPrefetch * n + j0);
        prefetch_l2(ph + (long long)kRecordPrefetch * n + j1);
      }
      const uint4 h0 = __ldcs(ph + j0), h1 = __ldcs(ph + j1);
      float k0 = __uint_as_float(h0.w), k1 = __uint_as_float(h1.w);
      const bool on0 = k0 > 0.f, on1 = k1 > 0.f;
      if (!on0 && !on1) continue;
      if (!on0) k0 = 0.f;
      if (!on1) k1 = 0.f;
      const int lv0 = v0 - vs, lv1 = v1 - vs;
      const int a0 = int(h0.x & 0xffffu), a1 = int(h0.x >> 16), a2 = int(h0.y & 0xffffu), a3 = int(h0.y >> 16);
      const int b0 = int(h1.x & 0xffffu), b1 = int(h1.x >> 16), b2 = int(h1.y & 0xffffu), b3 = int(h1.y >> 16);
      const int role0 = a0 == lv0 ? 0 : (a1 == lv0 ? 1 : (a2 == lv0 ? 2 : 3));
      const int role1 = b0 == lv1 ? 0 : (b1 == lv1 ? 1 : (b2 == lv1 ? 2 : 3));
      const pv3 xh[4] = {pv3_of(pos.ld(vs + a0), pos.ld(vs + b0)), pv3_of(pos.ld(vs + a1), pos.ld(vs + b1)),
                         pv3_of(pos.ld(vs + a2), pos.ld(vs + b2)), pv3_of(pos.ld(vs + a3), pos.ld(vs + b3))};
      pbending_add(xh, pf2(__uint_as_float(h0.z), __uint_as_float(h1.z)), pf2(k0, k1), role0, role1, f, H);
    }
  }
  const pf md = pf2(in0.w, in1.w) * pfs(c.dt2r);
  f = pfma(pv3_of(vec3<float>{in0.x, in0.y, in0.z}, vec3<float>{in1.x, in1.y, in1.z}) - x, md, f);
  H.xx = H.xx + md;
  H.yy = H.yy + md;
  H.zz = H.zz + md;
  if (c.has_contacts) {
    vec3<float> fl = lane0(f);
    sym3<float> hl = lane0(H);
    if (act0) contacts_add<float>(c, v0, xs0, fl, hl);
    vec3<float> fr = lane1(f);
    sym3<float> hr = lane1(H);
    if (act1) contacts_add<float>(c, v1, xs1, fr, hr);
    f = pv3_of(fl, fr);
    H = {pf2(hl.xx, hr.xx), pf2(hl.yy, hr.yy), pf2(hl.zz, hr.zz), pf2(hl.xy, hr.xy), pf2(hl.xz, hr.xz), pf2(hl.yz, hr.yz)};
  }
  // 3x3 solve by adjugate (sdet, sadj_mul)
  const pf cxx = pfms(H.yz, H.yz, H.yy * H.zz), cyy = pfms(H.xz, H.xz, H.xx * H.zz), czz = pfms(H.xy, H.xy, H.xx * H.yy);
  const pf cxy = pfms(H.xy, H.zz, H.xz * H.yz), cxz = pfms(H.xz, H.yy, H.xy * H.yz), cyz = pfms(H.xx, H.yz, H.xy * H.xz);
  const pf det = pfma(H.xz, cxz, pfma(H.xy, cxy, H.xx * cxx));
  const pv3 ad = {pfma(cxz, f.z, pfma(cxy, f.y, cxx * f.x)), pfma(cyz, f.z, pfma(cyy, f.y, cxy * f.x)),
                  pfma(czz, f.z, pfma(cyz, f.y, cxz * f.x))};
  const pf inv = pdiv(pfs(1.f), det);
  const pv3 xn = pfma(ad, inv, x);
  const vec3<float> xn0 = lane0(xn), xn1 = lane1(xn);
  const float d0 = det.v.x, d1 = det.v.y;
  if (act0) {
    if (!isfinite(d0)) set_err(c.err, 1);
    else if (!(fabsf(d0) > 1e-8f)) set_err(c.err, 4);
    else if (!(isfinite(xn0.x) && isfinite(xn0.y) && isfinite(xn0.z))) set_err(c.err, 1);
    else pos.st(v0, xn0);
  }
  if (act1) {
    if (!isfinite(d1)) set_err(c.err, 1);
    else if (!(fabsf(d1) > 1e-8f)) set_err(c.err, 4);
    else if (!(isfinite(xn1.x) && isfinite(xn1.y) && isfinite(xn1.z))) set_err(c.err, 1);
    else pos.st(v1, xn1);
  }
}

// PAIR (FP32 only): each thread solves two vertices of a color at once with paired FP32 instructions
// (solve_ell16_pair).
// HD (not with PAIR): the model has damped hinges (Ell16View::hinge_kd).
template <typename R, int MODE, bool SMEM, int OCC, bool PAIR = false, bool HD = false>
__global__ void __launch_bounds__(OCC ? 256 : 512, OCC ? OCC : 1) k_persistent_ell16(StepCtx<R> c, PersistentPlan p,
                                                                                    Ell16View e) {
  static_assert(!(PAIR && HD), "the paired kernel does not evaluate hinge damping");
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
        if constexpr (PAIR) {
          const int bd = blockDim.x;
          for (int j = threadIdx.x; j < b - a; j += 2 * bd) {
            const bool has1 = j + bd < b - a;
            const int v0 = __ldg(p.color_verts + a + j);
            const int v1 = has1 ? __ldg(p.color_verts + a + j + bd) : v0;
            solve_ell16_pair(c, pos, e, r, b - a, j, has1 ? j + bd : j, v0, v1, has1, vs);
          }
        } else {
          for (int j = threadIdx.x; j < b - a; j += blockDim.x)
            solve_ell16<R, MODE, HD>(c, pos, e, r, b - a, j, __ldg(p.color_verts + a + j), vs, it);
        }
        __syncthreads();
      }
    }
    for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) finalize_particle(c, pos, i);
  }
}

}  // namespace vbd
