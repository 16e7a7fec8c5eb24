// Hand-written adjoint of the fixed-iteration VBD step (one substep: membrane, bending, tetrahedra and springs
// with their damping, particle-shape contacts on static shapes).
//
// Forward map of one substep (vbd_kernels.cuh, CSR path, one lane per vertex):
//   y   = q + (qd + (g + f_ext / m) dt) dt                    inertial target, also the first iterate
//   for it < I, for color c, for v in c (Jacobi within the color, positions x of the color's start):
//       g_v = (m / dt^2)(y_v - x_v) + sum_e f_e,v(x),   H_v = (m / dt^2) I + sum_e H_e,v(x)
//       x_v <- x_v + H_v^-1 g_v          (skipped when |det H_v| <= 1e-8)
//   q_out = x,   qd_out = (x - q) / dt
//
// Reverse of one color update x' = x + D(x), D_v = H_v^-1 g_v, given the adjoint a = dL/dx':
//   w = H_v^-1 a_v        (H_v is symmetric)
//   dL/dg_v = w,   dL/dH_v = -w D_v^T   (only its symmetric part meets the symmetric dH)
//   dL/dx = a + [dg_v/dx]^T w + [dH_v/dx] : (-w D_v^T),   likewise for y and the element parameters.
// The element terms f_e,v and H_e,v are differentiated with forward-mode dual numbers over the
// element's vertex coordinates (and the triangle's mu, lambda), running the same element routines
// as the forward pass. Vertices of one color are never neighbours, so the vertices written through
// atomics (the neighbours, the triangle parameters) are never read by the same launch.
// A contact term and a damped element depend on positions x and, through friction and damping, on the
// positions at the start of the substep, q; the derivatives in q are accumulated per vertex (adj_xp) and
// join dL/dq_in at the end. The contact set, the contact points and normals and the penalty
// stiffness are held fixed (the derivative of the step for its contacts; the AVBD ramp is off).
#pragma once
#include "vbd_dual.cuh"
#include "vbd_kernels.cuh"

namespace vbd {

template <typename R>
struct AdjCtx {
  StepCtx<R> c;           // model arrays (CSR) and dt
  const R* x;             // [V*3] positions at the start of the color (the forward state)
  const R* y;             // [V*3] inertial targets
  R* adj_x;               // [V*3] in: dL/dx', out: dL/dx (in place)
  R* adj_y;               // [V*3] accumulated dL/dy
  R* adj_mu;              // [T] accumulated dL/dmu (triangle), may be NULL
  R* adj_lambda;          // [T] accumulated dL/dlambda, may be NULL
  R* adj_xp;              // [V*3] accumulated dL/dq through the contact terms (contacts only)
};

// mass used by the solve (0 for a fixed particle), as forward_particle stores it
template <typename R>
__device__ __forceinline__ R solve_mass(const StepCtx<R>& c, int v) {
  const float m = c.mass[v];
  return ((c.flags[v] & 1) && m != 0.f) ? R(m) : R(0);
}

template <typename R>
__device__ __forceinline__ vec3<R> ldx(const R* a, int i) {
  return {a[3 * i], a[3 * i + 1], a[3 * i + 2]};
}

template <typename R>
__device__ __forceinline__ void atomic_add3(R* a, int i, vec3<R> v) {
  atomicAdd(a + 3 * i, v.x);
  atomicAdd(a + 3 * i + 1, v.y);
  atomicAdd(a + 3 * i + 2, v.z);
}

// <g_bar, df> + <H_bar, dH> for one derivative slot k (H_bar symmetric, stored as 6 with the
// off-diagonal entries counted twice)
template <typename R, int N>
__device__ __forceinline__ R contract(const vec3<Dual<R, N>>& f, const sym3<Dual<R, N>>& H, vec3<R> gb,
                                      const sym3<R>& Hb, int k) {
  return gb.x * f.x.d[k] + gb.y * f.y.d[k] + gb.z * f.z.d[k] + Hb.xx * H.xx.d[k] + Hb.yy * H.yy.d[k] +
         Hb.zz * H.zz.d[k] + R(2) * (Hb.xy * H.xy.d[k] + Hb.xz * H.xz.d[k] + Hb.yz * H.yz.d[k]);
}

template <typename R>
__device__ __forceinline__ void assemble(const StepCtx<R>& c, const R* X, int v, vec3<R>& f, sym3<R>& H) {
  for (int a = c.face_off[v]; a < c.face_off[v + 1]; ++a) {
    const int t = c.face_adj[a] >> 2, ord = c.face_adj[a] & 3;
    const float4 mat = c.tri_mat[t];
    if (!(mat.x > 0.f || mat.y > 0.f)) continue;
    const int4 ti = c.tri_idx[t];
    const float4 dm = c.tri_pose[t];
    const R pose[4] = {R(dm.x), R(dm.y), R(dm.z), R(dm.w)};
    vec3<R> xp[3];
    if (mat.z > 0.f) xp[0] = ld3<R>(c.qprev[ti.x]), xp[1] = ld3<R>(c.qprev[ti.y]), xp[2] = ld3<R>(c.qprev[ti.z]);
    membrane_add<R>(ord, ldx(X, ti.x), ldx(X, ti.y), ldx(X, ti.z), pose, R(mat.x), R(mat.y), R(mat.z), R(mat.w), c.dt,
                    xp, f, H);
  }
  for (int a = c.edge_off[v]; a < c.edge_off[v + 1]; ++a) {
    const int e = c.edge_adj[a] >> 2, ord = c.edge_adj[a] & 3;
    const float4 pr = c.edge_prop[e];
    if (!(pr.z > 0.f)) continue;
    const int4 ei = c.edge_idx[e];
    const vec3<R> xs[4] = {ldx(X, ei.x), ldx(X, ei.y), ldx(X, ei.z), ldx(X, ei.w)};
    vec3<R> xp[4];
    if (pr.w > 0.f)
      xp[0] = ld3<R>(c.qprev[ei.x]), xp[1] = ld3<R>(c.qprev[ei.y]), xp[2] = ld3<R>(c.qprev[ei.z]),
      xp[3] = ld3<R>(c.qprev[ei.w]);
    bending_add<R>(ord, xs, R(pr.x), R(pr.y), R(pr.z), R(pr.w), c.dt, xp, f, H);
  }
  if (c.tet_off) {  // tetrahedra (solve_elasticity adds them after the hinges)
    for (int a = c.tet_off[v]; a < c.tet_off[v + 1]; ++a) {
      const int t = c.tet_adj[a] >> 2, ord = c.tet_adj[a] & 3;
      const float4 r0 = c.tet_pose[3 * t], r1 = c.tet_pose[3 * t + 1], r2 = c.tet_pose[3 * t + 2];
      if (!(r0.w > 0.f || r1.w > 0.f)) continue;
      const int4 ti = c.tet_idx[t];
      const R dm[9] = {R(r0.x), R(r0.y), R(r0.z), R(r1.x), R(r1.y), R(r1.z), R(r2.x), R(r2.y), R(r2.z)};
      const vec3<R> xs[4] = {ldx(X, ti.x), ldx(X, ti.y), ldx(X, ti.z), ldx(X, ti.w)};
      vec3<R> xp[4];
      if (r2.w > 0.f)
        xp[0] = ld3<R>(c.qprev[ti.x]), xp[1] = ld3<R>(c.qprev[ti.y]), xp[2] = ld3<R>(c.qprev[ti.z]),
        xp[3] = ld3<R>(c.qprev[ti.w]);
      tet_add<R>(ord, xs, xp, dm, R(r0.w), R(r1.w), R(r2.w), c.dt, f, H);
    }
  }
  if (c.spr_off) {  // springs to other colors, then springs within the color: all at the color's start state
    for (int pass = 0; pass < 2; ++pass) {
      const int* off = pass == 0 ? c.spr_off : c.sspr_off;
      const int* adj = pass == 0 ? c.spr_adj : c.sspr_adj;
      for (int a = off[v]; a < off[v + 1]; ++a) {
        const int sp = adj[a] >> 1, end = adj[a] & 1;
        const int2 ij = c.spr_idx[sp];
        const float4 pr = c.spr_prop[sp];
        const vec3<R> xa = pr.z != 0.f ? ld3<R>(c.qprev[v]) : zero3<R>();
        spring_add<R>(end, ldx(X, v), ldx(X, end == 0 ? ij.y : ij.x), xa, R(pr.x), R(pr.y), R(pr.z), c.dt, f, H);
      }
    }
  }
}

// element and contact terms of vertex v at positions X (the forward pass of the adjoint's sweep)
template <typename R>
__device__ __forceinline__ void assemble_all(const StepCtx<R>& c, const R* X, int v, vec3<R>& f, sym3<R>& H) {
  assemble(c, X, v, f, H);
  if (c.has_contacts) contacts_add<R>(c, v, ldx(X, v), f, H);
}

// Contact terms of vertex v with dual numbers over its position x (slots 0-2) and its position at the start of the
// substep (slots 3-5, c.qprev), as contacts_add_n evaluates them for static shapes; their derivatives contracted
// with (w, H_bar) add to ax and to adj_xp.
template <typename R>
__device__ __forceinline__ void contacts_adjoint(const StepCtx<R>& c, int v, vec3<R> x, vec3<R> w, const sym3<R>& Hb,
                                                 vec3<R>& ax, R* adj_xp) {
  int n = c.slot_cnt[v];
  if (n > c.K) n = c.K;
  if (n <= 0) return;
  using D6 = Dual<R, 6>;
  const vec3<R> xp = ld3<R>(c.qprev[v]);
  const vec3<D6> xd = {D6::seed(x.x, 0), D6::seed(x.y, 1), D6::seed(x.z, 2)};
  const vec3<D6> xpd = {D6::seed(xp.x, 3), D6::seed(xp.y, 4), D6::seed(xp.z, 5)};
  const D6 r = D6(R(c.radius[v]));
  const D6 dt = D6(c.dt);
  vec3<R> gxp = zero3<R>();
  for (int j = 0; j < n; ++j) {
    const int t = c.slots[v * c.K + j];
    const vec3<D6> bx = {D6(R(c.c_body_pos[3 * t])), D6(R(c.c_body_pos[3 * t + 1])), D6(R(c.c_body_pos[3 * t + 2]))};
    const vec3<D6> nn = {D6(R(c.c_normal[3 * t])), D6(R(c.c_normal[3 * t + 1])), D6(R(c.c_normal[3 * t + 2]))};
    const D6 pen = -(dot(nn, xd - bx) - r);
    if (!(pen > D6(R(0)))) continue;
    const vec3<D6> bv = {D6(R(c.c_body_vel[3 * t])), D6(R(c.c_body_vel[3 * t + 1])), D6(R(c.c_body_vel[3 * t + 2]))};
    const vec3<D6> rel = (xd - xpd) - bv * dt;
    vec3<D6> fd = {D6(R(0)), D6(R(0)), D6(R(0))};
    sym3<D6> Hd = szero<D6>();
    contact_add<D6>(pen, nn, rel, D6(R(c.c_k[t])), D6(R(c.c_kd[t])), D6(R(c.c_mu[t])), D6(c.fric_eps), dt, fd, Hd);
    ax = ax + vec3<R>{contract(fd, Hd, w, Hb, 0), contract(fd, Hd, w, Hb, 1), contract(fd, Hd, w, Hb, 2)};
    gxp = gxp + vec3<R>{contract(fd, Hd, w, Hb, 3), contract(fd, Hd, w, Hb, 4), contract(fd, Hd, w, Hb, 5)};
  }
  atomic_add3(adj_xp, v, gxp);  // neighbours' damped elements add to the same entry in this launch
}

// dL/dx of an element's vertices from its dual-number terms: slot 3j+k of vertex j (the solved vertex's part to ax,
// the others through atomics) and, from slot `sp` on, of the vertices' start positions into adj_xp.
template <typename R, int N>
__device__ __forceinline__ void scatter_element(const AdjCtx<R>& A, int v, const int* vid, int nv, int sp,
                                                const vec3<Dual<R, N>>& fd, const sym3<Dual<R, N>>& Hd, vec3<R> w,
                                                const sym3<R>& Hb, vec3<R>& ax) {
  for (int j = 0; j < nv; ++j) {
    const vec3<R> gj = {contract(fd, Hd, w, Hb, 3 * j), contract(fd, Hd, w, Hb, 3 * j + 1),
                        contract(fd, Hd, w, Hb, 3 * j + 2)};
    if (vid[j] == v)
      ax = ax + gj;
    else
      atomic_add3(A.adj_x, vid[j], gj);
    if (sp > 0)
      atomic_add3(A.adj_xp, vid[j], vec3<R>{contract(fd, Hd, w, Hb, sp + 3 * j), contract(fd, Hd, w, Hb, sp + 3 * j + 1),
                                            contract(fd, Hd, w, Hb, sp + 3 * j + 2)});
  }
}

// Membrane term of face t for the solved vertex v over the face's 9 coordinates (slots 0-8), mu and lambda (9, 10)
// and, for a damped face (N = 20), the 9 coordinates of the face's start positions (11-19).
template <typename R, int N>
__device__ __forceinline__ void membrane_adjoint(const AdjCtx<R>& A, int v, int t, int ord, vec3<R> w,
                                                 const sym3<R>& Hb, vec3<R>& ax) {
  const StepCtx<R>& c = A.c;
  using D = Dual<R, N>;
  const float4 mat = c.tri_mat[t];
  const int4 ti = c.tri_idx[t];
  const int vid[3] = {ti.x, ti.y, ti.z};
  const float4 dm = c.tri_pose[t];
  vec3<D> xs[3], xp[3];
  for (int j = 0; j < 3; ++j) {
    const vec3<R> p = ldx(A.x, vid[j]);
    xs[j] = {D::seed(p.x, 3 * j), D::seed(p.y, 3 * j + 1), D::seed(p.z, 3 * j + 2)};
    if (N > 11) {
      const vec3<R> pp = ld3<R>(c.qprev[vid[j]]);
      xp[j] = {D::seed(pp.x, 11 + 3 * j), D::seed(pp.y, 12 + 3 * j), D::seed(pp.z, 13 + 3 * j)};
    }
  }
  const D pose[4] = {D(R(dm.x)), D(R(dm.y)), D(R(dm.z)), D(R(dm.w))};
  vec3<D> fd = {D(R(0)), D(R(0)), D(R(0))};
  sym3<D> Hd = szero<D>();
  membrane_add<D>(ord, xs[0], xs[1], xs[2], pose, D::seed(R(mat.x), 9), D::seed(R(mat.y), 10),
                  D(R(N > 11 ? mat.z : 0.f)), D(R(mat.w)), D(c.dt), xp, fd, Hd);
  scatter_element<R, N>(A, v, vid, 3, N > 11 ? 11 : 0, fd, Hd, w, Hb, ax);
  if (A.adj_mu) atomicAdd(A.adj_mu + t, contract(fd, Hd, w, Hb, 9));
  if (A.adj_lambda) atomicAdd(A.adj_lambda + t, contract(fd, Hd, w, Hb, 10));
}

// Bending term of hinge e over its 12 coordinates (slots 0-11) and, for a damped hinge (N = 24), the 12
// coordinates of its start positions (12-23).
template <typename R, int N>
__device__ __forceinline__ void bending_adjoint(const AdjCtx<R>& A, int v, int e, int ord, vec3<R> w,
                                                const sym3<R>& Hb, vec3<R>& ax) {
  const StepCtx<R>& c = A.c;
  using D = Dual<R, N>;
  const float4 pr = c.edge_prop[e];
  const int4 ei = c.edge_idx[e];
  const int vid[4] = {ei.x, ei.y, ei.z, ei.w};
  vec3<D> xs[4], xp[4];
  for (int j = 0; j < 4; ++j) {
    const vec3<R> p = ldx(A.x, vid[j]);
    xs[j] = {D::seed(p.x, 3 * j), D::seed(p.y, 3 * j + 1), D::seed(p.z, 3 * j + 2)};
    if (N > 12) {
      const vec3<R> pp = ld3<R>(c.qprev[vid[j]]);
      xp[j] = {D::seed(pp.x, 12 + 3 * j), D::seed(pp.y, 13 + 3 * j), D::seed(pp.z, 14 + 3 * j)};
    }
  }
  vec3<D> fd = {D(R(0)), D(R(0)), D(R(0))};
  sym3<D> Hd = szero<D>();
  bending_add<D>(ord, xs, D(R(pr.x)), D(R(pr.y)), D(R(pr.z)), D(R(N > 12 ? pr.w : 0.f)), D(c.dt), xp, fd, Hd);
  scatter_element<R, N>(A, v, vid, 4, N > 12 ? 12 : 0, fd, Hd, w, Hb, ax);
}

// Tetrahedron term over its 12 coordinates (slots 0-11) and, for a damped tet (N = 24), its 12 start coordinates.
template <typename R, int N>
__device__ __forceinline__ void tet_adjoint(const AdjCtx<R>& A, int v, int t, int ord, vec3<R> w, const sym3<R>& Hb,
                                            vec3<R>& ax) {
  const StepCtx<R>& c = A.c;
  using D = Dual<R, N>;
  const float4 r0 = c.tet_pose[3 * t], r1 = c.tet_pose[3 * t + 1], r2 = c.tet_pose[3 * t + 2];
  const int4 ti = c.tet_idx[t];
  const int vid[4] = {ti.x, ti.y, ti.z, ti.w};
  const D dm[9] = {D(R(r0.x)), D(R(r0.y)), D(R(r0.z)), D(R(r1.x)), D(R(r1.y)), D(R(r1.z)),
                   D(R(r2.x)), D(R(r2.y)), D(R(r2.z))};
  vec3<D> xs[4], xp[4];
  for (int j = 0; j < 4; ++j) {
    const vec3<R> p = ldx(A.x, vid[j]);
    xs[j] = {D::seed(p.x, 3 * j), D::seed(p.y, 3 * j + 1), D::seed(p.z, 3 * j + 2)};
    if (N > 12) {
      const vec3<R> pp = ld3<R>(c.qprev[vid[j]]);
      xp[j] = {D::seed(pp.x, 12 + 3 * j), D::seed(pp.y, 13 + 3 * j), D::seed(pp.z, 14 + 3 * j)};
    }
  }
  vec3<D> fd = {D(R(0)), D(R(0)), D(R(0))};
  sym3<D> Hd = szero<D>();
  tet_add<D>(ord, xs, xp, dm, D(R(r0.w)), D(R(r1.w)), D(R(N > 12 ? r2.w : 0.f)), D(c.dt), fd, Hd);
  scatter_element<R, N>(A, v, vid, 4, N > 12 ? 12 : 0, fd, Hd, w, Hb, ax);
}

// Spring term of entry (spring << 1) | end of vertex v over x_v (slots 0-2), the other end (3-5) and v's start
// position (6-8, read by the damping).
template <typename R>
__device__ __forceinline__ void spring_adjoint(const AdjCtx<R>& A, int v, int a, vec3<R> w, const sym3<R>& Hb,
                                               vec3<R>& ax) {
  const StepCtx<R>& c = A.c;
  using D = Dual<R, 9>;
  const int sp = a >> 1, end = a & 1;
  const int2 ij = c.spr_idx[sp];
  const float4 pr = c.spr_prop[sp];
  const int o = end == 0 ? ij.y : ij.x;
  const vec3<R> pv = ldx(A.x, v), po = ldx(A.x, o), pa = ld3<R>(c.qprev[v]);
  const vec3<D> xv = {D::seed(pv.x, 0), D::seed(pv.y, 1), D::seed(pv.z, 2)};
  const vec3<D> xo = {D::seed(po.x, 3), D::seed(po.y, 4), D::seed(po.z, 5)};
  const vec3<D> xa = {D::seed(pa.x, 6), D::seed(pa.y, 7), D::seed(pa.z, 8)};
  vec3<D> fd = {D(R(0)), D(R(0)), D(R(0))};
  sym3<D> Hd = szero<D>();
  spring_add<D>(end, xv, xo, xa, D(R(pr.x)), D(R(pr.y)), D(R(pr.z)), D(c.dt), fd, Hd);
  ax = ax + vec3<R>{contract(fd, Hd, w, Hb, 0), contract(fd, Hd, w, Hb, 1), contract(fd, Hd, w, Hb, 2)};
  atomic_add3(A.adj_x, o, vec3<R>{contract(fd, Hd, w, Hb, 3), contract(fd, Hd, w, Hb, 4), contract(fd, Hd, w, Hb, 5)});
  atomic_add3(A.adj_xp, v, vec3<R>{contract(fd, Hd, w, Hb, 6), contract(fd, Hd, w, Hb, 7), contract(fd, Hd, w, Hb, 8)});
}

template <typename R>
__global__ void k_adjoint_color(AdjCtx<R> A, const int* __restrict__ verts, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const StepCtx<R>& c = A.c;
  const int v = verts[k];
  const R m = solve_mass(c, v);
  if (m == R(0)) return;  // fixed particle: no update, the adjoint passes through unchanged
  const R md = m * c.dt2r;
  const vec3<R> x = ldx(A.x, v);
  // forward quantities at this color's start
  vec3<R> f = md * (ldx(A.y, v) - x);
  sym3<R> H = sdiag(md);
  assemble_all(c, A.x, v, f, H);
  const R det = sdet(H);
  if (!(fabs(double(det)) > 1e-8) || !isfinite(double(det))) return;  // update skipped: D = 0
  const R idet = R(1) / det;
  const vec3<R> D = sadj_mul(H, f) * idet;
  const vec3<R> a = ldx(A.adj_x, v);
  const vec3<R> w = sadj_mul(H, a) * idet;
  // H_bar = -sym(w D^T)
  const sym3<R> Hb = {-w.x * D.x, -w.y * D.y, -w.z * D.z, R(-0.5) * (w.x * D.y + w.y * D.x),
                      R(-0.5) * (w.x * D.z + w.z * D.x), R(-0.5) * (w.y * D.z + w.z * D.y)};
  // inertia term: g = md (y - x)
  vec3<R> ax = a - md * w;
  atomic_add3(A.adj_y, v, md * w);
  // membranes: 9 coordinates + (mu, lambda) [+ 9 start coordinates with damping]
  for (int q = c.face_off[v]; q < c.face_off[v + 1]; ++q) {
    const int t = c.face_adj[q] >> 2, ord = c.face_adj[q] & 3;
    const float4 mat = c.tri_mat[t];
    if (!(mat.x > 0.f || mat.y > 0.f)) continue;
    if (mat.z > 0.f)
      membrane_adjoint<R, 20>(A, v, t, ord, w, Hb, ax);
    else
      membrane_adjoint<R, 11>(A, v, t, ord, w, Hb, ax);
  }
  // bending hinges: 12 coordinates [+ 12 start coordinates with damping]
  for (int q = c.edge_off[v]; q < c.edge_off[v + 1]; ++q) {
    const int e = c.edge_adj[q] >> 2, ord = c.edge_adj[q] & 3;
    const float4 pr = c.edge_prop[e];
    if (!(pr.z > 0.f)) continue;
    if (pr.w > 0.f)
      bending_adjoint<R, 24>(A, v, e, ord, w, Hb, ax);
    else
      bending_adjoint<R, 12>(A, v, e, ord, w, Hb, ax);
  }
  if (c.tet_off) {
    for (int q = c.tet_off[v]; q < c.tet_off[v + 1]; ++q) {
      const int t = c.tet_adj[q] >> 2, ord = c.tet_adj[q] & 3;
      const float4 r0 = c.tet_pose[3 * t], r1 = c.tet_pose[3 * t + 1], r2 = c.tet_pose[3 * t + 2];
      if (!(r0.w > 0.f || r1.w > 0.f)) continue;
      if (r2.w > 0.f)
        tet_adjoint<R, 24>(A, v, t, ord, w, Hb, ax);
      else
        tet_adjoint<R, 12>(A, v, t, ord, w, Hb, ax);
    }
  }
  if (c.spr_off) {
    for (int q = c.spr_off[v]; q < c.spr_off[v + 1]; ++q) spring_adjoint(A, v, c.spr_adj[q], w, Hb, ax);
    for (int q = c.sspr_off[v]; q < c.sspr_off[v + 1]; ++q) spring_adjoint(A, v, c.sspr_adj[q], w, Hb, ax);
  }
  if (c.has_contacts) contacts_adjoint(c, v, x, w, Hb, ax, A.adj_xp);
  A.adj_x[3 * v] = ax.x;
  A.adj_x[3 * v + 1] = ax.y;
  A.adj_x[3 * v + 2] = ax.z;
}

// one color of the forward sweep on plain (x, y) arrays: the state the adjoint differentiates
template <typename R>
__global__ void k_record_color(StepCtx<R> c, const R* __restrict__ xin, const R* __restrict__ y, R* xout,
                               const int* __restrict__ verts, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int v = verts[k];
  const R m = solve_mass(c, v);
  if (m == R(0)) return;
  const R md = m * c.dt2r;
  const vec3<R> x = ldx(xin, v);
  vec3<R> f = md * (ldx(y, v) - x);
  sym3<R> H = sdiag(md);
  assemble_all(c, xin, v, f, H);
  const R det = sdet(H);
  if (!(fabs(double(det)) > 1e-8) || !isfinite(double(det))) return;
  const vec3<R> xn = x + sadj_mul(H, f) * (R(1) / det);
  xout[3 * v] = xn.x;
  xout[3 * v + 1] = xn.y;
  xout[3 * v + 2] = xn.z;
}

// y (inertial target) and the mass flag of every particle, as forward_particle computes them
template <typename R>
__global__ void k_record_forward(StepCtx<R> c, R* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.V) return;
  forward_particle(c, GlobalPos<R>{c.pos}, i);
  const vec3<R> p = ld3<R>(c.inertia[i]);
  y[3 * i] = p.x;
  y[3 * i + 1] = p.y;
  y[3 * i + 2] = p.z;
}

// dL/dx of the last iterate from dL/dq_out and dL/dqd_out (q_out = x, qd_out = (x - q) / dt)
template <typename R>
__global__ void k_adjoint_begin(int n3, const R* aq, const R* aqd, R inv_dt, R* ax, R* ay) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n3) return;
  ax[i] = (aq ? aq[i] : R(0)) + (aqd ? aqd[i] * inv_dt : R(0));
  ay[i] = R(0);
}

// dL/dq_in, dL/dqd_in from dL/dy (the first iterate is y), the direct qd_out term and the contact terms' dL/dq
// (axp, or NULL)
template <typename R>
__global__ void k_adjoint_end(StepCtx<R> c, const R* ax, const R* ay, const R* axp, const R* aqd, R* aq_in,
                              R* aqd_in) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.V) return;
  const bool moves = (c.flags[i] & 1) && c.inv_mass[i] != 0.f;
  for (int j = 0; j < 3; ++j) {
    const R gy = ay[3 * i + j] + ax[3 * i + j];
    aq_in[3 * i + j] = gy - (aqd ? aqd[3 * i + j] / c.dt : R(0)) + (axp ? axp[3 * i + j] : R(0));
    if (aqd_in) aqd_in[3 * i + j] = moves ? gy * c.dt : R(0);
  }
}

// the substep's start positions where the contact terms read them (c.qprev), for the adjoint's recomputation
template <typename R>
__global__ void k_adjoint_qprev(StepCtx<R> c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < c.V) c.qprev[i] = pk4(vec3<R>{c.q_in[3 * i], c.q_in[3 * i + 1], c.q_in[3 * i + 2]}, R(0));
}

// q_out = x, qd_out = (x - q) / dt
template <typename R>
__global__ void k_record_finish(StepCtx<R> c, const R* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * c.V) return;
  c.q_out[i] = x[i];
  c.qd_out[i] = (x[i] - c.q_in[i]) / c.dt;
}

}  // namespace vbd
