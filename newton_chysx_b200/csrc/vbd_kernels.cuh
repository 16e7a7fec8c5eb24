// Device side of the B200 cloth VBD step.
//
// One routine, solve_group<R, L, MODE>, performs the work of the reference's solve_elasticity
// (particle_vbd_kernels.py:3135-3273) plus the per-color contact accumulation
// (particle_vbd_kernels.py:2900-2967 with rigid_vbd_kernels.py:762-834) and the AVBD penalty update
// (rigid_vbd_kernels.py:3755-3799) for one vertex, using L lanes of a warp:
//   - the vertex's adjacency (faces, then hinges) is split round-robin over the L lanes;
//   - the 9 partial sums (force 3, symmetric Hessian 6) are combined with xor-shuffles;
//   - lane 0 adds inertia and contact terms, solves the 3x3 system and writes the new position.
// Two schedulers call it: k_color (one launch per color, any model size) and k_persistent (one
// launch per substep; a CTA takes whole instances from a work queue and sweeps all their colors
// with __syncthreads between colors).
//
// Position update: the reference accumulates a displacement d and writes q = q_prev + d after every
// color (apply_truncation_ts with t = 1 and no bound when self-contact is off,
// particle_vbd_kernels.py:2877-2897). That is q += H^-1 f; this code applies it to q directly.
#pragma once
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <type_traits>

#include "vbd_elements.cuh"
#include "vbd_selfcontact.cuh"

namespace vbd {

enum Mode { MODE_FP32 = 0, MODE_MIXED = 1, MODE_FP64 = 2 };

template <typename R>
struct StepCtx {
  using P4 = pos4_t<R>;
  // packed model (solver-owned)
  const int4* __restrict__ tri_idx;
  const float4* __restrict__ tri_pose;
  const float4* __restrict__ tri_mat;  // mu, lambda, damping, area
  const int4* __restrict__ edge_idx;
  const float4* __restrict__ edge_prop;  // rest angle, rest length, ke, kd
  const int* __restrict__ face_off;      // [V+1], one int per entry
  const int* __restrict__ face_adj;      // (tri << 2) | order
  const int* __restrict__ edge_off;
  const int* __restrict__ edge_adj;  // (edge << 2) | order; boundary hinges are left out
  // model per particle (caller-owned, reference layout)
  const float* __restrict__ mass;
  const float* __restrict__ inv_mass;
  const int* __restrict__ flags;
  const float* __restrict__ radius;
  const float* __restrict__ gravity;
  // state (caller-owned)
  R* q_in;
  R* q_out;
  const R* qd_in;
  R* qd_out;
  const R* f_ext;
  // solver scratch
  P4* pos;      // current positions (w unused)
  P4* qprev;    // positions at the start of the step
  P4* inertia;  // inertial target; w = mass, or 0 for a fixed particle
  // contacts
  int has_contacts;
  int K;
  int* slot_cnt;  // [V]
  int* slots;     // [V*K]
  const int* c_count;
  int c_max;
  const int* c_particle;
  const int* c_shape;
  const float* c_body_pos;
  const float* c_body_vel;
  const float* c_normal;
  float* c_k;     // per-contact penalty stiffness (AVBD k)
  float* c_ke;    // per-contact averaged stiffness (ceiling)
  float* c_kd;
  float* c_mu;
  float soft_ke, soft_kd, soft_mu;
  const float* shape_ke;
  const float* shape_kd;
  const float* shape_mu;
  const int* shape_body;
  const float* body_com;
  const float* body_q;
  const float* body_q_prev;
  const float* body_qd;
  float k_start;
  R beta;
  R dt, dt2r, fric_eps;
  float fp64_thr;
  int* err;
  double* residual;  // [iterations] (MIXED)
  int V;
  int S;  // shape count
  // self-contact (per-color schedule): positions move as q = q_cd + disp, see vbd_collide.cuh
  int dual_in_solve;  // 1: AVBD penalty update fused into the solve (positions fixed within an iteration)
  P4* disp;           // displacement since the last detection, or null
  P4* pos_cd;         // positions at the last detection
  const int* ent_off;   // [V+1] per-vertex self-contact entries
  const unsigned* ent;  // (kind << 31) | (slot << 29) | pair
  const int4* vt_pairs;  // per pair its vertices: (t0, t1, t2, vertex)
  const int4* ee_pairs;  // per pair its vertices: (a0, a1, b0, b1)
  double sc_radius, sc_ee_eps;
  // springs and tetrahedra (solve_group<..., SOFT = true>)
  const int2* __restrict__ spr_idx;     // endpoints
  const float4* __restrict__ spr_prop;  // rest length, ke, kd
  const int* __restrict__ spr_off;      // [V+1] springs whose other end has another color: (spring << 1) | end
  const int* __restrict__ spr_adj;
  const int* __restrict__ sspr_off;     // [V+1] springs whose ends share a color (summed before the color's solve)
  const int* __restrict__ sspr_adj;
  int n_same_springs;                   // entries of sspr_adj; 0 = no pre-pass
  R* spr_acc;                           // [V, 9] pre-pass sums: f xyz, H xx yy zz xy xz yz
  const int4* __restrict__ tet_idx;
  const float4* __restrict__ tet_pose;  // [3 per tet]: rows of rest D^-1, w = mu, lambda, damping
  const int* __restrict__ tet_off;      // [V+1]
  const int* __restrict__ tet_adj;      // (tet << 2) | order
};

__device__ __forceinline__ void set_err(int* err, int bit) {
  if (err) atomicOr(err, bit);
}

// FP64 sum of |f|^2 over the lanes of a warp that reach this call (any subset: lanes that returned early for a
// fixed vertex are absent), one atomic per group of converged lanes into slot (iteration, warp mod 32); the host
// adds the 32 slots. Per-lane atomics on 32 shared addresses cost a mixed-precision substep ~60 % more.
__device__ __forceinline__ void residual_add(double* residual, int iteration, double r2) {
  namespace cg = cooperative_groups;
  const cg::coalesced_group g = cg::coalesced_threads();
  const double s = cg::reduce(g, r2, cg::plus<double>());
  if (g.thread_rank() == 0) atomicAdd(residual + 32 * iteration + ((threadIdx.x >> 5) & 31), s);
}

__device__ __forceinline__ vec3<float> ldv3(const float* a, int i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

// rotate v by quaternion (x, y, z, w), in A
template <typename A>
__device__ __forceinline__ vec3<A> qrot(const float* q, vec3<A> v) {
  const vec3<A> u = {A(q[0]), A(q[1]), A(q[2])};
  const A w = A(q[3]);
  return v * (A(2) * w * w - A(1)) + cross(u, v) * (A(2) * w) + u * (A(2) * dot(u, v));
}

// body transform X (p, q xyzw) applied to point p, in A
template <typename A>
__device__ __forceinline__ vec3<A> xform_point(const float* X, vec3<A> p) {
  return qrot<A>(X + 3, p) + vec3<A>{A(X[0]), A(X[1]), A(X[2])};
}

template <typename A>
__device__ __forceinline__ vec3<A> ldv3a(const float* a, int i) {
  return {A(a[3 * i]), A(a[3 * i + 1]), A(a[3 * i + 2])};
}

// Where the current positions live during the sweep: the solver's global float4/double4 array, or
// (persistent kernel, FP32) a packed float3 copy of one instance in shared memory.
template <typename R>
struct GlobalPos {
  pos4_t<R>* p;
  __device__ __forceinline__ vec3<R> ld(int i) const { return ld3<R>(p[i]); }
  __device__ __forceinline__ void st(int i, vec3<R> v) const { p[i] = pk4(v, R(0)); }
};

struct SmemPos {
  float* s;  // 3 floats per particle of the instance
  int base;  // first particle of the instance
  __device__ __forceinline__ vec3<float> ld(int i) const {
    const float* a = s + 3 * (i - base);
    return {a[0], a[1], a[2]};
  }
  __device__ __forceinline__ void st(int i, vec3<float> v) const {
    float* a = s + 3 * (i - base);
    a[0] = v.x;
    a[1] = v.y;
    a[2] = v.z;
  }
};

// ---------------------------------------------------------------------------------------------
// forward step of one particle: particle_vbd_kernels.py:1782-1807
template <typename R, typename P>
__device__ __forceinline__ void forward_particle(const StepCtx<R>& c, const P& pos, int i) {
  const vec3<R> q = {c.q_in[3 * i], c.q_in[3 * i + 1], c.q_in[3 * i + 2]};
  const int fl = c.flags[i];
  const float im = c.inv_mass[i];
  const float m = c.mass[i];
  const R msolve = ((fl & 1) && m != 0.f) ? R(m) : R(0);
  c.qprev[i] = pk4(q, R(0));
  if (!(fl & 1) || im == 0.f) {
    c.inertia[i] = pk4(q, msolve);
    pos.st(i, q);
    if (c.disp) c.disp[i] = pk4(zero3<R>(), R(0));
    return;
  }
  const vec3<R> g = {R(c.gravity[0]), R(c.gravity[1]), R(c.gravity[2])};
  vec3<R> fe = zero3<R>();
  if (c.f_ext) fe = {c.f_ext[3 * i], c.f_ext[3 * i + 1], c.f_ext[3 * i + 2]};
  const vec3<R> v = vec3<R>{c.qd_in[3 * i], c.qd_in[3 * i + 1], c.qd_in[3 * i + 2]} + (g + fe * R(im)) * c.dt;
  const vec3<R> d = v * c.dt;
  c.inertia[i] = pk4(q + d, msolve);
  pos.st(i, q + d);
  if (c.disp) c.disp[i] = pk4(d, R(0));
}

// velocity update and state write-back: particle_vbd_kernels.py:1900-1903, solver_vbd.py:2335-2337
template <typename R, typename P>
__device__ __forceinline__ void finalize_particle(const StepCtx<R>& c, const P& pos, int i) {
  const vec3<R> p = pos.ld(i);
  const vec3<R> qp = ld3<R>(c.qprev[i]);
  const vec3<R> v = (p - qp) * (R(1) / c.dt);
  c.q_in[3 * i] = p.x;
  c.q_in[3 * i + 1] = p.y;
  c.q_in[3 * i + 2] = p.z;
  c.q_out[3 * i] = p.x;
  c.q_out[3 * i + 1] = p.y;
  c.q_out[3 * i + 2] = p.z;
  c.qd_out[3 * i] = v.x;
  c.qd_out[3 * i + 1] = v.y;
  c.qd_out[3 * i + 2] = v.z;
}

// contact terms of one particle (lane 0 of the group), evaluated and accumulated in A (R, or double for the mixed
// mode's FP64 contact path)
template <typename R, typename A = R>
__device__ __forceinline__ void contacts_add_n(const StepCtx<R>& c, int v, int n, vec3<A> x, vec3<A>& f, sym3<A>& H) {
  if (n <= 0) return;
  if (n > c.K) n = c.K;
  int ids[8];
  for (int j = 0; j < n; ++j) ids[j] = c.slots[v * c.K + j];
  // contact index order, as the reference's launch order over contacts
  for (int a = 1; a < n; ++a) {
    int key = ids[a], b = a - 1;
    while (b >= 0 && ids[b] > key) {
      ids[b + 1] = ids[b];
      --b;
    }
    ids[b + 1] = key;
  }
  const A r = A(c.radius[v]);
  const A dt = A(c.dt);
  for (int j = 0; j < n; ++j) {
    const int t = ids[j];
    const int s = c.c_shape[t];
    const int b = (c.shape_body && s >= 0) ? c.shape_body[s] : -1;
    const vec3<A> bp = ldv3a<A>(c.c_body_pos, t);
    const float* X = (b >= 0 && c.body_q) ? c.body_q + 7 * b : nullptr;
    const vec3<A> bx = X ? xform_point<A>(X, bp) : bp;
    const vec3<float> nf = ldv3(c.c_normal, t);
    const vec3<A> nn = {A(nf.x), A(nf.y), A(nf.z)};
    const A pen = -(dot(nn, x - bx) - r);
    A k = A(c.c_k[t]);
    if (c.beta != R(0) && c.dual_in_solve) {
      // AVBD penalty ramp with the position at the start of this iteration (unchanged until now)
      k = vmin(k + A(c.beta) * vmax(A(0), pen), A(c.c_ke[t]));
      c.c_k[t] = float(k);
    }
    if (pen > A(0)) {
      const vec3<A> dx = x - ld3<A>(c.qprev[v]);
      // velocity of the contact point (rigid_vbd_kernels.py:806-819)
      const vec3<A> bvl = ldv3a<A>(c.c_body_vel, t);
      vec3<A> bv = bvl;
      if (X) {
        bv = qrot<A>(X + 3, bvl);
        if (c.body_q_prev) {
          const vec3<A> bxp = xform_point<A>(c.body_q_prev + 7 * b, bp);
          bv = (bx - bxp) * (A(1) / dt) + bv;
        } else if (c.body_qd) {
          const float* qd = c.body_qd + 6 * b;
          const vec3<A> com = c.body_com ? ldv3a<A>(c.body_com, b) : vec3<A>{A(0), A(0), A(0)};
          const vec3<A> rr = bx - xform_point<A>(X, com);
          bv = vec3<A>{A(qd[0]), A(qd[1]), A(qd[2])} + cross(vec3<A>{A(qd[3]), A(qd[4]), A(qd[5])}, rr) + bv;
        }
      }
      const vec3<A> rel = dx - bv * dt;
      contact_add<A>(pen, nn, rel, k, A(c.c_kd[t]), A(c.c_mu[t]), A(c.fric_eps), dt, f, H);
    }
  }
}

// contacts_add_n with the particle's contact count read here
template <typename R>
__device__ __forceinline__ void contacts_add(const StepCtx<R>& c, int v, vec3<R> x, vec3<R>& f, sym3<R>& H) {
  contacts_add_n<R>(c, v, c.slot_cnt[v], x, f, H);
}

// Contact terms and the 3x3 block solve H dlt = f of one vertex whose (f, H) hold its element and inertia sums.
// extra: nine more sums (f xyz, then H xx yy zz xy xz yz) added after the contacts, or null. r2 = |f|^2 of the full
// sums in FP64 (the mixed mode's residual). Returns the determinant used; the caller applies the reference's
// |det H| > 1e-8 test.
// FP32, FP64: all in R, the reference's arithmetic.
// MIXED: a vertex with contacts widens its FP32 sums to FP64, adds the contact terms in FP64 and solves in FP64.
// The contact damping stiffness kd ke / dt along the normal (1.9e8 N/m for the reference's default shape material,
// kd = 100 averaged with the model's, over ke = 6,250, at dt = 1/600 s) is 1e8 times the membrane, bending and
// inertia stiffness of a fine sheet; an FP32 sum of both keeps nothing of the latter (its rounding is ~10 N/m), so
// the tangential part of the block is lost and the FP32 step of such a vertex can move it by metres. In FP64 the
// stiff normal direction is a rank-one term known to 1e-16 and the tangential block survives. Vertices without
// contacts solve in FP64 only when their FP32 block is ill-conditioned (|det H| < thr max|H|^3).
template <typename R, int MODE>
__device__ __forceinline__ double contacts_and_solve(const StepCtx<R>& c, int v, int ncont, vec3<R> x, vec3<R> f,
                                                     sym3<R> H, const R* extra, vec3<R>& dlt, double& r2) {
  if (MODE == MODE_MIXED && ncont > 0) {
    const vec3<double> xd = {double(x.x), double(x.y), double(x.z)};
    vec3<double> fd = {double(f.x), double(f.y), double(f.z)};
    sym3<double> Hd = {double(H.xx), double(H.yy), double(H.zz), double(H.xy), double(H.xz), double(H.yz)};
    contacts_add_n<R, double>(c, v, ncont, xd, fd, Hd);
    if (extra) {
      fd = fd + vec3<double>{double(extra[0]), double(extra[1]), double(extra[2])};
      Hd = Hd + sym3<double>{double(extra[3]), double(extra[4]), double(extra[5]),
                             double(extra[6]), double(extra[7]), double(extra[8])};
    }
    r2 = dot(fd, fd);
    const double det = sdet(Hd);
    const vec3<double> rr = sadj_mul(Hd, fd) * (1.0 / det);
    dlt = {R(rr.x), R(rr.y), R(rr.z)};
    return det;
  }
  if (ncont > 0) contacts_add_n<R>(c, v, ncont, x, f, H);
  if (extra) {
    f = f + vec3<R>{extra[0], extra[1], extra[2]};
    H = H + sym3<R>{extra[3], extra[4], extra[5], extra[6], extra[7], extra[8]};
  }
  r2 = double(f.x) * double(f.x) + double(f.y) * double(f.y) + double(f.z) * double(f.z);
  if (MODE == MODE_MIXED) {
    const R hmax = vmax(vmax(vmax(vabs(H.xx), vabs(H.yy)), vmax(vabs(H.zz), vabs(H.xy))), vmax(vabs(H.xz), vabs(H.yz)));
    const R d = sdet(H);
    if (!(vabs(d) >= R(c.fp64_thr) * hmax * hmax * hmax)) {  // ill-conditioned or not finite: FP64
      const sym3<double> Hd = {double(H.xx), double(H.yy), double(H.zz), double(H.xy), double(H.xz), double(H.yz)};
      const vec3<double> fd = {double(f.x), double(f.y), double(f.z)};
      const double det = sdet(Hd);
      const vec3<double> rr = sadj_mul(Hd, fd) * (1.0 / det);
      dlt = {R(rr.x), R(rr.y), R(rr.z)};
      return det;
    }
    dlt = sadj_mul(H, f) * (R(1) / d);
    return double(d);
  }
  const R d = sdet(H);
  dlt = sadj_mul(H, f) * (R(1) / d);
  return double(d);
}

// ---------------------------------------------------------------------------------------------
// One vertex solved by L lanes. All lanes of the warp must call this (it shuffles).
// Self-contact term of one entry of vertex v's list (see vbd_collide.cuh for the encoding).
template <typename R, typename P>
__device__ __forceinline__ void self_contact_add(const StepCtx<R>& c, const P& pos, unsigned code, vec3<R>& f,
                                                 sym3<R>& H) {
  const int pair = int(code & 0x1FFFFFFFu), slot = int((code >> 29) & 3u);
  const int4 q = __ldg((code >> 31 ? c.ee_pairs : c.vt_pairs) + pair);
  const int ids[4] = {q.x, q.y, q.z, q.w};
  vec3<R> x[4], xa[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) x[k] = pos.ld(ids[k]), xa[k] = ld3<R>(c.qprev[ids[k]]);
  const R eps_u = c.fric_eps * c.dt;
  if (code >> 31)
    sc_ee_add<R>(slot, x, xa, R(c.sc_radius), R(c.soft_ke), R(c.soft_kd), R(c.soft_mu), eps_u, c.dt, R(c.sc_ee_eps), f, H);
  else
    sc_vt_add<R>(slot, x, xa, R(c.sc_radius), R(c.soft_ke), R(c.soft_kd), R(c.soft_mu), eps_u, c.dt, f, H);
}

// Spring term of one entry (spring << 1) | end of vertex v's spring list.
template <typename R, typename P>
__device__ __forceinline__ void spring_entry_add(const StepCtx<R>& c, const P& pos, int v, int a, vec3<R>& f,
                                                 sym3<R>& H) {
  const int sp = a >> 1, end = a & 1;
  const int2 ij = __ldg(c.spr_idx + sp);
  const float4 pr = __ldg(c.spr_prop + sp);
  const vec3<R> xa = pr.z != 0.f ? ld3<R>(c.qprev[v]) : zero3<R>();
  spring_add<R>(end, pos.ld(v), pos.ld(end == 0 ? ij.y : ij.x), xa, R(pr.x), R(pr.y), R(pr.z), c.dt, f, H);
}

// Tetrahedron term of one entry (tet << 2) | order.
template <typename R, typename P>
__device__ __forceinline__ void tet_entry_add(const StepCtx<R>& c, const P& pos, int a, vec3<R>& f, sym3<R>& H) {
  const int t = a >> 2, ord = a & 3;
  const float4 r0 = __ldg(c.tet_pose + 3 * t), r1 = __ldg(c.tet_pose + 3 * t + 1), r2 = __ldg(c.tet_pose + 3 * t + 2);
  if (!(r0.w > 0.f || r1.w > 0.f)) return;  // the reference skips tets with mu <= 0 and lambda <= 0
  const int4 ti = __ldg(c.tet_idx + t);
  const R dm[9] = {R(r0.x), R(r0.y), R(r0.z), R(r1.x), R(r1.y), R(r1.z), R(r2.x), R(r2.y), R(r2.z)};
  vec3<R> x[4], xp[4];
  x[0] = pos.ld(ti.x);
  x[1] = pos.ld(ti.y);
  x[2] = pos.ld(ti.z);
  x[3] = pos.ld(ti.w);
  if (r2.w > 0.f) {
    xp[0] = ld3<R>(c.qprev[ti.x]);
    xp[1] = ld3<R>(c.qprev[ti.y]);
    xp[2] = ld3<R>(c.qprev[ti.z]);
    xp[3] = ld3<R>(c.qprev[ti.w]);
  }
  tet_add<R>(ord, x, xp, dm, R(r0.w), R(r1.w), R(r2.w), c.dt, f, H);
}

// Sum of the springs of vertex v whose two ends share v's color, at the positions before the color's
// solve (accumulate_spring_force_and_hessian, particle_vbd_kernels.py:2347-2397, runs before the solve
// of each color, so both ends see the other's position from before it); the solve adds it.
template <typename R, typename P>
__device__ __forceinline__ void spring_prepass_vertex(const StepCtx<R>& c, const P& pos, int v) {
  const int b = __ldg(c.sspr_off + v), e = __ldg(c.sspr_off + v + 1);
  if (b == e) return;
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  for (int k = b; k < e; ++k) spring_entry_add<R>(c, pos, v, __ldg(c.sspr_adj + k), f, H);
  R* o = c.spr_acc + 9 * size_t(v);
  o[0] = f.x, o[1] = f.y, o[2] = f.z, o[3] = H.xx, o[4] = H.yy, o[5] = H.zz, o[6] = H.xy, o[7] = H.xz, o[8] = H.yz;
}

// SC: self-contact on. The vertex's self-contact entries join its faces and hinges in the lane split, and
// the solve adds its step to the displacement since the last detection instead of moving the vertex
// (the truncation pass that follows each color moves it, as apply_truncation_ts does).
// SOFT: the model has springs or tetrahedra; the vertex's tets and cross-color springs join the lane split
// after its hinges (solve_elasticity, particle_vbd_kernels.py:3136-3280, adds tets after hinges and the
// pre-accumulated springs and contacts last).
template <typename R, int L, int MODE, typename P, bool SC = false, bool SOFT = false>
__device__ __forceinline__ void solve_group(const StepCtx<R>& c, const P& pos, int v, bool valid, int sub,
                                            int iteration) {
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  R m = R(0);
  if (valid) m = R(c.inertia[v].w);
  const bool active = valid && m != R(0);
  if (active) {
    const int fb = __ldg(c.face_off + v), fe = __ldg(c.face_off + v + 1);
    const int eb = __ldg(c.edge_off + v), ee = __ldg(c.edge_off + v + 1);
    const int nf = fe - fb;
    int nfe = nf + (ee - eb);
    int tb = 0, nfet = nfe, sb = 0;
    if (SOFT) {
      tb = __ldg(c.tet_off + v);
      nfet = nfe + (__ldg(c.tet_off + v + 1) - tb);
      sb = __ldg(c.spr_off + v);
      nfe = nfet + (__ldg(c.spr_off + v + 1) - sb);  // from here on: every element entry
    }
    int cb = 0, n = nfe;
    if (SC) {
      cb = __ldg(c.ent_off + v);
      n += __ldg(c.ent_off + v + 1) - cb;
    }
    if (SC && !SOFT) {
      // faces, hinges and self-contact entries each start at lane 0, so that a round of the lanes runs one kind of
      // term instead of diverging between kinds: 8.71 against 8.84 ms per substep on a 256 x 256 sheet draped on a
      // sphere, 16.4 against 17.5 ms on 2,048 batched 16 x 16 sheets. (The same loops written with lambdas over the
      // accumulators measured 9.04 ms: written out here.)
      for (int k = sub; k < nf; k += L) {
        const int a = __ldg(c.face_adj + fb + k);
        const int t = a >> 2, ord = a & 3;
        const float4 mat = __ldg(c.tri_mat + t);
        if (mat.x > 0.f || mat.y > 0.f) {
          const int4 ti = __ldg(c.tri_idx + t);
          const float4 dm = __ldg(c.tri_pose + t);
          const R pose[4] = {R(dm.x), R(dm.y), R(dm.z), R(dm.w)};
          vec3<R> xp[3];
          if (mat.z > 0.f) {
            xp[0] = ld3<R>(c.qprev[ti.x]);
            xp[1] = ld3<R>(c.qprev[ti.y]);
            xp[2] = ld3<R>(c.qprev[ti.z]);
          }
          membrane_add<R>(ord, pos.ld(ti.x), pos.ld(ti.y), pos.ld(ti.z), pose, R(mat.x), R(mat.y), R(mat.z), R(mat.w),
                          c.dt, xp, f, H);
        }
      }
      for (int k = sub; k < ee - eb; k += L) {
        const int a = __ldg(c.edge_adj + eb + k);
        const int e = a >> 2, ord = a & 3;
        const float4 pr = __ldg(c.edge_prop + e);
        if (pr.z > 0.f) {
          const int4 ei = __ldg(c.edge_idx + e);
          vec3<R> x[4];
          x[0] = pos.ld(ei.x);
          x[1] = pos.ld(ei.y);
          x[2] = pos.ld(ei.z);
          x[3] = pos.ld(ei.w);
          vec3<R> xp[4];
          if (pr.w > 0.f) {
            xp[0] = ld3<R>(c.qprev[ei.x]);
            xp[1] = ld3<R>(c.qprev[ei.y]);
            xp[2] = ld3<R>(c.qprev[ei.z]);
            xp[3] = ld3<R>(c.qprev[ei.w]);
          }
          bending_add<R>(ord, x, R(pr.x), R(pr.y), R(pr.z), R(pr.w), c.dt, xp, f, H);
        }
      }
      for (int k = sub; k < n - nfe; k += L) self_contact_add<R>(c, pos, __ldg(c.ent + cb + k), f, H);
      n = 0;  // the round-robin loop below has nothing left
    }
    for (int it = sub; it < n; it += L) {
      if (SC && it >= nfe) {
        self_contact_add<R>(c, pos, __ldg(c.ent + cb + (it - nfe)), f, H);
      } else if (SOFT && it >= nfet) {
        spring_entry_add<R>(c, pos, v, __ldg(c.spr_adj + sb + (it - nfet)), f, H);
      } else if (SOFT && it >= nf + (ee - eb)) {
        tet_entry_add<R>(c, pos, __ldg(c.tet_adj + tb + (it - nf - (ee - eb))), f, H);
      } else if (it < nf) {
        const int a = __ldg(c.face_adj + fb + it);
        const int t = a >> 2, ord = a & 3;
        const float4 mat = __ldg(c.tri_mat + t);
        if (mat.x > 0.f || mat.y > 0.f) {
          const int4 ti = __ldg(c.tri_idx + t);
          const float4 dm = __ldg(c.tri_pose + t);
          const R pose[4] = {R(dm.x), R(dm.y), R(dm.z), R(dm.w)};
          const vec3<R> x0 = pos.ld(ti.x), x1 = pos.ld(ti.y), x2 = pos.ld(ti.z);
          vec3<R> xp[3];
          if (mat.z > 0.f) {
            xp[0] = ld3<R>(c.qprev[ti.x]);
            xp[1] = ld3<R>(c.qprev[ti.y]);
            xp[2] = ld3<R>(c.qprev[ti.z]);
          }
          membrane_add<R>(ord, x0, x1, x2, pose, R(mat.x), R(mat.y), R(mat.z), R(mat.w), c.dt, xp, f, H);
        }
      } else {
        const int a = __ldg(c.edge_adj + eb + (it - nf));
        const int e = a >> 2, ord = a & 3;
        const float4 pr = __ldg(c.edge_prop + e);
        if (pr.z > 0.f) {
          const int4 ei = __ldg(c.edge_idx + e);
          vec3<R> x[4];
          x[0] = pos.ld(ei.x);
          x[1] = pos.ld(ei.y);
          x[2] = pos.ld(ei.z);
          x[3] = pos.ld(ei.w);
          vec3<R> xp[4];
          if (pr.w > 0.f) {
            xp[0] = ld3<R>(c.qprev[ei.x]);
            xp[1] = ld3<R>(c.qprev[ei.y]);
            xp[2] = ld3<R>(c.qprev[ei.z]);
            xp[3] = ld3<R>(c.qprev[ei.w]);
          }
          bending_add<R>(ord, x, R(pr.x), R(pr.y), R(pr.z), R(pr.w), c.dt, xp, f, H);
        }
      }
    }
  }
  if (L > 1) {
    f.x = group_sum<L>(f.x);
    f.y = group_sum<L>(f.y);
    f.z = group_sum<L>(f.z);
    H.xx = group_sum<L>(H.xx);
    H.yy = group_sum<L>(H.yy);
    H.zz = group_sum<L>(H.zz);
    H.xy = group_sum<L>(H.xy);
    H.xz = group_sum<L>(H.xz);
    H.yz = group_sum<L>(H.yz);
  }
  const bool leader = active && sub == 0;
  if (SC && valid && !active && sub == 0) c.disp[v] = pk4(zero3<R>(), R(0));  // as the reference's solve does
  vec3<R> x = zero3<R>();
  vec3<R> dlt = zero3<R>();
  double det_used = 0.0, r2 = 0.0;
  if (leader) {
    x = pos.ld(v);
    const vec3<R> in = ld3<R>(c.inertia[v]);
    const R md = m * c.dt2r;
    f = f + md * (in - x);
    H.xx += md;
    H.yy += md;
    H.zz += md;
    const R* extra = nullptr;
    if (SOFT && c.n_same_springs && __ldg(c.sspr_off + v + 1) > __ldg(c.sspr_off + v)) extra = c.spr_acc + 9 * size_t(v);
    det_used = contacts_and_solve<R, MODE>(c, v, c.has_contacts ? c.slot_cnt[v] : 0, x, f, H, extra, dlt, r2);
  }
  if (MODE == MODE_MIXED && c.residual) {
    // FP64 reduction of |f|^2 (the force residual the block solve removes): warp sum, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    if ((threadIdx.x & 31) == 0 && r2 != 0.0) atomicAdd(c.residual + 32 * iteration, r2);
  }
  if (!leader) return;
  // the reference updates only when |det H| > 1e-8 (a NaN determinant fails that test too)
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
  if (SC)
    c.disp[v] = pk4(ld3<R>(c.disp[v]) + dlt, R(0));
  else
    pos.st(v, xn);
}

// ---------------------------------------------------------------------------------------------
template <typename R>
__global__ void k_forward(StepCtx<R> c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.V) return;
  forward_particle(c, GlobalPos<R>{c.pos}, i);
  if (c.has_contacts) c.slot_cnt[i] = 0;
}

template <typename R>
__global__ void k_finalize(StepCtx<R> c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.V) return;
  finalize_particle(c, GlobalPos<R>{c.pos}, i);
}

// Per-contact setup (init_body_particle_contacts, rigid_vbd_kernels.py:2318-2361) and the
// particle -> contact slot table. Must run after the slot counters were cleared.
template <typename R>
__global__ void k_contact_prepare(StepCtx<R> c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int count = *c.c_count;
  if (count > c.c_max) count = c.c_max;
  if (t >= count) return;
  const int p = c.c_particle[t];
  const int s = c.c_shape[t];
  if (p < 0 || p >= c.V || s < 0 || s >= c.S) {
    set_err(c.err, 8);
    return;
  }
  const float ke = 0.5f * (c.soft_ke + c.shape_ke[s]);
  const float kd = 0.5f * (c.soft_kd + c.shape_kd[s]);
  const float mu = sqrtf(c.soft_mu * c.shape_mu[s]);
  c.c_ke[t] = ke;
  c.c_kd[t] = kd;
  c.c_mu[t] = mu;
  c.c_k[t] = c.k_start < 0.f ? ke : fminf(c.k_start, ke);
  const int slot = atomicAdd(c.slot_cnt + p, 1);
  if (slot < c.K)
    c.slots[p * c.K + slot] = t;
  else
    set_err(c.err, 2);
}

// With self-contact the kernel is latency-bound on its chains of dependent loads (entry, pair, element, positions);
// capping it at 72 registers (some spills) lets 7 CTAs of 128 threads share an SM instead of 4: 8.79 ms against
// 9.21 ms per substep on a 256 x 256 sheet draped on a sphere (80: 8.98 ms, 64: 8.89 ms).
template <typename R, int L, int MODE, bool SC = false, bool SOFT = false>
__global__ void __maxnreg__(SC ? 72 : 255) k_color(StepCtx<R> c, const int* __restrict__ verts, int n, int iteration) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int grp = gid / L, sub = gid % L;
  const bool valid = grp < n;
  const int v = valid ? __ldg(verts + grp) : 0;
  solve_group<R, L, MODE, GlobalPos<R>, SC, SOFT>(c, GlobalPos<R>{c.pos}, v, valid, sub, iteration);
}

// Same-color spring sums of one color's vertices (per-color schedule), before that color's solve.
template <typename R>
__global__ void k_spring_prepass(StepCtx<R> c, const int* __restrict__ verts, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) spring_prepass_vertex<R>(c, GlobalPos<R>{c.pos}, __ldg(verts + i));
}

// AVBD penalty update of every contact at the start of an iteration (update_duals_body_particle_contacts,
// rigid_vbd_kernels.py:3755-3799); used when positions can move between an iteration's start and a
// vertex's color (self-contact truncation), where the update cannot be fused into the solve.
template <typename R>
__global__ void k_contact_duals(StepCtx<R> c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int count = *c.c_count;
  if (count > c.c_max) count = c.c_max;
  if (t >= count) return;
  const int v = c.c_particle[t];
  const int s = c.c_shape[t];
  if (v < 0 || v >= c.V || s < 0 || s >= c.S) return;
  const int b = (c.shape_body && s >= 0) ? c.shape_body[s] : -1;
  const vec3<R> bp = ldv3a<R>(c.c_body_pos, t);
  const vec3<R> bx = (b >= 0 && c.body_q) ? xform_point<R>(c.body_q + 7 * b, bp) : bp;
  const vec3<float> nf = ldv3(c.c_normal, t);
  const vec3<R> nn = {R(nf.x), R(nf.y), R(nf.z)};
  const R pen = -(dot(nn, ld3<R>(c.pos[v]) - bx) - R(c.radius[v]));
  c.c_k[t] = float(vmin(R(c.c_k[t]) + c.beta * vmax(R(0), pen), R(c.c_ke[t])));
}

struct PersistentPlan {
  int W;                      // instances
  const int* inst_order;      // [W] processing order (largest first)
  const int* inst_vstart;     // [W+1]
  const int* inst_cptr;       // [W+1] into color_ranges: instance w owns ranges[cptr[w] .. cptr[w+1]]
  const int* color_ranges;    // per instance: ncol+1 offsets into color_verts
  const int* color_verts;     // particle ids grouped by instance then color
  int* queue;                 // work counter, zero before launch
  int iterations;
};

// One launch per substep. SMEM: the instance's positions stay in shared memory (3 floats per
// particle) from the forward step to the write-back, so every neighbour gather of the sweep is a
// shared-memory load; otherwise they live in the solver's global float4 array.
template <typename R, int L, int MODE, bool SMEM, bool SOFT = false>
__global__ void k_persistent(StepCtx<R> c, PersistentPlan p) {
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
    const int per_round = blockDim.x / L;
    const int grp_local = threadIdx.x / L, sub = threadIdx.x % L;
    for (int it = 0; it < p.iterations; ++it) {
      for (int col = cb; col + 1 < ce; ++col) {
        const int a = __ldg(p.color_ranges + col), b = __ldg(p.color_ranges + col + 1);
        if (SOFT && c.n_same_springs) {
          for (int g = a + threadIdx.x; g < b; g += blockDim.x) spring_prepass_vertex<R>(c, pos, __ldg(p.color_verts + g));
          __syncthreads();
        }
        for (int base = a; base < b; base += per_round) {
          const int g = base + grp_local;
          const bool valid = g < b;
          const int v = valid ? __ldg(p.color_verts + g) : 0;
          solve_group<R, L, MODE, Pos, false, SOFT>(c, pos, v, valid, sub, it);
        }
        __syncthreads();
      }
    }
    for (int i = vs + threadIdx.x; i < ve; i += blockDim.x) finalize_particle(c, pos, i);
  }
}

// One warp per instance (small instances): each warp of the CTA takes instances from the work queue on its own,
// so a color needs only __syncwarp between its rounds, not a CTA barrier, and eight instances run side by side
// in a CTA of 256. SMEM: each warp keeps its instance's positions in its own slice of shared memory (slice
// floats per warp).
template <typename R, int L, int MODE, bool SMEM, bool SOFT>
__global__ void k_persistent_warp(StepCtx<R> c, PersistentPlan p, int slice) {
  extern __shared__ float s_pos[];
  const int lane = threadIdx.x & 31;
  float* mine = s_pos + size_t(threadIdx.x >> 5) * size_t(slice);
  for (;;) {
    int q = 0;
    if (lane == 0) q = atomicAdd(p.queue, 1);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= p.W) return;
    const int w = __ldg(p.inst_order + q);
    const int vs = __ldg(p.inst_vstart + w), ve = __ldg(p.inst_vstart + w + 1);
    using Pos = typename std::conditional<SMEM, SmemPos, GlobalPos<R>>::type;
    Pos pos;
    if constexpr (SMEM) {
      pos = SmemPos{mine, vs};
    } else {
      pos = GlobalPos<R>{c.pos};
    }
    for (int i = vs + lane; i < ve; i += 32) forward_particle(c, pos, i);
    __syncwarp();
    const int cb = __ldg(p.inst_cptr + w), ce = __ldg(p.inst_cptr + w + 1);
    constexpr int per_round = 32 / L;
    const int grp_local = lane / L, sub = lane % L;
    for (int it = 0; it < p.iterations; ++it) {
      for (int col = cb; col + 1 < ce; ++col) {
        const int a = __ldg(p.color_ranges + col), b = __ldg(p.color_ranges + col + 1);
        if (SOFT && c.n_same_springs) {
          for (int g = a + lane; g < b; g += 32) spring_prepass_vertex<R>(c, pos, __ldg(p.color_verts + g));
          __syncwarp();
        }
        for (int base = a; base < b; base += per_round) {
          const int g = base + grp_local;
          const bool valid = g < b;
          const int v = valid ? __ldg(p.color_verts + g) : 0;
          solve_group<R, L, MODE, Pos, false, SOFT>(c, pos, v, valid, sub, it);
        }
        __syncwarp();
      }
    }
    for (int i = vs + lane; i < ve; i += 32) finalize_particle(c, pos, i);
    __syncwarp();
  }
}

}  // namespace vbd
