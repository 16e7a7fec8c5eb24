// Per-element force / Hessian contributions for one vertex of the cloth VBD step.
//
// Each function adds the element's contribution for one of its vertices to (f, H). The math is
// that of the reference kernels; the formulation is rewritten for the GPU:
//  * membrane  - particle_vbd_kernels.py:865-1025 (stable Neo-Hookean membrane + Rayleigh damping).
//                Same formulas; the Hessian is accumulated as a symmetric 3x3.
//  * bending   - particle_vbd_kernels.py:1057-1190 (dihedral angle energy k (theta - theta0)^2 / 2,
//                k = ke * rest_length, Hessian k dtheta dtheta^T). The reference forms all four
//                dtheta/dx_k through 3x3 products of projected skew matrices
//                (compute_normalized_vector_derivative / compute_angle_derivative, :1028-1054).
//                Because the unit normals n1, n2 are orthogonal to the unit edge e and
//                n2 = cos(theta) n1 + sin(theta) (e x n1), that expression reduces exactly to the classic
//                dihedral gradient (Bridson et al. 2003, "Simulation of clothing with folds and
//                wrinkles"), with N1 = x02 x x03, N2 = x13 x x12 (formed as x02 x e and e x x13):
//                  dtheta/dx0 = -|e| / |N1| n1
//                  dtheta/dx1 = -|e| / |N2| n2
//                  dtheta/dx2 =  (x03 . e) / |N1| n1 + (x13 . e) / |N2| n2
//                  dtheta/dx3 = -(x02 . e) / |N1| n1 - (x12 . e) / |N2| n2
//                i.e. alpha n1 + beta n2 with two scalars chosen by the vertex's role, the same
//                instructions for every lane of a warp. Only the solved vertex's derivative is formed
//                unless damping needs all four.
//  * contact   - rigid_vbd_kernels.py:727-759, 891-934 (penalty, approach damping, IPC-smoothed
//                isotropic friction).
//  * spring    - particle_vbd_kernels.py:2299-2343 (linear spring with damping).
//  * tetrahedron - particle_vbd_kernels.py:335-473 (volumetric stable Neo-Hookean), contracted to the
//                vertex's 3x3 block in closed form.
#pragma once
#include "vbd_math.cuh"

namespace vbd {

// Membrane contribution of one triangle for the vertex of order `ord` (0, 1, 2).
// pose = D^-1 row-major (00, 01, 10, 11); mat = (mu, lambda, damping, area).
// lnh_floor: the floor of |lambda + mu| in alpha = 1 + mu / (lambda + mu), 1e-6 for material values (the
// reference's); 0 when mu and lambda come pre-multiplied by the area (stencil records), whose builder checks
// the floor on the material values instead.
template <typename R>
__host__ __device__ __forceinline__ void membrane_add(int ord, vec3<R> x0, vec3<R> x1, vec3<R> x2, const R pose[4],
                                                      R mu, R lmbd, R damping, R area, R dt, const vec3<R>* xp,
                                                      vec3<R>& f, sym3<R>& H, R lnh_floor = R(1.0e-6)) {
  const vec3<R> x01 = x1 - x0, x02 = x2 - x0;
  const R D00 = pose[0], D01 = pose[1], D10 = pose[2], D11 = pose[3];
  const vec3<R> f0 = x01 * D00 + x02 * D10;
  const vec3<R> f1 = x01 * D01 + x02 * D11;
  const R f00 = dot(f0, f0), f11 = dot(f1, f1), f01 = dot(f0, f1);
  const R Jsq = vmax(f00 * f11 - f01 * f01, R(1.0e-20));
  const R invJ = vrsqrt(Jsq);
  const R J = Jsq * invJ;
  const R lnh = lmbd + mu;
  const R lsafe = lnh_floor > R(0) ? (lnh < R(0) ? R(-1) : R(1)) * vmax(vabs(lnh), lnh_floor) : (lnh == R(0) ? R(1) : lnh);
  const R alpha = R(1) + vdiv_fast(mu, lsafe);
  const R s = lnh * (J - alpha);
  const R m0 = R(ord == 0), m1 = R(ord == 1), m2 = R(ord == 2);
  const R d0 = D00 * (m1 - m0) + D10 * (m2 - m0);
  const R d1 = D01 * (m1 - m0) + D11 * (m2 - m0);
  // with g0 = (f11 f0 - f01 f1) / J and g1 = (f00 f1 - f01 f0) / J the derivative of J is dJ = g0 d0 + g1 d1 =
  // e0 f0 + e1 f1, and the force -(P0 d0 + P1 d1) with P_i = mu f_i + s g_i is -(c0 f0 + c1 f1): scalar
  // coefficients instead of the vectors g0, g1
  const R e0 = invJ * (f11 * d0 - f01 * d1), e1 = invJ * (f00 * d1 - f01 * d0);
  const vec3<R> dJ = e0 * f0 + e1 * f1;
  // the terms go straight into (f, H), scaled by the area through their scalar coefficients
  const R c0 = area * (mu * d0 + s * e0), c1 = area * (mu * d1 + s * e1);
  f = f - c0 * f0 - c1 * f1;
  const R r = vmax(R(0), s) * invJ;
  const vec3<R> w = f1 * d0 - f0 * d1;
  const R Ic = area * (mu * (d0 * d0 + d1 * d1) + r * (d0 * d0 * f11 + d1 * d1 * f00 - R(2) * d0 * d1 * f01));
  H.xx += Ic;
  H.yy += Ic;
  H.zz += Ic;
  souter_add(H, dJ, area * (lnh - r));
  souter_add(H, w, -(area * r));
  if (damping > R(0)) {
    const R G00 = R(0.5) * (f00 - R(1)), G11 = R(0.5) * (f11 - R(1)), G01 = R(0.5) * f01;
    const R Gsq = G00 * G00 + G11 * G11 + R(2) * G01 * G01;
    if (Gsq >= R(1.0e-20)) {
      const R inv_dt = R(1) / dt;
      const vec3<R> v01 = (x01 - (xp[1] - xp[0])) * inv_dt, v02 = (x02 - (xp[2] - xp[0])) * inv_dt;
      const vec3<R> df0 = v01 * D00 + v02 * D10, df1 = v01 * D01 + v02 * D11;
      const R C = vsqrt(Gsq);
      const R n00 = G00 / C, n01 = G01 / C, n11 = G11 / C;
      const R dG00 = dot(f0, df0), dG11 = dot(f1, df1), dG01 = R(0.5) * (dot(f0, df1) + dot(f1, df0));
      const R dC = n00 * dG00 + n11 * dG11 + R(2) * n01 * dG01;
      const vec3<R> dCdx = d0 * (n00 * f0 + n01 * f1) + d1 * (n01 * f0 + n11 * f1);
      const R kmu = area * mu * damping;
      f = f + (-kmu * dC) * dCdx;
      souter_add(H, dCdx, kmu * inv_dt);
      const R dCl = dG00 + dG11;
      const vec3<R> dCldx = d0 * f0 + d1 * f1;
      const R kl = area * lmbd * damping;
      f = f + (-kl * dCl) * dCldx;
      souter_add(H, dCldx, kl * inv_dt);
    }
  }
}

// Dihedral bending contribution of hinge (x0 opposite-0, x1 opposite-1, x2-x3 the shared edge) for
// the vertex of order `ord` (0..3). prop = (rest_angle, rest_length, ke, kd). xp = previous positions
// of the four vertices, read only when kd > 0.
template <typename R>
__host__ __device__ __forceinline__ void bending_add_coef(R ca, R cb, R dd, const vec3<R> x[4], R rest_angle,
                                                          R rest_length, R ke, R kd, R dt, const vec3<R>* xp,
                                                          vec3<R>& f, sym3<R>& H) {
  // with x03 = x02 + e and x12 = x13 - e: N1 = x02 x x03 = x02 x e, N2 = x13 x x12 = e x x13
  const vec3<R> x02 = x[2] - x[0], x13 = x[3] - x[1], e = x[3] - x[2];
  const vec3<R> N1 = cross(x02, e), N2 = cross(e, x13);
  const R s1 = dot(N1, N1), s2 = dot(N2, N2), se = dot(e, e);
  // |N1|, |N2|, |e| < 1e-6 (degenerate hinge): no contribution
  const R eps2 = R(1.0e-12);
  if (s1 < eps2 || s2 < eps2 || se < eps2) return;
  const R ile = vrsqrt(se);
  const R le = se * ile;  // |e|
  // theta = atan2((n1 x n2) . e/|e|, n1 . n2) on the unnormalised normals (atan2 ignores their common factor
  // |N1| |N2| > 0); N1 x N2 = (x02 . N2) e, so (N1 x N2) . e/|e| = (x02 . N2) |e|
  const R theta = vatan2(dot(x02, N2) * le, dot(N1, N2));
  const R k = ke * rest_length;
  const R dE = k * (theta - rest_angle);
  // dtheta/dx_ord = a N1 + b N2. With u1 = x02 . e/|e| and u2 = x13 . e/|e| (x03 . e = x02 . e + |e|^2,
  // x12 . e = x13 . e - |e|^2):  a |N1|^2 = -|e|, 0, u1 + |e|, -u1  and  b |N2|^2 = 0, -|e|, u2, |e| - u2  for
  // ord = 0, 1, 2, 3: (c_a |e| + d u1) / |N1|^2 and (c_b |e| + d u2) / |N2|^2 with per-role constants, one
  // instruction stream for every lane of a warp whatever the roles of their hinges
  const R q1 = vrcp(s1), q2 = vrcp(s2);
  const R u1 = dot(x02, e) * ile, u2 = dot(x13, e) * ile;
  const R a = (ca * le + dd * u1) * q1;
  const R b = (cb * le + dd * u2) * q2;
  const vec3<R> d = a * N1 + b * N2;
  f = f + (-dE) * d;
  R hk = k;
  if (kd > R(0)) {
    const R il1 = vrsqrt(s1), il2 = vrsqrt(s2);
    const vec3<R> n1 = N1 * il1, n2 = N2 * il2, eh = e * ile;
    const vec3<R> x03 = x02 + e, x12 = x13 - e;
    const vec3<R> d0 = (-le * il1) * n1, d1 = (-le * il2) * n2;
    const vec3<R> d2 = (dot(x03, eh) * il1) * n1 + (dot(x13, eh) * il2) * n2;
    const vec3<R> d3 = (-dot(x02, eh) * il1) * n1 - (dot(x12, eh) * il2) * n2;
    const R inv_dt = R(1) / dt;
    const R dth = (dot(d0, x[0] - xp[0]) + dot(d1, x[1] - xp[1]) + dot(d2, x[2] - xp[2]) + dot(d3, x[3] - xp[3])) *
                  inv_dt;
    const R dc = kd * k;
    f = f + (-dc * dth) * d;
    hk = k + dc * inv_dt;
  }
  souter_add(H, d, hk);
}

// The per-role constants of bending_add_coef for the vertex of order `ord`.
template <typename R>
__host__ __device__ __forceinline__ void bending_add(int ord, const vec3<R> x[4], R rest_angle, R rest_length, R ke,
                                                     R kd, R dt, const vec3<R>* xp, vec3<R>& f, sym3<R>& H) {
  const R ca = ord == 0 ? R(-1) : (ord == 2 ? R(1) : R(0));
  const R cb = ord == 1 ? R(-1) : (ord == 3 ? R(1) : R(0));
  const R dd = ord == 2 ? R(1) : (ord == 3 ? R(-1) : R(0));
  bending_add_coef<R>(ca, cb, dd, x, rest_angle, rest_length, ke, kd, dt, xp, f, H);
}

// Penalty contact with a static or moving shape point. pen > 0 is the penetration depth, n the unit
// normal, rel the particle's displacement this step relative to the shape point.
template <typename R>
__host__ __device__ __forceinline__ void contact_add(R pen, vec3<R> n, vec3<R> rel, R ke, R kd, R mu, R fric_eps,
                                                     R dt, vec3<R>& f, sym3<R>& H) {
  const R fn = pen * ke;
  vec3<R> force = n * fn;
  R hn = ke;
  if (dot(n, rel) < R(0)) {
    const R hd = kd * ke / dt;
    hn += hd;
    force = force - n * (hd * dot(n, rel));
  }
  souter_add(H, n, hn);
  // friction: u_t = rel - n (n.rel); IPC smoothing with eps_u = fric_eps * dt
  const R eps_u = fric_eps * dt;
  const vec3<R> ut = rel - n * dot(n, rel);
  const R un = length(ut);
  if (un > R(0)) {
    const R f1 = un > eps_u ? R(1) / un : (-un / eps_u + R(2)) / eps_u;
    const R scale = mu * fn * f1;
    force = force - scale * ut;
    // scale (I - n n^T)
    H.xx += scale;
    H.yy += scale;
    H.zz += scale;
    souter_add(H, n, -scale);
  }
  f = f + force;
}

// Linear spring between the solved vertex (end `end` of the spring: 0 or 1) and its partner,
// particle_vbd_kernels.py:2299-2343 (evaluate_spring_force_and_hessian_both_vertices): with d = x_0 - x_1
// and l = max(|d|, 1e-8), the elastic force on end 0 is ke (l0 - l) / l d (the negative on end 1), the
// Hessian ke (I - l0 / l (I - d d^T / l^2)) = ke (1 - l0 / l) I + ke l0 / l^3 d d^T, and damping adds
// (kd / dt) H (x_prev - x) to the force and (kd / dt) H to the Hessian. xa = the vertex's position at the
// start of the step, read only when kd != 0.
template <typename R>
__host__ __device__ __forceinline__ void spring_add(int end, vec3<R> x, vec3<R> x_other, vec3<R> xa, R rest, R ke,
                                                    R kd, R dt, vec3<R>& f, sym3<R>& H) {
  const vec3<R> d = end == 0 ? x - x_other : x_other - x;
  const R l = vmax(length(d), R(1.0e-8));
  const R il = R(1) / l;
  const vec3<R> base = (ke * (rest - l) * il) * d;
  sym3<R> h = sdiag(ke * (R(1) - rest * il));
  souter_add(h, d, ke * rest * il * il * il);
  vec3<R> force = end == 0 ? base : -base;
  if (kd != R(0)) {
    const R c = kd / dt;
    force = force + c * smul(h, xa - x);
    h = (R(1) + c) * h;
  }
  f = f + force;
  H = H + h;
}

// Volumetric stable Neo-Hookean tetrahedron, particle_vbd_kernels.py:335-473, for the vertex of order
// `ord` (0..3). dm = rest D^-1 (row-major 3x3), mat = (mu, lambda, damping). With F = Ds D^-1 (columns
// F_0, F_1, F_2), cof(F) the cofactor matrix (columns F_1 x F_2, F_2 x F_0, F_0 x F_1), V the rest volume
// 1 / (6 det D^-1) and m the vertex's row of d vec(F) / dx (row ord-1 of D^-1, or minus the sum of its rows
// for ord 0), the reference's 9x9 forms contract in closed form to
//   f = -V (mu F m + s cof(F) m),  s = lambda_nh (det F - alpha)
//   H =  V (mu |m|^2 I + lambda_nh g g^T),  g = cof(F) m
// with lambda_nh = lambda + mu, alpha = 1 + mu / lambda_nh (|lambda_nh| floored at 1e-6). Damping adds
// -damping V (mu Fdot m + lambda_nh (cof(F) : Fdot) g) to f and scales H by 1 + damping / dt.
template <typename R>
__host__ __device__ __forceinline__ void tet_add(int ord, const vec3<R> x[4], const vec3<R>* xp, const R dm[9], R mu,
                                                 R lmbd, R damping, R dt, vec3<R>& f, sym3<R>& H) {
  const R det_dm = dm[0] * (dm[4] * dm[8] - dm[5] * dm[7]) - dm[1] * (dm[3] * dm[8] - dm[5] * dm[6]) +
                   dm[2] * (dm[3] * dm[7] - dm[4] * dm[6]);
  const R vol = R(1) / (det_dm * R(6));
  const vec3<R> c1 = x[1] - x[0], c2 = x[2] - x[0], c3 = x[3] - x[0];
  const vec3<R> F0 = c1 * dm[0] + c2 * dm[3] + c3 * dm[6];
  const vec3<R> F1 = c1 * dm[1] + c2 * dm[4] + c3 * dm[7];
  const vec3<R> F2 = c1 * dm[2] + c2 * dm[5] + c3 * dm[8];
  const vec3<R> C0 = cross(F1, F2), C1 = cross(F2, F0), C2 = cross(F0, F1);
  const R J = dot(F0, C0);
  const R lnh = lmbd + mu;
  const R lsafe = (lnh < R(0) ? R(-1) : R(1)) * vmax(vabs(lnh), R(1.0e-6));
  const R alpha = R(1) + vdiv_fast(mu, lsafe);
  const R s = lnh * (J - alpha);
  // row selection by comparisons, not by a computed index, so that dm stays in registers
  vec3<R> m;
  if (ord == 0)
    m = {-(dm[0] + dm[3] + dm[6]), -(dm[1] + dm[4] + dm[7]), -(dm[2] + dm[5] + dm[8])};
  else if (ord == 1)
    m = {dm[0], dm[1], dm[2]};
  else if (ord == 2)
    m = {dm[3], dm[4], dm[5]};
  else
    m = {dm[6], dm[7], dm[8]};
  const vec3<R> Fm = F0 * m.x + F1 * m.y + F2 * m.z;
  const vec3<R> g = C0 * m.x + C1 * m.y + C2 * m.z;
  vec3<R> force = (-vol) * (mu * Fm + s * g);
  sym3<R> h = sdiag(vol * mu * dot(m, m));
  souter_add(h, g, vol * lnh);
  if (damping > R(0)) {
    const R inv_dt = R(1) / dt;
    const vec3<R> d0 = x[0] - xp[0];
    const vec3<R> e1 = ((x[1] - xp[1]) - d0) * inv_dt, e2 = ((x[2] - xp[2]) - d0) * inv_dt,
                  e3 = ((x[3] - xp[3]) - d0) * inv_dt;
    const vec3<R> G0 = e1 * dm[0] + e2 * dm[3] + e3 * dm[6];
    const vec3<R> G1 = e1 * dm[1] + e2 * dm[4] + e3 * dm[7];
    const vec3<R> G2 = e1 * dm[2] + e2 * dm[5] + e3 * dm[8];
    const R cfd = dot(C0, G0) + dot(C1, G1) + dot(C2, G2);
    force = force + (-damping * vol) * (mu * (G0 * m.x + G1 * m.y + G2 * m.z) + (lnh * cfd) * g);
    h = (R(1) + damping * inv_dt) * h;
  }
  f = f + force;
  H = H + h;
}

}  // namespace vbd
