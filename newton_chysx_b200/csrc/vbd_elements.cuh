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
//                wrinkles"), with N1 = x02 x x03, N2 = x13 x x12:
//                  dtheta/dx0 = -|e| / |N1| n1
//                  dtheta/dx1 = -|e| / |N2| n2
//                  dtheta/dx2 =  (x03 . e) / |N1| n1 + (x13 . e) / |N2| n2
//                  dtheta/dx3 = -(x02 . e) / |N1| n1 - (x12 . e) / |N2| n2
//                i.e. alpha n1 + beta n2 with two scalars chosen by the vertex's role, the same
//                instructions for every lane of a warp. Only the solved vertex's derivative is formed
//                unless damping needs all four.
//  * contact   - rigid_vbd_kernels.py:727-759, 891-934 (penalty, approach damping, IPC-smoothed
//                isotropic friction).
#pragma once
#include "vbd_math.cuh"

namespace vbd {

// Membrane contribution of one triangle for the vertex of order `ord` (0, 1, 2).
// pose = D^-1 row-major (00, 01, 10, 11); mat = (mu, lambda, damping, area).
template <typename R>
__host__ __device__ __forceinline__ void membrane_add(int ord, vec3<R> x0, vec3<R> x1, vec3<R> x2, const R pose[4],
                                                      R mu, R lmbd, R damping, R area, R dt, const vec3<R>* xp,
                                                      vec3<R>& f, sym3<R>& H) {
  const vec3<R> x01 = x1 - x0, x02 = x2 - x0;
  const R D00 = pose[0], D01 = pose[1], D10 = pose[2], D11 = pose[3];
  const vec3<R> f0 = x01 * D00 + x02 * D10;
  const vec3<R> f1 = x01 * D01 + x02 * D11;
  const R f00 = dot(f0, f0), f11 = dot(f1, f1), f01 = dot(f0, f1);
  const R Jsq = vmax(f00 * f11 - f01 * f01, R(1.0e-20));
  const R invJ = vrsqrt(Jsq);
  const R J = Jsq * invJ;
  const R lnh = lmbd + mu;
  const R lsafe = (lnh < R(0) ? R(-1) : R(1)) * vmax(vabs(lnh), R(1.0e-6));
  const R alpha = R(1) + mu / lsafe;
  const vec3<R> g0 = invJ * (f11 * f0 - f01 * f1);
  const vec3<R> g1 = invJ * (f00 * f1 - f01 * f0);
  const R s = lnh * (J - alpha);
  const R m0 = R(ord == 0), m1 = R(ord == 1), m2 = R(ord == 2);
  const R d0 = D00 * (m1 - m0) + D10 * (m2 - m0);
  const R d1 = D01 * (m1 - m0) + D11 * (m2 - m0);
  // force = -(P0 d0 + P1 d1),  P_i = mu f_i + s g_i
  vec3<R> force = -((mu * f0 + s * g0) * d0 + (mu * f1 + s * g1) * d1);
  const R r = vmax(R(0), s) * invJ;
  const vec3<R> dJ = g0 * d0 + g1 * d1;
  const vec3<R> w = f1 * d0 - f0 * d1;
  const R Ic = mu * (d0 * d0 + d1 * d1) + r * (d0 * d0 * f11 + d1 * d1 * f00 - R(2) * d0 * d1 * f01);
  sym3<R> h = sdiag(Ic);
  souter_add(h, dJ, lnh - r);
  souter_add(h, w, -r);
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
      const R kmu = mu * damping;
      force = force + (-kmu * dC) * dCdx;
      souter_add(h, dCdx, kmu * inv_dt);
      const R dCl = dG00 + dG11;
      const vec3<R> dCldx = d0 * f0 + d1 * f1;
      const R kl = lmbd * damping;
      force = force + (-kl * dCl) * dCldx;
      souter_add(h, dCldx, kl * inv_dt);
    }
  }
  f = f + force * area;
  H = H + area * h;
}

// Dihedral bending contribution of hinge (x0 opposite-0, x1 opposite-1, x2-x3 the shared edge) for
// the vertex of order `ord` (0..3). prop = (rest_angle, rest_length, ke, kd). xp = previous positions
// of the four vertices, read only when kd > 0.
template <typename R>
__host__ __device__ __forceinline__ void bending_add(int ord, const vec3<R> x[4], R rest_angle, R rest_length, R ke,
                                                     R kd, R dt, const vec3<R>* xp, vec3<R>& f, sym3<R>& H) {
  const vec3<R> x02 = x[2] - x[0], x03 = x[3] - x[0], x13 = x[3] - x[1], x12 = x[2] - x[1], e = x[3] - x[2];
  const vec3<R> N1 = cross(x02, x03), N2 = cross(x13, x12);
  const R s1 = dot(N1, N1), s2 = dot(N2, N2), se = dot(e, e);
  // |N1|, |N2|, |e| < 1e-6 (degenerate hinge): no contribution
  const R eps2 = R(1.0e-12);
  if (s1 < eps2 || s2 < eps2 || se < eps2) return;
  const R il1 = vrsqrt(s1), il2 = vrsqrt(s2), ile = vrsqrt(se);
  const vec3<R> n1 = N1 * il1, n2 = N2 * il2, eh = e * ile;
  const R s = dot(cross(n1, n2), eh);
  const R c = dot(n1, n2);
  const R theta = vatan2(s, c);
  const R k = ke * rest_length;
  const R dE = k * (theta - rest_angle);
  const R le = se * ile;  // |e|
  // dtheta/dx_ord = alpha n1 + beta n2
  R alpha, beta;
  if (ord <= 1) {
    alpha = ord == 0 ? -le * il1 : R(0);
    beta = ord == 1 ? -le * il2 : R(0);
  } else {
    const vec3<R> a1 = ord == 2 ? x03 : -x02;
    const vec3<R> a2 = ord == 2 ? x13 : -x12;
    alpha = dot(a1, eh) * il1;
    beta = dot(a2, eh) * il2;
  }
  const vec3<R> d = alpha * n1 + beta * n2;
  f = f + (-dE) * d;
  R hk = k;
  if (kd > R(0)) {
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

}  // namespace vbd
