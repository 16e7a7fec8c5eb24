// CPU oracle for the cloth Vertex Block Descent step. TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the reference algorithm (newton/_src/solvers/vbd), templated on the
// real type so that one source gives the FP32 oracle and the all-FP64 oracle. Only the test suite,
// the smoke check and the CPU-baseline leg of the benchmark may load this library; nothing in the
// product path calls it.
//
// Parity pins: tests/golden/*.npz hold outputs of the reference's own kernel bodies executed in
// float64 (tests/golden/make_golden.py); tests/test_oracle.py checks this file against them.
//
// Followed reference code (file:line within the reference project):
//   membrane   particle_vbd_kernels.py:865-1025   evaluate_neo_hookean_membrane_force_hessian
//   bending    particle_vbd_kernels.py:1028-1190  compute_normalized_vector_derivative,
//                                                 compute_angle_derivative,
//                                                 evaluate_dihedral_angle_based_bending_force_hessian
//   contact    rigid_vbd_kernels.py:314-330, 727-834, 891-934, 2318-2361, 3755-3799
//   step       particle_vbd_kernels.py:1782-1807 (forward_step), 1900-1903 (update_velocity),
//              2877-2897 (apply_truncation_ts), 2900-2967 (contact accumulation),
//              3135-3273 (solve_elasticity, the non-tile accumulation order)
//              solver_vbd.py:1575-1622, 1669-1766, 2151-2337, 2339-2376, 2763-2774 (sequencing)
//   adjacency  particle_vbd_kernels.py:639-738, 774-825 (count/fill order)
//   springs    particle_vbd_kernels.py:2299-2397; tetrahedra :154-224, 335-546 (stable Neo-Hookean)
//   contacts   geometry/kernels.py:1001-1140 for PLANE (infinite) and SPHERE shapes
//   self-contact particle_vbd_kernels.py:1193-1222 (barrier), 1225-1238 (damping), 1371-1506 (edge-edge),
//              1599-1745 (vertex-triangle), 1748-1779 (friction), 1930-2071 (accumulation),
//              2475-2741 (division planes, step fractions), 2744-2897 (truncation);
//              geometry/kernels.py:64-128 (triangle closest point), 1252-1497 (detection semantics);
//              math/__init__.py orthonormal_basis; solver_vbd.py:1669-1766, 2151-2337, 2834-2850
//   edge-edge closest points: Warp native (closest_point_edge_edge), restated from Ericson 2005 sec. 5.1.9
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>
#include <numeric>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename R>
struct V3 {
  R x, y, z;
};
template <typename R>
struct M3 {
  R m[3][3];
};

template <typename R> inline V3<R> v3(R a, R b, R c) { return {a, b, c}; }
template <typename R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <typename R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename R> inline V3<R> operator*(R s, V3<R> a) { return {a.x * s, a.y * s, a.z * s}; }
template <typename R> inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <typename R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R> inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }

template <typename R> inline M3<R> mzero() {
  M3<R> r;
  std::memset(&r, 0, sizeof(r));
  return r;
}
template <typename R> inline M3<R> ident() {
  M3<R> r = mzero<R>();
  r.m[0][0] = r.m[1][1] = r.m[2][2] = R(1);
  return r;
}
template <typename R> inline M3<R> operator+(M3<R> a, const M3<R>& b) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a.m[i][j] += b.m[i][j];
  return a;
}
template <typename R> inline M3<R> operator-(M3<R> a, const M3<R>& b) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a.m[i][j] -= b.m[i][j];
  return a;
}
template <typename R> inline M3<R> operator*(M3<R> a, R s) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a.m[i][j] *= s;
  return a;
}
template <typename R> inline M3<R> operator*(R s, M3<R> a) { return a * s; }
template <typename R> inline M3<R> operator/(M3<R> a, R s) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a.m[i][j] /= s;
  return a;
}
template <typename R> inline M3<R> operator-(M3<R> a) { return a * R(-1); }
template <typename R> inline M3<R> operator*(const M3<R>& a, const M3<R>& b) {
  M3<R> r = mzero<R>();
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) r.m[i][j] += a.m[i][k] * b.m[k][j];
  return r;
}
template <typename R> inline V3<R> operator*(const M3<R>& a, V3<R> v) {
  return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z, a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
          a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
template <typename R> inline M3<R> transpose(const M3<R>& a) {
  M3<R> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
  return r;
}
template <typename R> inline M3<R> outer(V3<R> a, V3<R> b) {
  M3<R> r;
  R av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = av[i] * bv[j];
  return r;
}
template <typename R> inline M3<R> skew(V3<R> a) {
  M3<R> r = mzero<R>();
  r.m[0][1] = -a.z;
  r.m[0][2] = a.y;
  r.m[1][0] = a.z;
  r.m[1][2] = -a.x;
  r.m[2][0] = -a.y;
  r.m[2][1] = a.x;
  return r;
}
template <typename R> inline R det(const M3<R>& a) {
  return a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
         a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
         a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
}
// Inverse by adjugate / determinant (the standard closed form).
template <typename R> inline M3<R> inverse(const M3<R>& a, R d) {
  M3<R> r;
  R inv = R(1) / d;
  r.m[0][0] = (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) * inv;
  r.m[0][1] = (a.m[0][2] * a.m[2][1] - a.m[0][1] * a.m[2][2]) * inv;
  r.m[0][2] = (a.m[0][1] * a.m[1][2] - a.m[0][2] * a.m[1][1]) * inv;
  r.m[1][0] = (a.m[1][2] * a.m[2][0] - a.m[1][0] * a.m[2][2]) * inv;
  r.m[1][1] = (a.m[0][0] * a.m[2][2] - a.m[0][2] * a.m[2][0]) * inv;
  r.m[1][2] = (a.m[0][2] * a.m[1][0] - a.m[0][0] * a.m[1][2]) * inv;
  r.m[2][0] = (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]) * inv;
  r.m[2][1] = (a.m[0][1] * a.m[2][0] - a.m[0][0] * a.m[2][1]) * inv;
  r.m[2][2] = (a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0]) * inv;
  return r;
}
template <typename R> inline R rmax(R a, R b) { return a > b ? a : b; }
template <typename R> inline R rmin(R a, R b) { return a < b ? a : b; }
template <typename R> inline R rsign(R a) { return a < R(0) ? R(-1) : R(1); }

// ------------------------------------------------------------------------------------ membrane
// particle_vbd_kernels.py:865-1025 (stable Neo-Hookean membrane, Rayleigh damping on ||G||_F, tr G)
template <typename R>
void membrane(int v_order, V3<R> x0, V3<R> x1, V3<R> x2, V3<R> p0, V3<R> p1, V3<R> p2, const R pose[4], R area,
              R mu, R lmbd, R damping, R dt, V3<R>& force, M3<R>& hessian) {
  V3<R> x01 = x1 - x0, x02 = x2 - x0;
  R D00 = pose[0], D01 = pose[1], D10 = pose[2], D11 = pose[3];
  V3<R> f0 = x01 * D00 + x02 * D10;
  V3<R> f1 = x01 * D01 + x02 * D11;
  R f0f0 = dot(f0, f0), f1f1 = dot(f1, f1), f0f1 = dot(f0, f1);
  R Jsq = f0f0 * f1f1 - f0f1 * f0f1;
  Jsq = rmax(Jsq, R(1.0e-20));
  R J = std::sqrt(Jsq);
  R invJ = R(1) / J;
  R mu_nh = mu;
  R l_nh = lmbd + mu;
  R l_safe = rsign(l_nh) * rmax(std::fabs(l_nh), R(1.0e-6));
  R alpha = R(1) + mu_nh / l_safe;
  V3<R> g0 = invJ * (f1f1 * f0 - f0f1 * f1);
  V3<R> g1 = invJ * (f0f0 * f1 - f0f1 * f0);
  R s = l_nh * (J - alpha);
  V3<R> P0 = mu_nh * f0 + s * g0;
  V3<R> P1 = mu_nh * f1 + s * g1;
  R m0 = R(v_order == 0), m1 = R(v_order == 1), m2 = R(v_order == 2);
  R df0 = D00 * (m1 - m0) + D10 * (m2 - m0);
  R df1 = D01 * (m1 - m0) + D11 * (m2 - m0);
  force = -(P0 * df0 + P1 * df1);
  R s_clamp = rmax(R(0), s);
  R r = s_clamp * invJ;
  R c1 = l_nh - r;
  R df0sq = df0 * df0, df1sq = df1 * df1;
  V3<R> dJ = g0 * df0 + g1 * df1;
  V3<R> w = f1 * df0 - f0 * df1;
  R Ic = mu_nh * (df0sq + df1sq) + r * (df0sq * f1f1 + df1sq * f0f0 - R(2) * df0 * df1 * f0f1);
  hessian = Ic * ident<R>() + c1 * outer(dJ, dJ) - r * outer(w, w);
  if (damping > R(0)) {
    R G00 = R(0.5) * (f0f0 - R(1)), G11 = R(0.5) * (f1f1 - R(1)), G01 = R(0.5) * f0f1;
    R Gsq = G00 * G00 + G11 * G11 + R(2) * G01 * G01;
    if (Gsq >= R(1.0e-20)) {
      R inv_dt = R(1) / dt;
      V3<R> p01 = p1 - p0, p02 = p2 - p0;
      V3<R> vx01 = (x01 - p01) * inv_dt, vx02 = (x02 - p02) * inv_dt;
      V3<R> df0dt = vx01 * D00 + vx02 * D10;
      V3<R> df1dt = vx01 * D01 + vx02 * D11;
      R Cmu = std::sqrt(Gsq);
      R n00 = G00 / Cmu, n01 = G01 / Cmu, n11 = G11 / Cmu;
      R dG00 = dot(f0, df0dt), dG11 = dot(f1, df1dt);
      R dG01 = R(0.5) * (dot(f0, df1dt) + dot(f1, df0dt));
      R dCmu_dt = n00 * dG00 + n11 * dG11 + R(2) * n01 * dG01;
      V3<R> dCmu0 = n00 * f0 + n01 * f1;
      V3<R> dCmu1 = n01 * f0 + n11 * f1;
      V3<R> dCmu_dx = df0 * dCmu0 + df1 * dCmu1;
      R kd_mu = mu * damping;
      force = force + (-kd_mu * dCmu_dt) * dCmu_dx;
      hessian = hessian + (kd_mu * inv_dt) * outer(dCmu_dx, dCmu_dx);
      R dCl_dt = dG00 + dG11;
      V3<R> dCl_dx = df0 * f0 + df1 * f1;
      R kd_l = lmbd * damping;
      force = force + (-kd_l * dCl_dt) * dCl_dx;
      hessian = hessian + (kd_l * inv_dt) * outer(dCl_dx, dCl_dx);
    }
  }
  force = force * area;
  hessian = hessian * area;
}

// ------------------------------------------------------------------------------------ bending
// particle_vbd_kernels.py:1028-1054
template <typename R> M3<R> normalized_vector_derivative(R len, V3<R> nhat, const M3<R>& dvec) {
  M3<R> P = ident<R>() - outer(nhat, nhat);
  return (R(1) / len) * (P * dvec);
}
template <typename R>
V3<R> angle_derivative(V3<R> n1, V3<R> n2, V3<R> e, const M3<R>& dn1, const M3<R>& dn2, R s, R c, const M3<R>& sk1,
                       const M3<R>& sk2) {
  V3<R> dsin = transpose(sk1 * dn2 - sk2 * dn1) * e;
  V3<R> dcos = transpose(dn1) * n2 + transpose(dn2) * n1;
  return dsin * c - dcos * s;
}

// particle_vbd_kernels.py:1057-1190 (dihedral-angle bending, all four angle derivatives)
template <typename R>
void bending(int v_order, const V3<R> x[4], const V3<R> xp[4], bool boundary, R rest_angle, R rest_length, R stiffness,
             R damping, R dt, V3<R>& force, M3<R>& hessian) {
  force = v3<R>(0, 0, 0);
  hessian = mzero<R>();
  if (boundary) return;
  const R eps = R(1.0e-6);
  V3<R> x0 = x[0], x1 = x[1], x2 = x[2], x3 = x[3];
  V3<R> x02 = x2 - x0, x03 = x3 - x0, x13 = x3 - x1, x12 = x2 - x1, e = x3 - x2;
  V3<R> n1 = cross(x02, x03), n2 = cross(x13, x12);
  R n1n = length(n1), n2n = length(n2), en = length(e);
  if (n1n < eps || n2n < eps || en < eps) return;
  V3<R> n1h = n1 / n1n, n2h = n2 / n2n, eh = e / en;
  R s = dot(cross(n1h, n2h), eh);
  R c = dot(n1h, n2h);
  R theta = std::atan2(s, c);
  R k = stiffness * rest_length;
  R dE = k * (theta - rest_angle);
  M3<R> sk_e = skew(e), sk_x03 = skew(x03), sk_x02 = skew(x02), sk_x13 = skew(x13), sk_x12 = skew(x12);
  M3<R> sk_n1 = skew(n1h), sk_n2 = skew(n2h);
  M3<R> Z = mzero<R>();
  M3<R> dn1_0 = normalized_vector_derivative(n1n, n1h, sk_e);
  M3<R> dn2_1 = normalized_vector_derivative(n2n, n2h, -sk_e);
  M3<R> dn1_2 = normalized_vector_derivative(n1n, n1h, -sk_x03);
  M3<R> dn2_2 = normalized_vector_derivative(n2n, n2h, sk_x13);
  M3<R> dn1_3 = normalized_vector_derivative(n1n, n1h, sk_x02);
  M3<R> dn2_3 = normalized_vector_derivative(n2n, n2h, -sk_x12);
  V3<R> dth[4];
  dth[0] = angle_derivative(n1h, n2h, eh, dn1_0, Z, s, c, sk_n1, sk_n2);
  dth[1] = angle_derivative(n1h, n2h, eh, Z, dn2_1, s, c, sk_n1, sk_n2);
  dth[2] = angle_derivative(n1h, n2h, eh, dn1_2, dn2_2, s, c, sk_n1, sk_n2);
  dth[3] = angle_derivative(n1h, n2h, eh, dn1_3, dn2_3, s, c, sk_n1, sk_n2);
  V3<R> d = dth[v_order];
  force = -dE * d;
  hessian = k * outer(d, d);
  if (damping > R(0)) {
    R inv_dt = R(1) / dt;
    R dtheta_dt = (dot(dth[0], x0 - xp[0]) + dot(dth[1], x1 - xp[1]) + dot(dth[2], x2 - xp[2]) +
                   dot(dth[3], x3 - xp[3])) *
                  inv_dt;
    R dc = damping * k;
    force = force + (-dc * dtheta_dt) * d;
    hessian = hessian + (dc * inv_dt) * outer(d, d);
  }
}

// ------------------------------------------------------------------------------------ contact
// rigid_vbd_kernels.py:891-934 (isotropic friction with IPC regularisation)
template <typename R>
void friction(R mu, R normal_load, V3<R> n, V3<R> u, R eps_u, V3<R>& f, M3<R>& K) {
  R dnu = dot(n, u);
  V3<R> ut = u - n * dnu;
  R un = length(ut);
  if (un > R(0)) {
    R f1 = un > eps_u ? R(1) / un : (-un / eps_u + R(2)) / eps_u;
    R scale = mu * normal_load * f1;
    f = -(scale * ut);
    K = scale * (ident<R>() - outer(n, n));
  } else {
    f = v3<R>(0, 0, 0);
    K = mzero<R>();
  }
}

// rigid_vbd_kernels.py:727-759 (penalty + damping + friction)
template <typename R>
void contact_force(R pen, V3<R> n, V3<R> rel, R ke, R kd, R mu, R fric_eps, R dt, V3<R>& force, M3<R>& hessian) {
  R fn = pen * ke;
  force = n * fn;
  hessian = ke * outer(n, n);
  if (dot(n, rel) < R(0)) {
    R dc = kd * ke;
    M3<R> Hd = (dc / dt) * outer(n, n);
    hessian = hessian + Hd;
    force = force - Hd * rel;
  }
  V3<R> ff;
  M3<R> fH;
  friction(mu, fn, n, rel, fric_eps * dt, ff, fH);
  force = force + ff;
  hessian = hessian + fH;
}

// ------------------------------------------------------------------------------------ springs, tetrahedra
// particle_vbd_kernels.py:2299-2343 (evaluate_spring_force_and_hessian_both_vertices): forces on both
// endpoints and the shared Hessian k (I - l0/l (I - d d^T / l^2)) plus damping (kd/dt) H.
template <typename R>
void spring_both(V3<R> x0, V3<R> x1, V3<R> xa0, V3<R> xa1, R l0, R ke, R kd, R dt, V3<R>& f0, V3<R>& f1, M3<R>& Ht) {
  const V3<R> diff = x0 - x1;
  R len = length(diff);
  len = rmax(len, R(1e-8));
  const V3<R> base = (ke * (l0 - len) / len) * diff;
  const M3<R> I = ident<R>();
  const M3<R> Hs = ke * (I - (l0 / len) * (I - outer(diff, diff) / (len * len)));
  const M3<R> hd = Hs * (kd / dt);
  f0 = base + hd * (xa0 - x0);
  f1 = -base + hd * (xa1 - x1);
  Ht = Hs + hd;
}

// particle_vbd_kernels.py:335-473 (evaluate_volumetric_neo_hookean_force_and_hessian) with the vertex block
// of assemble_tet_vertex_force_and_hessian (:154-224) written out: with P = V (mu F + s cof(F)) and the
// 9x9 Hessian V (mu I + lambda_nh c c^T), c = vec(cof F), the block for the vertex with row m of the rest
// inverse is  f = -V (mu F m + s cof(F) m),  h = V (mu |m|^2 I + lambda_nh g g^T),  g = cof(F) m.
template <typename R>
void tet_force(int order, const V3<R> x[4], const V3<R> xp[4], const R Dinv[9], R mu, R lmbd, R damping, R dt, V3<R>& f,
               M3<R>& h) {
  M3<R> D;
  for (int i = 0; i < 9; ++i) D.m[i / 3][i % 3] = Dinv[i];
  const R rest_volume = R(1) / (det(D) * R(6));
  M3<R> Ds;
  const V3<R> c1 = x[1] - x[0], c2 = x[2] - x[0], c3 = x[3] - x[0];
  Ds.m[0][0] = c1.x, Ds.m[1][0] = c1.y, Ds.m[2][0] = c1.z;
  Ds.m[0][1] = c2.x, Ds.m[1][1] = c2.y, Ds.m[2][1] = c2.z;
  Ds.m[0][2] = c3.x, Ds.m[1][2] = c3.y, Ds.m[2][2] = c3.z;
  const M3<R> F = Ds * D;
  const R J = det(F);
  const R mu_nh = mu, lmbd_nh = lmbd + mu;
  const R lsafe = rsign(lmbd_nh) * rmax(std::fabs(lmbd_nh), R(1e-6));
  const R alpha = R(1) + mu_nh / lsafe;
  M3<R> cof;  // cofactor: cof[a][i] = d det F / d F[a][i]
  cof.m[0][0] = F.m[1][1] * F.m[2][2] - F.m[1][2] * F.m[2][1];
  cof.m[0][1] = F.m[1][2] * F.m[2][0] - F.m[1][0] * F.m[2][2];
  cof.m[0][2] = F.m[1][0] * F.m[2][1] - F.m[1][1] * F.m[2][0];
  cof.m[1][0] = F.m[0][2] * F.m[2][1] - F.m[0][1] * F.m[2][2];
  cof.m[1][1] = F.m[0][0] * F.m[2][2] - F.m[0][2] * F.m[2][0];
  cof.m[1][2] = F.m[0][1] * F.m[2][0] - F.m[0][0] * F.m[2][1];
  cof.m[2][0] = F.m[0][1] * F.m[1][2] - F.m[0][2] * F.m[1][1];
  cof.m[2][1] = F.m[0][2] * F.m[1][0] - F.m[0][0] * F.m[1][2];
  cof.m[2][2] = F.m[0][0] * F.m[1][1] - F.m[0][1] * F.m[1][0];
  const R s = lmbd_nh * (J - alpha);
  V3<R> m;
  if (order == 0)
    m = v3<R>(-(Dinv[0] + Dinv[3] + Dinv[6]), -(Dinv[1] + Dinv[4] + Dinv[7]), -(Dinv[2] + Dinv[5] + Dinv[8]));
  else
    m = v3<R>(Dinv[3 * (order - 1)], Dinv[3 * (order - 1) + 1], Dinv[3 * (order - 1) + 2]);
  const V3<R> Fm = F * m, g = cof * m;
  f = (-rest_volume) * (mu_nh * Fm + s * g);
  h = rest_volume * ((mu_nh * dot(m, m)) * ident<R>() + lmbd_nh * outer(g, g));
  if (damping > R(0)) {
    const R inv_dt = R(1) / dt;
    M3<R> Dd;
    const V3<R> d0 = x[0] - xp[0];
    const V3<R> e1 = ((x[1] - xp[1]) - d0) * inv_dt, e2 = ((x[2] - xp[2]) - d0) * inv_dt, e3 = ((x[3] - xp[3]) - d0) * inv_dt;
    Dd.m[0][0] = e1.x, Dd.m[1][0] = e1.y, Dd.m[2][0] = e1.z;
    Dd.m[0][1] = e2.x, Dd.m[1][1] = e2.y, Dd.m[2][1] = e2.z;
    Dd.m[0][2] = e3.x, Dd.m[1][2] = e3.y, Dd.m[2][2] = e3.z;
    const M3<R> Fd = Dd * D;
    R cfd = 0;  // c . vec(F_dot)
    for (int a = 0; a < 3; ++a)
      for (int i = 0; i < 3; ++i) cfd += cof.m[a][i] * Fd.m[a][i];
    // P_damp = damping V (mu vec(F_dot) + lambda_nh c (c . vec(F_dot))), contracted with m
    f = f + (-damping * rest_volume) * (mu_nh * (Fd * m) + (lmbd_nh * cfd) * g);
    h = h * (R(1) + damping * inv_dt);
  }
}

// ------------------------------------------------------------------------------------ model
struct Model {
  int n, T, E, C, S;
  const double *mass, *inv_mass, *radius;
  const int* flags;
  const int* tri_indices;
  const double *tri_poses, *tri_materials, *tri_areas;
  const int* edge_indices;
  const double *edge_rest_angle, *edge_rest_length, *edge_bending_properties;
  const int *adj_face_offsets, *adj_faces, *adj_edge_offsets, *adj_edges;
  const int *color_offsets, *color_particles, *particle_colors;
  const double* gravity;
  double soft_ke, soft_kd, soft_mu;
  const double *shape_ke, *shape_kd, *shape_mu;
  double friction_epsilon, beta;
  // springs and tetrahedra (0 / null when the model has none)
  int spring_count;
  const int* spring_indices;  // [2 * spring_count]
  const double *spring_rest_length, *spring_stiffness, *spring_damping;
  int tet_count;
  const int* tet_indices;          // [4 * tet_count]
  const double *tet_poses, *tet_materials;  // rest D^-1 (row-major 3x3), (mu, lambda, damping)
  const int *adj_tet_offsets, *adj_tets;    // reference layout: two ints (tet, order) per entry
};

// Particle-shape contacts, and the bodies that carry shapes: shape_body[s] (-1 = static; NULL = all static),
// body_q / body_q_prev [B,7] (p, quat xyzw), body_qd [B,6] (linear, angular), body_com [B,3]; body_q_prev NULL
// when the body velocity comes from body_qd.
struct Contacts {
  int count, max;
  const int *particle, *shape;
  const double *body_pos, *body_vel, *normal;
  const int* shape_body;
  const double *body_q, *body_q_prev, *body_qd, *body_com;
};

template <typename R> inline V3<R> ld(const double* a, int i) { return {R(a[3 * i]), R(a[3 * i + 1]), R(a[3 * i + 2])}; }
template <typename R> inline V3<R> ld(const std::vector<V3<R>>& a, int i) { return a[i]; }

// v rotated by the unit quaternion q = (x, y, z, w) (wp.quat_rotate), in R.
template <typename R> inline V3<R> quat_rotate(const double* q, V3<R> v) {
  const V3<R> u = {R(q[0]), R(q[1]), R(q[2])};
  const R w = R(q[3]);
  return v * (R(2) * w * w - R(1)) + cross(u, v) * (R(2) * w) + u * (R(2) * dot(u, v));
}

// Body of contact c's shape, or -1.
inline int contact_body(const Contacts& C, int c) { return C.shape_body && C.body_q ? C.shape_body[C.shape[c]] : -1; }

// World position of contact c's point: transform_point(body_q[body], body_pos) (_eval_body_particle_contact,
// rigid_vbd_kernels.py:790-799; update_duals_body_particle_contacts, rigid_vbd_kernels.py:3755-3799).
template <typename R> inline V3<R> contact_point(const Contacts& C, int c) {
  const V3<R> bp = ld<R>(C.body_pos, c);
  const int b = contact_body(C, c);
  if (b < 0) return bp;
  const double* X = C.body_q + 7 * b;
  return quat_rotate<R>(X + 3, bp) + V3<R>{R(X[0]), R(X[1]), R(X[2])};
}

// Velocity of contact c's point (rigid_vbd_kernels.py:806-819): from the body's motion over the step when
// body_q_prev is given, else from its spatial velocity about its centre of mass; plus the contact's own velocity
// rotated into world.
template <typename R> inline V3<R> contact_velocity(const Contacts& C, int c, V3<R> bx, R dt) {
  const V3<R> bvl = ld<R>(C.body_vel, c);
  const int b = contact_body(C, c);
  if (b < 0) return bvl;
  const double* X = C.body_q + 7 * b;
  const V3<R> vrot = quat_rotate<R>(X + 3, bvl);
  if (C.body_q_prev) {
    const double* Xp = C.body_q_prev + 7 * b;
    const V3<R> bxp = quat_rotate<R>(Xp + 3, ld<R>(C.body_pos, c)) + V3<R>{R(Xp[0]), R(Xp[1]), R(Xp[2])};
    return (bx - bxp) / dt + vrot;
  }
  const V3<R> com = C.body_com ? ld<R>(C.body_com, b) : V3<R>{R(0), R(0), R(0)};
  const V3<R> r = bx - (quat_rotate<R>(X + 3, com) + V3<R>{R(X[0]), R(X[1]), R(X[2])});
  V3<R> v = {R(0), R(0), R(0)}, w = {R(0), R(0), R(0)};
  if (C.body_qd) {
    v = V3<R>{R(C.body_qd[6 * b]), R(C.body_qd[6 * b + 1]), R(C.body_qd[6 * b + 2])};
    w = V3<R>{R(C.body_qd[6 * b + 3]), R(C.body_qd[6 * b + 4]), R(C.body_qd[6 * b + 5])};
  }
  return v + cross(w, r) + vrot;
}

// ------------------------------------------------------------------------------------ self-contact
// Closest point on triangle (a, b, c) to p, with the reference's branch order
// (geometry/kernels.py:64-128): vertex regions A, B, C first, then edges AB, AC, BC, then the interior.
// feature: 0..2 vertex A..C, 3 edge AB, 4 edge AC, 5 edge BC, 6 interior.
template <typename R>
V3<R> tri_closest(V3<R> a, V3<R> b, V3<R> c, V3<R> p, R bary[3], int& feature) {
  const V3<R> ab = b - a, ac = c - a, ap = p - a;
  const R d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= R(0) && d2 <= R(0)) {
    bary[0] = 1, bary[1] = 0, bary[2] = 0, feature = 0;
    return a;
  }
  const V3<R> bp = p - b;
  const R d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= R(0) && d4 <= d3) {
    bary[0] = 0, bary[1] = 1, bary[2] = 0, feature = 1;
    return b;
  }
  const V3<R> cp = p - c;
  const R d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= R(0) && d5 <= d6) {
    bary[0] = 0, bary[1] = 0, bary[2] = 1, feature = 2;
    return c;
  }
  const R vc = d1 * d4 - d3 * d2;
  if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
    const R v = d1 / (d1 - d3);
    bary[0] = R(1) - v, bary[1] = v, bary[2] = 0, feature = 3;
    return a + v * ab;
  }
  const R vb = d5 * d2 - d1 * d6;
  if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
    const R v = d2 / (d2 - d6);
    bary[0] = R(1) - v, bary[1] = 0, bary[2] = v, feature = 4;
    return a + v * ac;
  }
  const R va = d3 * d6 - d5 * d4;
  if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
    const R v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    bary[0] = 0, bary[1] = R(1) - v, bary[2] = v, feature = 5;
    return b + v * (c - b);
  }
  const R denom = R(1) / (va + vb + vc);
  const R v = vb * denom, w = vc * denom;
  bary[0] = R(1) - v - w, bary[1] = v, bary[2] = w, feature = 6;
  return a + v * ab + w * ac;
}

template <typename R> inline R rclamp(R x, R lo, R hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Closest points of segments p1-q1 and p2-q2 (s, t and their distance). Warp's closest_point_edge_edge
// is native code outside the reference tree; this restates the published segment-segment method
// (C. Ericson, Real-Time Collision Detection, 2005, sec. 5.1.9), eps bounding the squared lengths of
// degenerate segments. Exactly parallel segments take s = 0.
template <typename R>
void edge_closest(V3<R> p1, V3<R> q1, V3<R> p2, V3<R> q2, R eps, R& s, R& t, R& dist) {
  const V3<R> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
  const R a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  if (a <= eps && e <= eps) {
    s = t = R(0);
  } else if (a <= eps) {
    s = R(0);
    t = rclamp(f / e, R(0), R(1));
  } else {
    const R c = dot(d1, r);
    if (e <= eps) {
      t = R(0);
      s = rclamp(-c / a, R(0), R(1));
    } else {
      const R b = dot(d1, d2);
      const R denom = a * e - b * b;
      s = denom != R(0) ? rclamp((b * f - c * e) / denom, R(0), R(1)) : R(0);
      t = (b * s + f) / e;
      if (t < R(0)) {
        t = R(0);
        s = rclamp(-c / a, R(0), R(1));
      } else if (t > R(1)) {
        t = R(1);
        s = rclamp((b - c) / a, R(0), R(1));
      }
    }
  }
  dist = length((p1 + d1 * s) - (p2 + d2 * t));
}

// math/__init__.py orthonormal_basis
template <typename R>
void onb(V3<R> n, V3<R>& b1, V3<R>& b2) {
  if (n.z < R(0)) {
    const R a = R(1) / (R(1) - n.z), b = n.x * n.y * a;
    b1 = v3<R>(R(1) - n.x * n.x * a, -b, n.x);
    b2 = v3<R>(b, n.y * n.y * a - R(1), -n.y);
  } else {
    const R a = R(1) / (R(1) + n.z), b = -n.x * n.y * a;
    b1 = v3<R>(R(1) - n.x * n.x * a, b, -n.x);
    b2 = v3<R>(b, R(1) - n.y * n.y * a, -n.y);
  }
}

// particle_vbd_kernels.py:1193-1222: dE/dd and d2E/dd2 of the self-contact barrier
template <typename R>
void sc_norm(R dis, R radius, R k, R& dEdD, R& d2E) {
  const R tau = radius * R(0.5), d_min = R(1.0e-5);
  if (tau > dis && dis > d_min) {
    const R k2 = tau * tau * k;
    dEdD = -k2 / dis;
    d2E = k2 / (dis * dis);
  } else if (dis <= d_min) {
    const R k2 = tau * tau * k;
    const R dm2 = d_min * d_min;
    dEdD = k2 * (dis - R(2) * d_min) / dm2;
    d2E = k2 / dm2;
  } else {
    dEdD = -k * (radius - dis);
    d2E = k;
  }
}

// particle_vbd_kernels.py:1748-1779 (compute_friction with T = [b1 b2])
template <typename R>
void sc_friction(R mu, R fn, V3<R> b1, V3<R> b2, V3<R> dx, R eps_u, V3<R>& f, M3<R>& H) {
  const R u0 = dot(b1, dx), u1 = dot(b2, dx);
  const R un = std::sqrt(u0 * u0 + u1 * u1);
  if (un > R(0)) {
    const R f1 = un > eps_u ? R(1) / un : (-un / eps_u + R(2)) / eps_u;
    f = (-mu * fn) * ((f1 * u0) * b1 + (f1 * u1) * b2);
    H = (mu * fn * f1) * (outer(b1, b1) + outer(b2, b2));
  } else {
    f = v3<R>(0, 0, 0);
    H = mzero<R>();
  }
}

// particle_vbd_kernels.py:1225-1238
template <typename R>
void sc_damp(V3<R> disp, V3<R> n, const M3<R>& H, R kd, R dt, V3<R>& f, M3<R>& Hd) {
  if (dot(disp, n) > R(0)) {
    Hd = (kd / dt) * H;
    f = Hd * disp;
  } else {
    f = v3<R>(0, 0, 0);
    Hd = mzero<R>();
  }
}

// Vertex-triangle contact on all four vertices (particle_vbd_kernels.py:1599-1745).
// x = (a, b, c, p), xa = the same at the start of the step.
template <typename R>
bool sc_vt(const V3<R> x[4], const V3<R> xa[4], R radius, R ke, R kd, R mu, R eps, R dt, V3<R> f[4], M3<R> H[4]) {
  R bary[3];
  int feat;
  const V3<R> cp = tri_closest(x[0], x[1], x[2], x[3], bary, feat);
  const V3<R> diff = x[3] - cp;
  const R dis = length(diff);
  const V3<R> n = diff / dis;
  if (!(R(0) < dis && dis < radius)) return false;
  const R bs[4] = {-bary[0], -bary[1], -bary[2], R(1)};
  R dEdD, d2E;
  sc_norm(dis, radius, ke, dEdD, d2E);
  const V3<R> cf = -dEdD * n;
  const M3<R> cH = d2E * outer(n, n);
  const V3<R> cpp = bary[0] * xa[0] + bary[1] * xa[1] + bary[2] * xa[2];
  const V3<R> dx = (x[3] - xa[3]) - (cp - cpp);
  V3<R> b1, b2;
  onb(n, b1, b2);
  V3<R> ff;
  M3<R> fH;
  sc_friction(mu, -dEdD, b1, b2, dx, eps * dt, ff, fH);
  const R sgn[4] = {R(-1), R(-1), R(-1), R(1)};
  for (int k = 0; k < 4; ++k) {
    f[k] = cf * bs[k];
    H[k] = cH * bs[k] * bs[k];
    V3<R> df;
    M3<R> dH;
    sc_damp(xa[k] - x[k], n * sgn[k], H[k], kd, dt, df, dH);
    f[k] = f[k] + (df + bs[k] * ff);
    H[k] = H[k] + (dH + (bs[k] * bs[k]) * fH);
  }
  return true;
}

// Edge-edge contact on the two vertices of the first edge (particle_vbd_kernels.py:1371-1506).
// x = (e1.v0, e1.v1, e2.v0, e2.v1).
template <typename R>
bool sc_ee(const V3<R> x[4], const V3<R> xa[4], R radius, R ke, R kd, R mu, R eps, R dt, R ee_eps, V3<R> f[2],
           M3<R> H[2]) {
  R s, t, dis;
  edge_closest(x[0], x[1], x[2], x[3], ee_eps, s, t, dis);
  const V3<R> c1 = x[0] + (x[1] - x[0]) * s, c2 = x[2] + (x[3] - x[2]) * t;
  const V3<R> n = (c1 - c2) / dis;
  if (!(R(0) < dis && dis < radius)) return false;
  const R bs[2] = {R(1) - s, s};
  R dEdD, d2E;
  sc_norm(dis, radius, ke, dEdD, d2E);
  const V3<R> cf = -dEdD * n;
  const M3<R> cH = d2E * outer(n, n);
  const V3<R> c1p = xa[0] + (xa[1] - xa[0]) * s, c2p = xa[2] + (xa[3] - xa[2]) * t;
  const V3<R> dx = (c1 - c1p) - (c2 - c2p);
  V3<R> b1, b2;
  onb(n, b1, b2);
  V3<R> ff;
  M3<R> fH;
  sc_friction(mu, -dEdD, b1, b2, dx, eps * dt, ff, fH);
  for (int k = 0; k < 2; ++k) {
    f[k] = cf * bs[k];
    H[k] = cH * bs[k] * bs[k];
    V3<R> df;
    M3<R> dH;
    sc_damp(xa[k] - x[k], n, H[k], kd, dt, df, dH);
    f[k] = f[k] + (df + bs[k] * ff);
    H[k] = H[k] + (dH + (bs[k] * bs[k]) * fH);
  }
  return true;
}

// particle_vbd_kernels.py:2475-2498 (coplanar segments never count here)
template <typename R>
bool seg_plane(V3<R> v, V3<R> dv, V3<R> n, V3<R> d, R eps_par, R near, R far) {
  const R nv = dot(n, dv), num = -dot(n, v - d);
  if (std::fabs(nv) < eps_par) return false;
  const R t = num / nv;
  return t >= near && t <= R(1) + far;
}

template <typename R> inline V3<R> normalize(V3<R> a) {
  const R l = length(a);
  return l > R(0) ? a / l : v3<R>(0, 0, 0);
}

// particle_vbd_kernels.py:2500-2558. x = (v, t1, t2, t3), dx their displacements; dummy[k] = no cut.
template <typename R>
void vt_plane(const V3<R> x[4], const V3<R> dx[4], bool dummy[4], V3<R>& n, V3<R>& d) {
  R bary[3];
  int feat;
  const V3<R> cp = tri_closest(x[1], x[2], x[3], x[0], bary, feat);
  const V3<R> nh = x[0] - cp;
  if (length(nh) < R(1e-12)) {
    for (int k = 0; k < 4; ++k) dummy[k] = false;
    n = v3<R>(0, 0, 0);
    d = x[0];
    return;
  }
  n = normalize(nh);
  const R dvn = rmax(-dot(n, dx[0]), R(0));
  const R dtn = rmax(rmax(dot(n, dx[1]), dot(n, dx[2])), rmax(dot(n, dx[3]), R(0)));
  if (dtn + dvn == R(0)) {
    d = cp + R(0.5) * nh;
  } else {
    const R l = rclamp(dtn / (dtn + dvn), R(0.05), R(0.95));
    d = cp + l * nh;
  }
  dummy[0] = dvn == R(0) ? true : !seg_plane(x[0], dx[0], n, d, R(1e-6), R(-1e-8), R(1e-8));
  for (int k = 1; k < 4; ++k)
    dummy[k] = dtn == R(0) ? true : !seg_plane(x[k], dx[k], n, d, R(1e-6), R(-1e-8), R(1e-8));
}

// particle_vbd_kernels.py:2561-2628
template <typename R>
V3<R> robust_pair_normal(V3<R> a0, V3<R> a1, V3<R> b0, V3<R> b1, R eps = R(1e-6)) {
  V3<R> d0 = a1 - a0, d1 = b1 - b0;
  const R l0 = length(d0), l1 = length(d1);
  d0 = l0 > eps ? d0 / l0 : v3<R>(0, 0, 0);
  d1 = l1 > eps ? d1 / l1 : v3<R>(0, 0, 0);
  V3<R> n = cross(d0, d1);
  R ln = length(n);
  if (ln > eps) return n / ln;
  V3<R> ref = d0;
  if (length(ref) <= eps) ref = d1;
  if (length(ref) <= eps) return v3<R>(1, 0, 0);
  const V3<R> bridge = R(0.5) * ((b0 + b1) - (a0 + a1));
  const R bl = length(bridge);
  if (bl > eps) {
    n = cross(ref, bridge / bl);
    ln = length(n);
    if (ln > eps) return n / ln;
  }
  V3<R> axis = v3<R>(1, 0, 0);
  if (std::fabs(dot(ref, axis)) > R(0.9)) axis = v3<R>(0, 1, 0);
  n = cross(ref, axis);
  ln = length(n);
  if (ln > eps) return n / ln;
  n = cross(ref, v3<R>(0, 0, 1));
  ln = length(n);
  if (ln > eps) return n / ln;
  return v3<R>(1, 0, 0);
}

// particle_vbd_kernels.py:2631-2702. x = (e0.v0, e0.v1, e1.v0, e1.v1).
template <typename R>
void ee_plane(const V3<R> x[4], const V3<R> dx[4], bool dummy[4], V3<R>& n, V3<R>& d) {
  R s, t, dist;
  edge_closest(x[0], x[1], x[2], x[3], R(1e-6), s, t, dist);
  const V3<R> c1 = x[0] + (x[1] - x[0]) * s, c2 = x[2] + (x[3] - x[2]) * t;
  const V3<R> nh = c1 - c2;
  if (length(nh) < R(1e-12)) {
    for (int k = 0; k < 4; ++k) dummy[k] = false;
    n = robust_pair_normal(x[0], x[1], x[2], x[3]);
    d = c1 * R(0.5) + c2 * R(0.5);
    return;
  }
  n = normalize(nh);
  const R de0 = rmax(rmax(-dot(n, dx[0]), -dot(n, dx[1])), R(0));
  const R de1 = rmax(rmax(dot(n, dx[2]), dot(n, dx[3])), R(0));
  if (de0 + de1 == R(0)) {
    d = c2 + R(0.5) * nh;
  } else {
    const R l = rclamp(de1 / (de1 + de0), R(0.05), R(0.95));
    d = c2 + l * nh;
  }
  for (int k = 0; k < 2; ++k) dummy[k] = de0 == R(0) ? true : !seg_plane(x[k], dx[k], n, d, R(1e-6), R(-1e-8), R(1e-6));
  for (int k = 2; k < 4; ++k) dummy[k] = de1 == R(0) ? true : !seg_plane(x[k], dx[k], n, d, R(1e-6), R(-1e-8), R(1e-6));
}

// particle_vbd_kernels.py:2724-2741
template <typename R>
R plane_t(V3<R> v, V3<R> dv, V3<R> n, V3<R> d, R eps, R gamma, R gamma_min = R(1e-3)) {
  const R den = dot(n, dv);
  if (std::fabs(den) < eps) return R(1);
  const R t = dot(n, d - v) / den;
  if (t < R(0)) return R(1);
  return rclamp(rmin(t * gamma, t - gamma_min), R(0), R(1));
}

struct SelfContact {
  double radius, margin, relaxation, edge_parallel_epsilon, rest_exclusion;
  int vertex_buffer, edge_buffer, interval;
  const double* rest_q;  // model.particle_q (rest-shape distance filter)
  const int *vt_filter_offsets, *vt_filter;  // sorted CSR per vertex, or null
  const int *ee_filter_offsets, *ee_filter;  // sorted CSR per edge, or null
  int brute_force;  // 1: test every primitive; 0: only those a uniform grid of boxes returns (same result)
};

// Candidate lists for box queries: every primitive whose box overlaps the query box, in increasing id
// (the candidates of a brute-force scan that survive its box test). Cell size >= the largest box, so
// a box covers at most 2 cells per axis.
template <typename R>
struct BoxGrid {
  double inv = 0.0;
  std::vector<std::pair<long long, int>> cells;
  static long long key(long long x, long long y, long long z) {
    return ((x & 0x1FFFFF) << 42) | ((y & 0x1FFFFF) << 21) | (z & 0x1FFFFF);
  }
  long long c(R x) const { return (long long)std::floor(double(x) * inv); }
  void build(const std::vector<V3<R>>& lo, const std::vector<V3<R>>& hi, double pad) {
    double ext = 0.0;
    for (size_t i = 0; i < lo.size(); ++i)
      ext = std::max(ext, double(std::max(std::max(hi[i].x - lo[i].x, hi[i].y - lo[i].y), hi[i].z - lo[i].z)));
    double size = std::max(ext, pad) * 1.01;
    if (!(size > 1e-9) || !(size < 1e30)) size = size < 1e30 ? 1e-9 : 1e30;
    inv = 1.0 / size;
    cells.clear();
    for (size_t i = 0; i < lo.size(); ++i)
      for (long long x = c(lo[i].x); x <= c(hi[i].x); ++x)
        for (long long y = c(lo[i].y); y <= c(hi[i].y); ++y)
          for (long long z = c(lo[i].z); z <= c(hi[i].z); ++z) cells.push_back({key(x, y, z), int(i)});
    std::sort(cells.begin(), cells.end());
  }
  void query(V3<R> qlo, V3<R> qhi, std::vector<int>& out) const {
    out.clear();
    for (long long x = c(qlo.x); x <= c(qhi.x); ++x)
      for (long long y = c(qlo.y); y <= c(qhi.y); ++y)
        for (long long z = c(qlo.z); z <= c(qhi.z); ++z) {
          auto r = std::equal_range(cells.begin(), cells.end(), std::make_pair(key(x, y, z), 0),
                                    [](const std::pair<long long, int>& a, const std::pair<long long, int>& b) {
                                      return a.first < b.first;
                                    });
          for (auto it = r.first; it != r.second; ++it) out.push_back(it->second);
        }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
  }
};

inline bool in_sorted(const int* off, const int* list, int row, int key) {
  if (!off) return false;
  int lo = off[row], hi = off[row + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (list[mid] > key) hi = mid; else lo = mid + 1;
  }
  return hi > off[row] && list[hi - 1] == key;
}

// Collision buffers of TriMeshCollisionDetector (tri_mesh_collision.py:18-40): per vertex
// vertex_buffer slots of (vertex, triangle), per edge edge_buffer slots of (edge, edge), -1 when empty.
template <typename R>
struct SCBuffers {
  std::vector<int> vt, vt_count, ee, ee_count;
  std::vector<R> vt_min, ee_min;
  int flags[4] = {0, 0, 0, 0};
};

// Brute-force detection with the semantics of vertex_triangle_collision_detection_kernel and
// edge_colliding_edges_detection_kernel (geometry/kernels.py:1252-1497): a primitive pair is recorded
// when its distance is below the margin, it is not topologically adjacent or filtered, and (with a
// positive exclusion radius) its rest-shape distance is not below that radius. Slots are filled in
// increasing primitive index; the count includes pairs past the buffer (overflow flag 0 / 2).
template <typename R>
void sc_detect(const Model& M, const SelfContact& S, const std::vector<V3<R>>& pos, SCBuffers<R>& B, int nthreads) {
  const int n = M.n, T = M.T, E = M.E, vb = S.vertex_buffer, eb = S.edge_buffer;
  const R margin = R(S.margin), rmin_q = R(S.rest_exclusion), eps = R(S.edge_parallel_epsilon);
  B.vt.assign(size_t(2) * n * vb, -1);
  B.vt_count.assign(n, 0);
  B.vt_min.assign(n, margin);
  B.ee.assign(size_t(2) * E * eb, -1);
  B.ee_count.assign(E, 0);
  B.ee_min.assign(E, margin);
  for (int k = 0; k < 4; ++k) B.flags[k] = 0;
  std::vector<V3<R>> tlo(T), thi(T), elo(E), ehi(E);
  auto vmin3 = [](V3<R> a, V3<R> b) { return v3<R>(rmin(a.x, b.x), rmin(a.y, b.y), rmin(a.z, b.z)); };
  auto vmax3 = [](V3<R> a, V3<R> b) { return v3<R>(rmax(a.x, b.x), rmax(a.y, b.y), rmax(a.z, b.z)); };
  for (int t = 0; t < T; ++t) {
    const int* ti = M.tri_indices + 3 * t;
    tlo[t] = vmin3(vmin3(pos[ti[0]], pos[ti[1]]), pos[ti[2]]);
    thi[t] = vmax3(vmax3(pos[ti[0]], pos[ti[1]]), pos[ti[2]]);
  }
  for (int e = 0; e < E; ++e) {
    const int* ei = M.edge_indices + 4 * e;
    elo[e] = vmin3(pos[ei[2]], pos[ei[3]]);
    ehi[e] = vmax3(pos[ei[2]], pos[ei[3]]);
  }
  auto overlap = [](V3<R> alo, V3<R> ahi, V3<R> blo, V3<R> bhi) {
    return alo.x <= bhi.x && alo.y <= bhi.y && alo.z <= bhi.z && ahi.x >= blo.x && ahi.y >= blo.y && ahi.z >= blo.z;
  };
  int ovf_v = 0, ovf_e = 0;
  BoxGrid<R> tgrid, egrid;
  if (!S.brute_force) {
    tgrid.build(tlo, thi, 2.0 * S.margin);
    egrid.build(elo, ehi, 2.0 * S.margin);
  }
  std::vector<int> all_t(T), all_e(E);
  std::iota(all_t.begin(), all_t.end(), 0);
  std::iota(all_e.begin(), all_e.end(), 0);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 16) reduction(| : ovf_v)
  for (int v = 0; v < n; ++v) {
    const V3<R> p = pos[v];
    const V3<R> lo = v3<R>(p.x - margin, p.y - margin, p.z - margin), hi = v3<R>(p.x + margin, p.y + margin, p.z + margin);
    int cnt = 0;
    R mn = margin;
    std::vector<int> cand;
    if (!S.brute_force) tgrid.query(lo, hi, cand);
    const std::vector<int>& list = S.brute_force ? all_t : cand;
    for (int t : list) {
      if (!overlap(lo, hi, tlo[t], thi[t])) continue;
      const int* ti = M.tri_indices + 3 * t;
      if (v == ti[0] || v == ti[1] || v == ti[2]) continue;
      if (in_sorted(S.vt_filter_offsets, S.vt_filter, v, t)) continue;
      R bary[3];
      int feat;
      const R dist = length(tri_closest(pos[ti[0]], pos[ti[1]], pos[ti[2]], p, bary, feat) - p);
      if (rmin_q > R(0)) {
        const V3<R> rv = ld<R>(S.rest_q, v);
        const R dref = length(tri_closest(ld<R>(S.rest_q, ti[0]), ld<R>(S.rest_q, ti[1]), ld<R>(S.rest_q, ti[2]), rv,
                                          bary, feat) - rv);
        if (dref < rmin_q) continue;
      }
      if (dist < margin) {
        mn = rmin(mn, dist);
        if (cnt < vb) {
          B.vt[2 * (size_t(v) * vb + cnt)] = v;
          B.vt[2 * (size_t(v) * vb + cnt) + 1] = t;
        } else {
          ovf_v = 1;
        }
        ++cnt;
      }
    }
    B.vt_count[v] = cnt;
    B.vt_min[v] = mn;
  }
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 16) reduction(| : ovf_e)
  for (int e = 0; e < E; ++e) {
    const int* ei = M.edge_indices + 4 * e;
    const V3<R> lo = elo[e] - v3<R>(margin, margin, margin), hi = ehi[e] + v3<R>(margin, margin, margin);
    int cnt = 0;
    R mn = margin;
    std::vector<int> cand;
    if (!S.brute_force) egrid.query(lo, hi, cand);
    const std::vector<int>& list = S.brute_force ? all_e : cand;
    for (int e2 : list) {
      if (!overlap(lo, hi, elo[e2], ehi[e2])) continue;
      const int* fi = M.edge_indices + 4 * e2;
      if (ei[2] == fi[2] || ei[2] == fi[3] || ei[3] == fi[2] || ei[3] == fi[3]) continue;
      if (in_sorted(S.ee_filter_offsets, S.ee_filter, e, e2)) continue;
      R s, t, dist;
      edge_closest(pos[ei[2]], pos[ei[3]], pos[fi[2]], pos[fi[3]], eps, s, t, dist);
      if (rmin_q > R(0)) {
        R dref;
        edge_closest(ld<R>(S.rest_q, ei[2]), ld<R>(S.rest_q, ei[3]), ld<R>(S.rest_q, fi[2]), ld<R>(S.rest_q, fi[3]), eps,
                     s, t, dref);
        if (dref < rmin_q) continue;
      }
      if (dist < margin) {
        mn = rmin(mn, dist);
        if (cnt < eb) {
          B.ee[2 * (size_t(e) * eb + cnt)] = e;
          B.ee[2 * (size_t(e) * eb + cnt) + 1] = e2;
        } else {
          ovf_e = 1;
        }
        ++cnt;
      }
    }
    B.ee_count[e] = cnt;
    B.ee_min[e] = mn;
  }
  B.flags[0] = ovf_v;
  B.flags[2] = ovf_e;
}

// accumulate_self_contact_force_and_hessian (particle_vbd_kernels.py:1930-2071), in the order of its
// thread ids run one after another: thread 4p+j takes slots j, j+4, ... of edge p, then of vertex p.
template <typename R>
void sc_accumulate(const Model& M, const SelfContact& S, const SCBuffers<R>& B, int color, const std::vector<V3<R>>& pos,
                   const std::vector<V3<R>>& q_prev, R dt, std::vector<V3<R>>& forces, std::vector<M3<R>>& hess) {
  const int n = M.n, E = M.E, vb = S.vertex_buffer, eb = S.edge_buffer;
  const int P = n > E ? n : E;
  const R radius = R(S.radius), ke = R(M.soft_ke), kd = R(M.soft_kd), mu = R(M.soft_mu), eps = R(M.friction_epsilon);
  const R ee_eps = R(S.edge_parallel_epsilon);
  const int* col = M.particle_colors;
  for (int p = 0; p < P; ++p)
    for (int j = 0; j < 4; ++j) {
      if (p < E)
        for (int k = j; k < eb; k += 4) {
          const int e2 = B.ee[2 * (size_t(p) * eb + k) + 1];
          if (e2 == -1) continue;
          const int* ei = M.edge_indices + 4 * p;
          const int* fi = M.edge_indices + 4 * e2;
          if (col[ei[2]] != color && col[ei[3]] != color) continue;
          const int ids[4] = {ei[2], ei[3], fi[2], fi[3]};
          V3<R> x[4], xa[4], f[2];
          M3<R> H[2];
          for (int m = 0; m < 4; ++m) x[m] = pos[ids[m]], xa[m] = q_prev[ids[m]];
          if (sc_ee(x, xa, radius, ke, kd, mu, eps, dt, ee_eps, f, H))
            for (int m = 0; m < 2; ++m)
              if (col[ids[m]] == color) {
                forces[ids[m]] = forces[ids[m]] + f[m];
                hess[ids[m]] = hess[ids[m]] + H[m];
              }
        }
      if (p < n)
        for (int k = j; k < vb; k += 4) {
          const int t = B.vt[2 * (size_t(p) * vb + k) + 1];
          if (t == -1) continue;
          const int* ti = M.tri_indices + 3 * t;
          const int ids[4] = {ti[0], ti[1], ti[2], p};
          if (col[p] != color && col[ti[0]] != color && col[ti[1]] != color && col[ti[2]] != color) continue;
          V3<R> x[4], xa[4], f[4];
          M3<R> H[4];
          for (int m = 0; m < 4; ++m) x[m] = pos[ids[m]], xa[m] = q_prev[ids[m]];
          if (sc_vt(x, xa, radius, ke, kd, mu, eps, dt, f, H)) {
            const int order[4] = {3, 0, 1, 2};  // particle first, then a, b, c, as the reference adds them
            for (int m : order)
              if (col[ids[m]] == color) {
                forces[ids[m]] = forces[ids[m]] + f[m];
                hess[ids[m]] = hess[ids[m]] + H[m];
              }
          }
        }
    }
}

// apply_planar_truncation_parallel_by_collision (particle_vbd_kernels.py:2744-2874): per-vertex minimum of
// the division-plane step fractions over all recorded pairs. pos = positions at the last detection.
template <typename R>
void sc_truncation_ts(const Model& M, const SelfContact& S, const SCBuffers<R>& B, const std::vector<V3<R>>& pos,
                      const std::vector<V3<R>>& disp, std::vector<R>& ts) {
  const int n = M.n, E = M.E, vb = S.vertex_buffer, eb = S.edge_buffer;
  const R eps = R(S.edge_parallel_epsilon), gamma = R(S.relaxation);
  for (int i = 0; i < n; ++i) ts[i] = R(1);
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < eb; ++k) {
      const int e2 = B.ee[2 * (size_t(e) * eb + k) + 1];
      if (e2 == -1) continue;
      const int* ei = M.edge_indices + 4 * e;
      const int* fi = M.edge_indices + 4 * e2;
      const int ids[4] = {ei[2], ei[3], fi[2], fi[3]};
      V3<R> x[4], dx[4], nn, d;
      bool dummy[4];
      for (int m = 0; m < 4; ++m) x[m] = pos[ids[m]], dx[m] = disp[ids[m]];
      ee_plane(x, dx, dummy, nn, d);
      for (int m = 0; m < 4; ++m)
        if (!dummy[m]) ts[ids[m]] = rmin(ts[ids[m]], plane_t(x[m], dx[m], nn, d, eps, gamma));
    }
  for (int v = 0; v < n; ++v)
    for (int k = 0; k < vb; ++k) {
      const int t = B.vt[2 * (size_t(v) * vb + k) + 1];
      if (t == -1) continue;
      const int* ti = M.tri_indices + 3 * t;
      const int ids[4] = {v, ti[0], ti[1], ti[2]};
      V3<R> x[4], dx[4], nn, d;
      bool dummy[4];
      for (int m = 0; m < 4; ++m) x[m] = pos[ids[m]], dx[m] = disp[ids[m]];
      vt_plane(x, dx, dummy, nn, d);
      for (int m = 0; m < 4; ++m)
        if (!dummy[m]) ts[ids[m]] = rmin(ts[ids[m]], plane_t(x[m], dx[m], nn, d, eps, gamma));
    }
}

// One SolverVBD.step without rigid bodies (static shapes only); S != nullptr turns particle
// self-contact on (solver_vbd.py:1669-1766, 2151-2337, 2834-2850).
template <typename R>
int step(const Model& M, double* q_in, const double* qd_in, const double* f_ext, const Contacts& Cn, R dt,
         int iterations, double* q_out, double* qd_out, int nthreads, const SelfContact* S = nullptr) {
  const int n = M.n;
  std::vector<V3<R>> pos(n), q_prev(n), inertia(n), disp(n), pos_cd(n), forces(n);
  std::vector<M3<R>> hess(n);
  for (int i = 0; i < n; ++i) pos[i] = ld<R>(q_in, i);
  const int cmax = Cn.max;
  const int ccount = Cn.count < cmax ? Cn.count : cmax;
  std::vector<R> pen_k(ccount), mat_kd(ccount), mat_mu(ccount), mat_ke(ccount);
  // init_body_particle_contacts (rigid_vbd_kernels.py:2318-2361), k_start = -1 when beta == 0
  const R k_start = M.beta == 0.0 ? R(-1) : R(1.0e2);
  for (int c = 0; c < ccount; ++c) {
    int s = Cn.shape[c];
    R ake = R(0.5) * (R(M.soft_ke) + R(M.shape_ke[s]));
    R akd = R(0.5) * (R(M.soft_kd) + R(M.shape_kd[s]));
    R amu = std::sqrt(R(M.soft_mu) * R(M.shape_mu[s]));
    mat_ke[c] = ake;
    mat_kd[c] = akd;
    mat_mu[c] = amu;
    pen_k[c] = k_start < R(0) ? ake : rmin(k_start, ake);
  }
  // _initialize_particles: pos_prev_collision_detection = q, displacements = 0 (after a collision
  // detection with self-contact on), forward_step
  SCBuffers<R> B;
  std::vector<R> ts(n, R(1));
  if (S) sc_detect(M, *S, pos, B, nthreads);
  const V3<R> g = ld<R>(M.gravity, 0);
  for (int i = 0; i < n; ++i) {
    pos_cd[i] = pos[i];
    q_prev[i] = pos[i];
    if (!(M.flags[i] & 1) || M.inv_mass[i] == 0.0) {
      inertia[i] = q_prev[i];
      disp[i] = v3<R>(0, 0, 0);
      continue;
    }
    V3<R> vel = ld<R>(qd_in, i) + (g + ld<R>(f_ext, i) * R(M.inv_mass[i])) * dt;
    inertia[i] = pos[i] + vel * dt;
    disp[i] = vel * dt;
  }
  // apply_truncation_ts: without self-contact t = 1, max_displacement = inf: pos = pos_cd + disp; with
  // it, t from the division planes of all recorded pairs and |disp| <= margin * relaxation / 2
  auto truncate = [&]() {
    if (!S) {
      for (int i = 0; i < n; ++i) pos[i] = pos_cd[i] + disp[i];
      return;
    }
    sc_truncation_ts(M, *S, B, pos_cd, disp, ts);
    const R max_d = R(S->margin) * R(S->relaxation) * R(0.5);
    for (int i = 0; i < n; ++i) {
      V3<R> d = disp[i] * ts[i];
      const R len = length(d);
      if (len > max_d) d = d * max_d / len;
      disp[i] = d;
      pos[i] = pos_cd[i] + d;
    }
  };
  truncate();
  const R dt2r = R(1) / (dt * dt);
  const R beta = R(M.beta);
  for (int it = 0; it < iterations; ++it) {
    // update_duals_body_particle_contacts (rigid_vbd_kernels.py:3755-3799)
    for (int c = 0; c < ccount; ++c) {
      int p = Cn.particle[c];
      V3<R> bx = contact_point<R>(Cn, c), nn = ld<R>(Cn.normal, c);
      R pen = -(dot(nn, pos[p] - bx) - R(M.radius[p]));
      pen = rmax(R(0), pen);
      pen_k[c] = rmin(pen_k[c] + beta * pen, mat_ke[c]);
    }
    if (S && ((S->interval == 0 && it == 0) || (S->interval >= 1 && it % S->interval == 0))) {
      // _collision_detection_penetration_free (solver_vbd.py:2834-2850)
      for (int i = 0; i < n; ++i) {
        pos_cd[i] = pos[i];
        disp[i] = v3<R>(0, 0, 0);
      }
      sc_detect(M, *S, pos, B, nthreads);
    }
    for (int i = 0; i < n; ++i) {
      forces[i] = v3<R>(0, 0, 0);
      hess[i] = mzero<R>();
    }
    for (int color = 0; color < M.C; ++color) {
      // accumulate_particle_body_contact_force_and_hessian (particle_vbd_kernels.py:2900-2967)
      for (int c = 0; c < ccount; ++c) {
        int p = Cn.particle[c];
        if (M.particle_colors[p] != color) continue;
        V3<R> bx = contact_point<R>(Cn, c), nn = ld<R>(Cn.normal, c);
        R pen = -(dot(nn, pos[p] - bx) - R(M.radius[p]));
        if (pen > R(0)) {
          V3<R> dx = pos[p] - q_prev[p];
          V3<R> bv = contact_velocity<R>(Cn, c, bx, dt);
          V3<R> rel = dx - bv * dt;
          V3<R> f;
          M3<R> H;
          contact_force(pen, nn, rel, pen_k[c], mat_kd[c], mat_mu[c], R(M.friction_epsilon), dt, f, H);
          forces[p] = forces[p] + f;
          hess[p] = hess[p] + H;
        }
      }
      // accumulate_spring_force_and_hessian (particle_vbd_kernels.py:2346-2397), in spring order
      for (int sp = 0; sp < M.spring_count; ++sp) {
        const int a = M.spring_indices[2 * sp], b = M.spring_indices[2 * sp + 1];
        if (M.particle_colors[a] != color && M.particle_colors[b] != color) continue;
        V3<R> f0, f1;
        M3<R> Hs;
        spring_both(pos[a], pos[b], q_prev[a], q_prev[b], R(M.spring_rest_length[sp]), R(M.spring_stiffness[sp]),
                    R(M.spring_damping[sp]), dt, f0, f1, Hs);
        if (M.particle_colors[a] == color) {
          forces[a] = forces[a] + f0;
          hess[a] = hess[a] + Hs;
        }
        if (M.particle_colors[b] == color) {
          forces[b] = forces[b] + f1;
          hess[b] = hess[b] + Hs;
        }
      }
      if (S) sc_accumulate(M, *S, B, color, pos, q_prev, dt, forces, hess);
      // solve_elasticity (particle_vbd_kernels.py:3135-3273)
      const int c0 = M.color_offsets[color], c1 = M.color_offsets[color + 1];
#pragma omp parallel for num_threads(nthreads) schedule(static)
      for (int k = c0; k < c1; ++k) {
        const int v = M.color_particles[k];
        if (!(M.flags[v] & 1) || M.mass[v] == 0.0) {
          disp[v] = v3<R>(0, 0, 0);
          continue;
        }
        R m = R(M.mass[v]);
        V3<R> f = m * (inertia[v] - pos[v]) * dt2r;
        M3<R> h = (m * dt2r) * ident<R>();
        for (int a = M.adj_face_offsets[v]; a < M.adj_face_offsets[v + 1]; a += 2) {
          int t = M.adj_faces[a], o = M.adj_faces[a + 1];
          const double* mat = M.tri_materials + 5 * t;
          if (mat[0] > 0.0 || mat[1] > 0.0) {
            const int* ti = M.tri_indices + 3 * t;
            R pose[4] = {R(M.tri_poses[4 * t]), R(M.tri_poses[4 * t + 1]), R(M.tri_poses[4 * t + 2]),
                         R(M.tri_poses[4 * t + 3])};
            V3<R> ft;
            M3<R> ht;
            membrane<R>(o, pos[ti[0]], pos[ti[1]], pos[ti[2]], q_prev[ti[0]], q_prev[ti[1]], q_prev[ti[2]], pose,
                        R(M.tri_areas[t]), R(mat[0]), R(mat[1]), R(mat[2]), dt, ft, ht);
            f = f + ft;
            h = h + ht;
          }
        }
        for (int a = M.adj_edge_offsets[v]; a < M.adj_edge_offsets[v + 1]; a += 2) {
          int e = M.adj_edges[a], o = M.adj_edges[a + 1];
          const double* bp = M.edge_bending_properties + 2 * e;
          if (bp[0] > 0.0) {
            const int* ei = M.edge_indices + 4 * e;
            bool boundary = ei[0] == -1 || ei[1] == -1;
            V3<R> xs[4], xps[4];
            for (int j = 0; j < 4; ++j) {
              int idx = ei[j] < 0 ? 0 : ei[j];
              xs[j] = pos[idx];
              xps[j] = q_prev[idx];
            }
            V3<R> fe;
            M3<R> he;
            bending<R>(o, xs, xps, boundary, R(M.edge_rest_angle[e]), R(M.edge_rest_length[e]), R(bp[0]), R(bp[1]), dt,
                       fe, he);
            f = f + fe;
            h = h + he;
          }
        }
        if (M.tet_count)
          for (int a = M.adj_tet_offsets[v]; a < M.adj_tet_offsets[v + 1]; a += 2) {
            const int t = M.adj_tets[a], o = M.adj_tets[a + 1];
            const double* tm = M.tet_materials + 3 * t;
            if (!(tm[0] > 0.0 || tm[1] > 0.0)) continue;
            const int* ti = M.tet_indices + 4 * t;
            V3<R> xs[4], xps[4];
            for (int j = 0; j < 4; ++j) xs[j] = pos[ti[j]], xps[j] = q_prev[ti[j]];
            R Dinv[9];
            for (int j = 0; j < 9; ++j) Dinv[j] = R(M.tet_poses[9 * t + j]);
            V3<R> ft;
            M3<R> ht;
            tet_force<R>(o, xs, xps, Dinv, R(tm[0]), R(tm[1]), R(tm[2]), dt, ft, ht);
            f = f + ft;
            h = h + ht;
          }
        h = h + hess[v];
        f = f + forces[v];
        R d = det(h);
        if (std::fabs(d) > R(1e-8)) disp[v] = disp[v] + inverse(h, d) * f;
      }
      truncate();
    }
  }
  for (int i = 0; i < n; ++i) {
    V3<R> v = (pos[i] - q_prev[i]) / dt;
    q_in[3 * i] = pos[i].x;
    q_in[3 * i + 1] = pos[i].y;
    q_in[3 * i + 2] = pos[i].z;
    q_out[3 * i] = pos[i].x;
    q_out[3 * i + 1] = pos[i].y;
    q_out[3 * i + 2] = pos[i].z;
    qd_out[3 * i] = v.x;
    qd_out[3 * i + 1] = v.y;
    qd_out[3 * i + 2] = v.z;
  }
  return 0;
}

}  // namespace

// ------------------------------------------------------------------------------------ particle-shape contacts
// create_soft_contacts (geometry/kernels.py:1001-1140) for static shapes of the analytic types, with the SDFs
// and gradients of geometry/kernels.py:132-600 (capsule and cylinder along the shape's local Z, straight
// cylinders): the particle in the shape frame, d and n from the shape's SDF, and for d < margin + radius the
// contact point x_local - n d and the normal mapped back to world. Contacts in particle-major order.
namespace sdf {
using D3 = V3<double>;
enum { PLANE = 1, HFIELD = 2, SPHERE = 3, CAPSULE = 4, ELLIPSOID = 5, CYLINDER = 6, BOX = 7, MESH = 8, CONE = 9, CONVEX_MESH = 10 };
inline double sgn(double x) { return x < 0.0 ? -1.0 : 1.0; }  // wp.sign: -1 below zero, 1 otherwise
inline D3 qrot(const double* q, D3 v) {  // q = (x, y, z, w)
  const D3 u = v3(q[0], q[1], q[2]);
  const double w = q[3];
  return v * (2.0 * w * w - 1.0) + cross(u, v) * (2.0 * w) + u * (2.0 * dot(u, v));
}
inline D3 normalize0(D3 a) {  // wp.normalize: the zero vector stays zero
  const double l = length(a);
  return l > 0.0 ? a / l : a;
}
// geometry/kernels.py:165-195
inline double sphere(D3 p, double r) { return length(p) - r; }
inline D3 sphere_grad(D3 p) {
  const double l = length(p);
  return l > 1.0e-8 ? p / l : v3(0.0, 0.0, 1.0);
}
// :198-259
inline double box(D3 p, double hx, double hy, double hz) {
  const double qx = std::fabs(p.x) - hx, qy = std::fabs(p.y) - hy, qz = std::fabs(p.z) - hz;
  const D3 e = v3(std::max(qx, 0.0), std::max(qy, 0.0), std::max(qz, 0.0));
  return length(e) + std::min(std::max(qx, std::max(qy, qz)), 0.0);
}
inline D3 box_grad(D3 p, double hx, double hy, double hz) {
  const double qx = std::fabs(p.x) - hx, qy = std::fabs(p.y) - hy, qz = std::fabs(p.z) - hz;
  if (qx > 0.0 || qy > 0.0 || qz > 0.0) {
    const D3 c = v3(std::min(std::max(p.x, -hx), hx), std::min(std::max(p.y, -hy), hy), std::min(std::max(p.z, -hz), hz));
    return normalize0(p - c);
  }
  if ((qx > qy && qx > qz) || (qy == 0.0 && qz == 0.0)) return v3(sgn(p.x), 0.0, 0.0);
  if ((qy > qx && qy > qz) || (qx == 0.0 && qz == 0.0)) return v3(0.0, sgn(p.y), 0.0);
  return v3(0.0, 0.0, sgn(p.z));
}
// :262-329 (up axis Z)
inline double capsule(D3 p, double r, double hh) {
  if (p.z > hh) return length(v3(p.x, p.y, p.z - hh)) - r;
  if (p.z < -hh) return length(v3(p.x, p.y, p.z + hh)) - r;
  return length(v3(p.x, p.y, 0.0)) - r;
}
inline D3 capsule_grad(D3 p, double hh) {
  D3 v = v3(p.x, p.y, 0.0), g = v3(0.0, 0.0, 1.0);
  if (p.z > hh) {
    v = v3(p.x, p.y, p.z - hh);
  } else if (p.z < -hh) {
    v = v3(p.x, p.y, p.z + hh);
    g = v3(0.0, 0.0, -1.0);
  }
  const double l = length(v);
  return l > 1.0e-8 ? v / l : g;
}
// :332-446 (straight cylinder, up axis Z)
inline double cylinder(D3 p, double r, double hh) {
  const double dx = length(v3(p.x, p.y, 0.0)) - r, dy = std::fabs(p.z) - hh;
  const double ex = std::max(dx, 0.0), ey = std::max(dy, 0.0);
  return std::min(std::max(dx, dy), 0.0) + std::sqrt(ex * ex + ey * ey);
}
inline D3 cylinder_grad(D3 p, double r, double hh) {
  const D3 v = v3(p.x, p.y, 0.0);
  const double vl = length(v);
  const D3 radial = vl > 1.0e-8 ? v / vl : v3(0.0, 0.0, 1.0);
  const D3 axial = v3(0.0, 0.0, sgn(p.z));
  const double dx = vl - r, dy = std::fabs(p.z) - hh;
  if (dx > 0.0 && dy > 0.0) {
    const D3 g = radial * dx + axial * dy;
    const double gl = length(g);
    return gl > 1.0e-8 ? g / gl : radial;
  }
  return dx > dy ? radial : axial;
}
// :449-512
inline void ellipsoid(D3 p, D3 radii, double& d, D3& n) {
  const D3 r = v3(std::max(std::fabs(radii.x), 1.0e-8), std::max(std::fabs(radii.y), 1.0e-8),
                  std::max(std::fabs(radii.z), 1.0e-8));
  const D3 ir = v3(1.0 / r.x, 1.0 / r.y, 1.0 / r.z);
  const D3 q0 = v3(p.x * ir.x, p.y * ir.y, p.z * ir.z);
  const D3 q1 = v3(p.x * ir.x * ir.x, p.y * ir.y * ir.y, p.z * ir.z * ir.z);
  const double k0 = length(q0), k1 = length(q1);
  d = k1 > 1.0e-8 ? k0 * (k0 - 1.0) / k1 : -std::min(std::min(r.x, r.y), r.z);
  n = v3(0.0, 0.0, 1.0);
  if (!(k1 < 1.0e-8)) {
    const D3 g = q1 * (k0 / k1);
    const double gl = length(g);
    if (gl > 1.0e-8) n = g / gl;
  }
}
// :141-161 (capped cone with top radius 0) and :515-564: base radius r at z = -hh, apex at z = +hh
inline double cone(D3 p, double r, double hh) {
  const double qx = std::sqrt(p.x * p.x + p.y * p.y), qy = p.z;
  const double k2x = -r, k2y = 2.0 * hh;  // (top radius - bottom radius, 2 hh)
  const double cax = qx - std::min(qx, qy < 0.0 ? r : 0.0), cay = std::fabs(qy) - hh;
  const double den = k2x * k2x + k2y * k2y;
  const double t = den > 0.0 ? std::min(std::max(((0.0 - qx) * k2x + (hh - qy) * k2y) / den, 0.0), 1.0) : 0.0;
  const double cbx = qx + k2x * t, cby = qy - hh + k2y * t;
  const double sg = (cbx < 0.0 && cay < 0.0) ? -1.0 : 1.0;
  return sg * std::sqrt(std::min(cax * cax + cay * cay, cbx * cbx + cby * cby));
}
inline D3 cone_grad(D3 p, double r, double hh) {
  if (hh <= 0.0) return v3(0.0, 0.0, sgn(p.z));
  const double rr = length(v3(p.x, p.y, 0.0));
  const double dx = rr - r * (hh - p.z) / (2.0 * hh), dy = std::fabs(p.z) - hh;
  if (dx > dy) return rr > 0.0 ? normalize0(v3(p.x / rr, p.y / rr, r / (2.0 * hh))) : v3(0.0, 0.0, 1.0);
  return v3(0.0, 0.0, sgn(p.z));
}
// utils/heightfield.py:94-205: grid g = (data_offset, nrow, ncol), extents e = (hx, hy, min_z, max_z), normalized
// elevations; the clamped point's cell triangle (diagonal from (col, row) to (col + 1, row + 1)) gives the plane
// distance and normal, and outside the footprint the lateral gap is folded in.
inline void heightfield(const int* g, const double* e, const double* elev, D3 p, double& d, D3& n) {
  const int nrow = g[1], ncol = g[2];
  if (nrow <= 1 || ncol <= 1) {
    d = 1.0e10, n = v3(0.0, 0.0, 1.0);
    return;
  }
  const double hx = e[0], hy = e[1], zmin = e[2], zr = e[3] - e[2];
  const double dx = 2.0 * hx / double(ncol - 1), dy = 2.0 * hy / double(nrow - 1);
  const double cx = std::min(std::max(p.x, -hx), hx), cy = std::min(std::max(p.y, -hy), hy);
  const double ox = p.x - cx, oy = p.y - cy, lat = ox * ox + oy * oy;
  const double colf = std::min(std::max((cx + hx) / dx, 0.0), double(ncol - 1));
  const double rowf = std::min(std::max((cy + hy) / dy, 0.0), double(nrow - 1));
  const int col = std::min(int(colf), ncol - 2), row = std::min(int(rowf), nrow - 2);
  const double fx = colf - col, fy = rowf - row;
  const double* z = elev + g[0] + long(row) * ncol + col;
  const double h00 = zmin + z[0] * zr, h10 = zmin + z[1] * zr, h01 = zmin + z[ncol] * zr, h11 = zmin + z[ncol + 1] * zr;
  const D3 v0 = v3(-hx + col * dx, -hy + row * dy, h00);
  const D3 e1 = fx >= fy ? v3(dx, 0.0, h10 - h00) : v3(dx, dy, h11 - h00);
  const D3 e2 = fx >= fy ? v3(dx, dy, h11 - h00) : v3(0.0, dy, h01 - h00);
  const D3 nrm = normalize0(cross(e1, e2));
  const double dp = dot(p - v0, nrm);
  if (lat > 0.0) {
    d = std::sqrt(lat + dp * dp);
    const D3 raw = v3(ox, oy, 0.0) + nrm * dp;
    n = dot(raw, raw) > 1.0e-20 ? normalize0(raw) : v3(0.0, 0.0, 1.0);
  } else {
    d = dp, n = nrm;
  }
}
// Triangle meshes (geometry/kernels.py:1091-1113 through wp.mesh_query_point_sign_normal, which is Warp-native):
// the closest point over all triangles (brute force; ties keep the lowest triangle) closer than max_dist, and the
// sign from the angle-weighted pseudo-normal of its feature (Baerentzen and Aanaes, IEEE TVCG 11(3), 2005): the
// face normal inside a triangle, the sum of the faces' unit normals on an edge, the angle-weighted sum at a vertex.
struct MeshQ {
  int V, T;
  const double* pts;
  const int* tri;
};
inline D3 mpt(const MeshQ& m, int v) { return v3(m.pts[3 * v], m.pts[3 * v + 1], m.pts[3 * v + 2]); }
inline D3 face_normal(const MeshQ& m, int t) {
  const D3 a = mpt(m, m.tri[3 * t]), b = mpt(m, m.tri[3 * t + 1]), c = mpt(m, m.tri[3 * t + 2]);
  return normalize0(cross(b - a, c - a));
}
inline bool mesh_query(const MeshQ& m, D3 p, double max_dist, D3& cp, double& sign) {
  double best = max_dist * max_dist;
  int bt = -1, feat = 6;
  for (int t = 0; t < m.T; ++t) {
    double w[3];
    int f;
    const D3 c = tri_closest(mpt(m, m.tri[3 * t]), mpt(m, m.tri[3 * t + 1]), mpt(m, m.tri[3 * t + 2]), p, w, f);
    const double d2 = dot(c - p, c - p);
    if (d2 < best) best = d2, bt = t, feat = f, cp = c;
  }
  if (bt < 0) return false;
  D3 pn = v3(0.0, 0.0, 0.0);
  const int* tv = m.tri + 3 * bt;
  if (feat == 6) {
    pn = face_normal(m, bt);
  } else if (feat >= 3) {  // edge AB, AC or BC: every face holding both ends
    const int e0 = feat == 5 ? tv[1] : tv[0], e1 = feat == 3 ? tv[1] : tv[2];
    for (int t = 0; t < m.T; ++t) {
      const int* u = m.tri + 3 * t;
      const bool h0 = u[0] == e0 || u[1] == e0 || u[2] == e0, h1 = u[0] == e1 || u[1] == e1 || u[2] == e1;
      if (h0 && h1) pn = pn + face_normal(m, t);
    }
  } else {  // vertex: incident faces weighted by their angle there
    const int v = tv[feat];
    for (int t = 0; t < m.T; ++t) {
      const int* u = m.tri + 3 * t;
      for (int k = 0; k < 3; ++k)
        if (u[k] == v) {
          const D3 x = mpt(m, u[k]), e1 = mpt(m, u[(k + 1) % 3]) - x, e2 = mpt(m, u[(k + 2) % 3]) - x;
          pn = pn + face_normal(m, t) * std::atan2(length(cross(e1, e2)), dot(e1, e2));
        }
    }
  }
  sign = dot(p - cp, pn) < 0.0 ? -1.0 : 1.0;
  return true;
}
// :568-589
inline double plane(D3 p, double w, double l) {
  if (w > 0.0 && l > 0.0) return std::max(std::max(std::fabs(p.x) - w, std::fabs(p.y) - l), std::fabs(p.z));
  return p.z;
}
}  // namespace sdf

extern "C" {

struct OracleModel {
  int n, T, E, C, S;
  const double *mass, *inv_mass, *radius;
  const int* flags;
  const int* tri_indices;
  const double *tri_poses, *tri_materials, *tri_areas;
  const int* edge_indices;
  const double *edge_rest_angle, *edge_rest_length, *edge_bending_properties;
  const int *adj_face_offsets, *adj_faces, *adj_edge_offsets, *adj_edges;
  const int *color_offsets, *color_particles, *particle_colors;
  const double* gravity;
  double soft_ke, soft_kd, soft_mu;
  const double *shape_ke, *shape_kd, *shape_mu;
  double friction_epsilon, beta;
  int spring_count;
  const int* spring_indices;
  const double *spring_rest_length, *spring_stiffness, *spring_damping;
  int tet_count;
  const int* tet_indices;
  const double *tet_poses, *tet_materials;
  const int *adj_tet_offsets, *adj_tets;
};

struct OracleContacts {
  int count, max;
  const int *particle, *shape;
  const double *body_pos, *body_vel, *normal;
  const int* shape_body;
  const double *body_q, *body_q_prev, *body_qd, *body_com;
};
static_assert(sizeof(OracleContacts) == sizeof(Contacts), "layout");

static_assert(sizeof(OracleModel) == sizeof(Model), "layout");

// precision: 64 = all-FP64 run, 32 = FP32 run (inputs rounded to float).
int oracle_vbd_step(const OracleModel* m, double* q_in, const double* qd_in, const double* f_ext,
                    const OracleContacts* c, double dt, int iterations, double* q_out, double* qd_out, int precision,
                    int nthreads) {
  Model M;
  std::memcpy(&M, m, sizeof(M));
  Contacts C;
  std::memcpy(&C, c, sizeof(C));
  if (nthreads < 1) nthreads = 1;
  if (precision == 64) return step<double>(M, q_in, qd_in, f_ext, C, dt, iterations, q_out, qd_out, nthreads);
  if (precision == 32)
    return step<float>(M, q_in, qd_in, f_ext, C, float(dt), iterations, q_out, qd_out, nthreads);
  return -1;
}

struct OracleSelfContact {
  double radius, margin, relaxation, edge_parallel_epsilon, rest_exclusion;
  int vertex_buffer, edge_buffer, interval;
  const double* rest_q;
  const int *vt_filter_offsets, *vt_filter, *ee_filter_offsets, *ee_filter;
  int brute_force;
};
static_assert(sizeof(OracleSelfContact) == sizeof(SelfContact), "layout");

// oracle_vbd_step with particle self-contact on.
int oracle_vbd_step_sc(const OracleModel* m, double* q_in, const double* qd_in, const double* f_ext,
                       const OracleContacts* c, const OracleSelfContact* sc, double dt, int iterations, double* q_out,
                       double* qd_out, int precision, int nthreads) {
  Model M;
  std::memcpy(&M, m, sizeof(M));
  SelfContact S;
  std::memcpy(&S, sc, sizeof(S));
  Contacts C;
  std::memcpy(&C, c, sizeof(C));
  if (nthreads < 1) nthreads = 1;
  if (precision == 64) return step<double>(M, q_in, qd_in, f_ext, C, dt, iterations, q_out, qd_out, nthreads, &S);
  if (precision == 32)
    return step<float>(M, q_in, qd_in, f_ext, C, float(dt), iterations, q_out, qd_out, nthreads, &S);
  return -1;
}

// One collision detection at positions q (n x 3). Outputs as TriMeshCollisionInfo: vt[2*n*vb],
// vt_count[n], vt_min[n], ee[2*E*eb], ee_count[E], ee_min[E], flags[4].
int oracle_collide(const OracleModel* m, const OracleSelfContact* sc, const double* q, int precision, int* vt,
                   int* vt_count, double* vt_min, int* ee, int* ee_count, double* ee_min, int* flags, int nthreads) {
  Model M;
  std::memcpy(&M, m, sizeof(M));
  SelfContact S;
  std::memcpy(&S, sc, sizeof(S));
  auto run = [&](auto tag) {
    using R = decltype(tag);
    std::vector<V3<R>> pos(M.n);
    for (int i = 0; i < M.n; ++i) pos[i] = ld<R>(q, i);
    SCBuffers<R> B;
    sc_detect(M, S, pos, B, nthreads < 1 ? 1 : nthreads);
    std::copy(B.vt.begin(), B.vt.end(), vt);
    std::copy(B.vt_count.begin(), B.vt_count.end(), vt_count);
    for (int i = 0; i < M.n; ++i) vt_min[i] = double(B.vt_min[i]);
    std::copy(B.ee.begin(), B.ee.end(), ee);
    std::copy(B.ee_count.begin(), B.ee_count.end(), ee_count);
    for (int i = 0; i < M.E; ++i) ee_min[i] = double(B.ee_min[i]);
    for (int k = 0; k < 4; ++k) flags[k] = B.flags[k];
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return 0;
}

// Self-contact pair terms. x/xa: 4 points (12 doubles). Vertex-triangle: x = (a, b, c, p), out = 4 forces
// then 4 Hessians (48). Edge-edge: x = (e1.v0, e1.v1, e2.v0, e2.v1), out = 2 forces, 2 Hessians (24).
// Return 1 when the pair is in contact.
int oracle_sc_vt(int precision, const double* x, const double* xa, double radius, double ke, double kd, double mu,
                 double eps, double dt, double* out) {
  int hit = 0;
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> X[4], XA[4], f[4];
    M3<R> H[4];
    for (int k = 0; k < 4; ++k) X[k] = ld<R>(x, k), XA[k] = ld<R>(xa, k);
    hit = sc_vt(X, XA, R(radius), R(ke), R(kd), R(mu), R(eps), R(dt), f, H);
    for (int k = 0; k < 4; ++k) {
      out[3 * k] = hit ? f[k].x : 0.0, out[3 * k + 1] = hit ? f[k].y : 0.0, out[3 * k + 2] = hit ? f[k].z : 0.0;
      for (int i = 0; i < 9; ++i) out[12 + 9 * k + i] = hit ? double(H[k].m[i / 3][i % 3]) : 0.0;
    }
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return hit;
}

int oracle_sc_ee(int precision, const double* x, const double* xa, double radius, double ke, double kd, double mu,
                 double eps, double dt, double ee_eps, double* out) {
  int hit = 0;
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> X[4], XA[4], f[2];
    M3<R> H[2];
    for (int k = 0; k < 4; ++k) X[k] = ld<R>(x, k), XA[k] = ld<R>(xa, k);
    hit = sc_ee(X, XA, R(radius), R(ke), R(kd), R(mu), R(eps), R(dt), R(ee_eps), f, H);
    for (int k = 0; k < 2; ++k) {
      out[3 * k] = hit ? f[k].x : 0.0, out[3 * k + 1] = hit ? f[k].y : 0.0, out[3 * k + 2] = hit ? f[k].z : 0.0;
      for (int i = 0; i < 9; ++i) out[6 + 9 * k + i] = hit ? double(H[k].m[i / 3][i % 3]) : 0.0;
    }
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return hit;
}

// Division plane of a pair and the step fractions of its four vertices. kind 0: vertex-triangle,
// x = (v, t1, t2, t3); kind 1: edge-edge. out = dummy[4], n[3], d[3], t[4] (14 doubles).
int oracle_sc_plane(int precision, int kind, const double* x, const double* dx, double eps, double gamma, double* out) {
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> X[4], DX[4], n, d;
    bool dummy[4];
    for (int k = 0; k < 4; ++k) X[k] = ld<R>(x, k), DX[k] = ld<R>(dx, k);
    if (kind == 0)
      vt_plane(X, DX, dummy, n, d);
    else
      ee_plane(X, DX, dummy, n, d);
    for (int k = 0; k < 4; ++k) out[k] = dummy[k] ? 1.0 : 0.0;
    out[4] = n.x, out[5] = n.y, out[6] = n.z, out[7] = d.x, out[8] = d.y, out[9] = d.z;
    for (int k = 0; k < 4; ++k) out[10 + k] = plane_t(X[k], DX[k], n, d, R(eps), R(gamma));
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return 0;
}

// Closest point on a triangle: x = (a, b, c, p); out = point[3], bary[3], feature.
int oracle_tri_closest(const double* x, double* out) {
  double bary[3];
  int feat;
  V3<double> c = tri_closest(ld<double>(x, 0), ld<double>(x, 1), ld<double>(x, 2), ld<double>(x, 3), bary, feat);
  out[0] = c.x, out[1] = c.y, out[2] = c.z, out[3] = bary[0], out[4] = bary[1], out[5] = bary[2], out[6] = feat;
  return 0;
}

// Closest points of two segments: x = (p1, q1, p2, q2); out = s, t, distance.
int oracle_edge_closest(const double* x, double eps, double* out) {
  edge_closest(ld<double>(x, 0), ld<double>(x, 1), ld<double>(x, 2), ld<double>(x, 3), eps, out[0], out[1], out[2]);
  return 0;
}

// dE/dd and d2E/dd2 of the self-contact barrier.
int oracle_sc_norm(double dis, double radius, double k, double* out) {
  sc_norm(dis, radius, k, out[0], out[1]);
  return 0;
}

// Tetrahedron term for the vertex of `order`: x, xp 12 doubles, Dinv 9 (row-major); out = force 3 + Hessian 9.
int oracle_tet(int precision, int order, const double* x, const double* xp, const double* Dinv, double mu, double lmbd,
               double damping, double dt, double* out) {
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> X[4], XP[4], f;
    M3<R> h;
    R D[9];
    for (int k = 0; k < 4; ++k) X[k] = ld<R>(x, k), XP[k] = ld<R>(xp, k);
    for (int k = 0; k < 9; ++k) D[k] = R(Dinv[k]);
    tet_force<R>(order, X, XP, D, R(mu), R(lmbd), R(damping), R(dt), f, h);
    out[0] = f.x, out[1] = f.y, out[2] = f.z;
    for (int i = 0; i < 9; ++i) out[3 + i] = h.m[i / 3][i % 3];
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return 0;
}

// Spring: x, xa 6 doubles; out = f0 3, f1 3, Hessian 9.
int oracle_spring(int precision, const double* x, const double* xa, double rest, double ke, double kd, double dt,
                  double* out) {
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> f0, f1;
    M3<R> H;
    spring_both<R>(ld<R>(x, 0), ld<R>(x, 1), ld<R>(xa, 0), ld<R>(xa, 1), R(rest), R(ke), R(kd), R(dt), f0, f1, H);
    out[0] = f0.x, out[1] = f0.y, out[2] = f0.z, out[3] = f1.x, out[4] = f1.y, out[5] = f1.z;
    for (int i = 0; i < 9; ++i) out[6 + i] = H.m[i / 3][i % 3];
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return 0;
}

// Vertex -> (tet, order) adjacency in the reference's fill order (particle_vbd_kernels.py:774-825).
int oracle_build_tet_adjacency(int n, int T4, const int* tets, int* offsets /*n+1*/, int* adj /*8 T4*/) {
  std::vector<int> cnt(n, 0), fill(n, 0);
  for (int t = 0; t < T4; ++t)
    for (int j = 0; j < 4; ++j) cnt[tets[4 * t + j]]++;
  offsets[0] = 0;
  for (int i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + 2 * cnt[i];
  for (int t = 0; t < T4; ++t)
    for (int j = 0; j < 4; ++j) {
      const int v = tets[4 * t + j];
      const int o = offsets[v] + 2 * fill[v]++;
      adj[o] = t;
      adj[o + 1] = j;
    }
  return 0;
}

// Element-level entry points (force 3 + Hessian 9 written to out[12]).
int oracle_membrane(int precision, int v_order, const double* x /*9*/, const double* xp /*9*/, const double* pose,
                    double area, double mu, double lmbd, double damping, double dt, double* out) {
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> f;
    M3<R> h;
    R p[4] = {R(pose[0]), R(pose[1]), R(pose[2]), R(pose[3])};
    membrane<R>(v_order, ld<R>(x, 0), ld<R>(x, 1), ld<R>(x, 2), ld<R>(xp, 0), ld<R>(xp, 1), ld<R>(xp, 2), p, R(area),
                R(mu), R(lmbd), R(damping), R(dt), f, h);
    out[0] = f.x, out[1] = f.y, out[2] = f.z;
    for (int i = 0; i < 9; ++i) out[3 + i] = h.m[i / 3][i % 3];
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return 0;
}

int oracle_bending(int precision, int v_order, const double* x /*12*/, const double* xp /*12*/, int boundary,
                   double rest_angle, double rest_length, double ke, double kd, double dt, double* out) {
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> xs[4], xps[4];
    for (int j = 0; j < 4; ++j) xs[j] = ld<R>(x, j), xps[j] = ld<R>(xp, j);
    V3<R> f;
    M3<R> h;
    bending<R>(v_order, xs, xps, boundary != 0, R(rest_angle), R(rest_length), R(ke), R(kd), R(dt), f, h);
    out[0] = f.x, out[1] = f.y, out[2] = f.z;
    for (int i = 0; i < 9; ++i) out[3 + i] = h.m[i / 3][i % 3];
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return 0;
}

int oracle_contact(int precision, double pen, const double* n, const double* rel, double ke, double kd, double mu,
                   double fric_eps, double dt, double* out) {
  auto run = [&](auto tag) {
    using R = decltype(tag);
    V3<R> f;
    M3<R> h;
    contact_force<R>(R(pen), ld<R>(n, 0), ld<R>(rel, 0), R(ke), R(kd), R(mu), R(fric_eps), R(dt), f, h);
    out[0] = f.x, out[1] = f.y, out[2] = f.z;
    for (int i = 0; i < 9; ++i) out[3 + i] = h.m[i / 3][i % 3];
  };
  if (precision == 64)
    run(double());
  else
    run(float());
  return 0;
}

// Vertex -> (element, order) adjacency in the reference's fill order (particle_vbd_kernels.py:639-738).
// Offsets count two ints per adjacency, as in the reference. Returns 0.
int oracle_build_adjacency(int n, int T, const int* tri, int E, const int* edges, int* face_offsets /*n+1*/,
                           int* faces /*6T*/, int* edge_offsets /*n+1*/, int* edge_adj /*<=8E*/) {
  std::vector<int> cnt(n, 0), fill(n, 0);
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 3; ++j) cnt[tri[3 * t + j]]++;
  face_offsets[0] = 0;
  for (int i = 0; i < n; ++i) face_offsets[i + 1] = face_offsets[i] + 2 * cnt[i];
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 3; ++j) {
      int v = tri[3 * t + j];
      int o = face_offsets[v] + 2 * fill[v]++;
      faces[o] = t;
      faces[o + 1] = j;
    }
  std::fill(cnt.begin(), cnt.end(), 0);
  std::fill(fill.begin(), fill.end(), 0);
  for (int e = 0; e < E; ++e) {
    const int* ei = edges + 4 * e;
    cnt[ei[2]]++;
    cnt[ei[3]]++;
    if (ei[0] != -1) cnt[ei[0]]++;
    if (ei[1] != -1) cnt[ei[1]]++;
  }
  edge_offsets[0] = 0;
  for (int i = 0; i < n; ++i) edge_offsets[i + 1] = edge_offsets[i] + 2 * cnt[i];
  auto put = [&](int v, int e, int order) {
    int o = edge_offsets[v] + 2 * fill[v]++;
    edge_adj[o] = e;
    edge_adj[o + 1] = order;
  };
  for (int e = 0; e < E; ++e) {
    const int* ei = edges + 4 * e;
    put(ei[2], e, 2);
    put(ei[3], e, 3);
    if (ei[0] != -1) put(ei[0], e, 0);
    if (ei[1] != -1) put(ei[1], e, 1);
  }
  return 0;
}

// Soft contacts of active particles against static shapes (geometry/kernels.py:1001-1140), for
// shape_type 0 = infinite ground plane through shape_pos with normal +Z, 1 = sphere of radius
// shape_radius centred at shape_pos. Contacts are emitted in (particle, shape) order.
int oracle_soft_contacts(int n, const double* q, const double* radius, const int* flags, int S,
                         const int* shape_type, const double* shape_pos, const double* shape_radius, double margin,
                         int max_contacts, int* particle, int* shape, double* body_pos, double* body_vel,
                         double* normal) {
  int count = 0;
  for (int i = 0; i < n; ++i) {
    if (!(flags[i] & 1)) continue;
    for (int s = 0; s < S; ++s) {
      double xl[3] = {q[3 * i] - shape_pos[3 * s], q[3 * i + 1] - shape_pos[3 * s + 1], q[3 * i + 2] - shape_pos[3 * s + 2]};
      double d, nn[3];
      if (shape_type[s] == 0) {
        d = xl[2];
        nn[0] = 0, nn[1] = 0, nn[2] = 1;
      } else {
        double L = std::sqrt(xl[0] * xl[0] + xl[1] * xl[1] + xl[2] * xl[2]);
        d = L - shape_radius[s];
        if (L > 1e-8) {
          nn[0] = xl[0] / L, nn[1] = xl[1] / L, nn[2] = xl[2] / L;
        } else {
          nn[0] = 0, nn[1] = 0, nn[2] = 1;
        }
      }
      if (d < margin + radius[i]) {
        if (count < max_contacts) {
          particle[count] = i;
          shape[count] = s;
          for (int j = 0; j < 3; ++j) {
            body_pos[3 * count + j] = shape_pos[3 * s + j] + xl[j] - nn[j] * d;
            body_vel[3 * count + j] = 0.0;
            normal[3 * count + j] = nn[j];
          }
        }
        ++count;
      }
    }
  }
  return count;
}


// shape_xform [S,7] = (position, quaternion xyzw) in the frame of body shape_body[s] (-1: world; shape_body or
// body_q NULL: every shape static), body_q [B,7]; shape_scale [S,3]. Contact points are written in the body's
// frame, normals in world. Returns the number of contacts found, or -1 for a shape type without an analytic SDF.
// Heightfield shapes (type 2) take grid hf_index[s]: hf_grid[3k..] = (data_offset, nrow, ncol),
// hf_ext[4k..] = (hx, hy, min_z, max_z) with the shape's scale applied, over the elevations `elev`.
int oracle_soft_contacts_shapes(int n, const double* q, const double* radius, const int* flags, int S,
                                const int* shape_type, const double* shape_xform, const double* shape_scale,
                                const int* hf_index, const int* hf_grid, const double* hf_ext, const double* elev,
                                const int* mesh_index, const int* mesh_vert_off, const int* mesh_tri_off,
                                const double* mesh_pts, const int* mesh_tris, const int* shape_flags,
                                const int* shape_world, const int* particle_world, double margin, int max_contacts,
                                int* particle, int* shape, double* body_pos, double* body_vel, double* normal,
                                const int* shape_body, const double* body_q) {
  using sdf::D3;
  for (int s = 0; s < S; ++s) {
    const int t = shape_type[s];
    if (t != sdf::PLANE && t != sdf::SPHERE && t != sdf::CAPSULE && t != sdf::ELLIPSOID && t != sdf::CYLINDER &&
        t != sdf::BOX && t != sdf::CONE && t != sdf::HFIELD && t != sdf::MESH && t != sdf::CONVEX_MESH)
      return -1;
    if (t == sdf::HFIELD && (!hf_index || !hf_grid || !hf_ext || !elev)) return -1;
    if ((t == sdf::MESH || t == sdf::CONVEX_MESH) && (!mesh_index || !mesh_vert_off || !mesh_tri_off || !mesh_pts ||
                                                       !mesh_tris))
      return -1;
  }
  int count = 0;
  for (int i = 0; i < n; ++i) {
    if (!(flags[i] & 1)) continue;
    const D3 x = v3(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
    for (int s = 0; s < S; ++s) {
      if (shape_flags && !(shape_flags[s] & 4)) continue;  // COLLIDE_PARTICLES (geometry/kernels.py:1033-1034)
      const int pw = particle_world ? particle_world[i] : -1, sw = shape_world ? shape_world[s] : -1;
      if (pw != -1 && sw != -1 && pw != sw) continue;  // geometry/kernels.py:1036-1043
      const double* X = shape_xform + 7 * s;  // X_bs
      const double* sc = shape_scale + 3 * s;
      // X_ws = body_q[body] X_bs (geometry/kernels.py:1045-1056)
      double Xw[7] = {X[0], X[1], X[2], X[3], X[4], X[5], X[6]};
      const int body = shape_body && body_q ? shape_body[s] : -1;
      if (body >= 0) {
        const double* B = body_q + 7 * body;
        const D3 pw = sdf::qrot(B + 3, v3(X[0], X[1], X[2])) + v3(B[0], B[1], B[2]);
        const double ax = B[3], ay = B[4], az = B[5], aw = B[6], bx = X[3], by = X[4], bz = X[5], bw = X[6];
        const double qw[4] = {aw * bx + bw * ax + ay * bz - az * by, aw * by + bw * ay + az * bx - ax * bz,
                              aw * bz + bw * az + ax * by - ay * bx, aw * bw - ax * bx - ay * by - az * bz};
        Xw[0] = pw.x, Xw[1] = pw.y, Xw[2] = pw.z, Xw[3] = qw[0], Xw[4] = qw[1], Xw[5] = qw[2], Xw[6] = qw[3];
      }
      const double qi[4] = {-Xw[3], -Xw[4], -Xw[5], Xw[6]};
      const D3 xl = sdf::qrot(qi, x - v3(Xw[0], Xw[1], Xw[2]));
      double d = 1.0e6;
      D3 nn = v3(0.0, 0.0, 0.0);
      switch (shape_type[s]) {
        case sdf::SPHERE: d = sdf::sphere(xl, sc[0]), nn = sdf::sphere_grad(xl); break;
        case sdf::BOX: d = sdf::box(xl, sc[0], sc[1], sc[2]), nn = sdf::box_grad(xl, sc[0], sc[1], sc[2]); break;
        case sdf::CAPSULE: d = sdf::capsule(xl, sc[0], sc[1]), nn = sdf::capsule_grad(xl, sc[1]); break;
        case sdf::CYLINDER: d = sdf::cylinder(xl, sc[0], sc[1]), nn = sdf::cylinder_grad(xl, sc[0], sc[1]); break;
        case sdf::ELLIPSOID: sdf::ellipsoid(xl, v3(sc[0], sc[1], sc[2]), d, nn); break;
        case sdf::CONE: d = sdf::cone(xl, sc[0], sc[1]), nn = sdf::cone_grad(xl, sc[0], sc[1]); break;
        case sdf::HFIELD: {
          const int k = hf_index[s];
          sdf::heightfield(hf_grid + 3 * k, hf_ext + 4 * k, elev, xl, d, nn);
          break;
        }
        case sdf::MESH:
        case sdf::CONVEX_MESH: {  // the query in the unscaled frame; distance and normal from the scaled point
          const int k = mesh_index[s];
          const sdf::MeshQ m{mesh_vert_off[k + 1] - mesh_vert_off[k], mesh_tri_off[k + 1] - mesh_tri_off[k],
                             mesh_pts + 3 * mesh_vert_off[k], mesh_tris + 3 * mesh_tri_off[k]};
          const double ms = std::min(std::min(std::fabs(sc[0]), std::fabs(sc[1])), std::fabs(sc[2]));
          D3 cp;
          double sg;
          if (sdf::mesh_query(m, v3(xl.x / sc[0], xl.y / sc[1], xl.z / sc[2]), margin + radius[i] / ms, cp, sg)) {
            const D3 delta = xl - v3(cp.x * sc[0], cp.y * sc[1], cp.z * sc[2]);
            d = length(delta) * sg;
            nn = sdf::normalize0(delta) * sg;
          }
          break;
        }
        default: d = sdf::plane(xl, sc[0] * 0.5, sc[1] * 0.5), nn = v3(0.0, 0.0, 1.0); break;
      }
      if (d < margin + radius[i]) {
        if (count < max_contacts) {
          const D3 bp = sdf::qrot(X + 3, xl - nn * d) + v3(X[0], X[1], X[2]);  // body frame
          const D3 wn = sdf::qrot(Xw + 3, nn);
          particle[count] = i;
          shape[count] = s;
          body_pos[3 * count] = bp.x, body_pos[3 * count + 1] = bp.y, body_pos[3 * count + 2] = bp.z;
          body_vel[3 * count] = body_vel[3 * count + 1] = body_vel[3 * count + 2] = 0.0;
          normal[3 * count] = wn.x, normal[3 * count + 1] = wn.y, normal[3 * count + 2] = wn.z;
        }
        ++count;
      }
    }
  }
  return count;
}

int oracle_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
