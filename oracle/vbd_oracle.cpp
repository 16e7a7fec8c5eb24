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
//   adjacency  particle_vbd_kernels.py:639-738 (count/fill order)
//   contacts   geometry/kernels.py:1001-1140 for PLANE (infinite) and SPHERE shapes
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
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
};

struct Contacts {
  int count, max;
  const int *particle, *shape;
  const double *body_pos, *body_vel, *normal;
};

template <typename R> inline V3<R> ld(const double* a, int i) { return {R(a[3 * i]), R(a[3 * i + 1]), R(a[3 * i + 2])}; }
template <typename R> inline V3<R> ld(const std::vector<V3<R>>& a, int i) { return a[i]; }

// One SolverVBD.step without self-contact and without rigid bodies (static shapes only).
template <typename R>
int step(const Model& M, double* q_in, const double* qd_in, const double* f_ext, const Contacts& Cn, R dt,
         int iterations, double* q_out, double* qd_out, int nthreads) {
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
  // _initialize_particles: pos_prev_collision_detection = q, displacements = 0, forward_step
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
  // apply_truncation_ts with t = 1, max_displacement = inf: pos = pos_cd + disp
  auto truncate = [&]() {
    for (int i = 0; i < n; ++i) pos[i] = pos_cd[i] + disp[i];
  };
  truncate();
  const R dt2r = R(1) / (dt * dt);
  const R beta = R(M.beta);
  for (int it = 0; it < iterations; ++it) {
    // update_duals_body_particle_contacts (rigid_vbd_kernels.py:3755-3799)
    for (int c = 0; c < ccount; ++c) {
      int p = Cn.particle[c];
      V3<R> bx = ld<R>(Cn.body_pos, c), nn = ld<R>(Cn.normal, c);
      R pen = -(dot(nn, pos[p] - bx) - R(M.radius[p]));
      pen = rmax(R(0), pen);
      pen_k[c] = rmin(pen_k[c] + beta * pen, mat_ke[c]);
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
        V3<R> bx = ld<R>(Cn.body_pos, c), nn = ld<R>(Cn.normal, c);
        R pen = -(dot(nn, pos[p] - bx) - R(M.radius[p]));
        if (pen > R(0)) {
          V3<R> dx = pos[p] - q_prev[p];
          V3<R> bv = ld<R>(Cn.body_vel, c);
          V3<R> rel = dx - bv * dt;
          V3<R> f;
          M3<R> H;
          contact_force(pen, nn, rel, pen_k[c], mat_kd[c], mat_mu[c], R(M.friction_epsilon), dt, f, H);
          forces[p] = forces[p] + f;
          hess[p] = hess[p] + H;
        }
      }
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
};

struct OracleContacts {
  int count, max;
  const int *particle, *shape;
  const double *body_pos, *body_vel, *normal;
};

static_assert(sizeof(OracleModel) == sizeof(Model), "layout");

// precision: 64 = all-FP64 run, 32 = FP32 run (inputs rounded to float).
int oracle_vbd_step(const OracleModel* m, double* q_in, const double* qd_in, const double* f_ext,
                    const OracleContacts* c, double dt, int iterations, double* q_out, double* qd_out, int precision,
                    int nthreads) {
  Model M;
  std::memcpy(&M, m, sizeof(M));
  Contacts C{c->count, c->max, c->particle, c->shape, c->body_pos, c->body_vel, c->normal};
  if (nthreads < 1) nthreads = 1;
  if (precision == 64) return step<double>(M, q_in, qd_in, f_ext, C, dt, iterations, q_out, qd_out, nthreads);
  if (precision == 32)
    return step<float>(M, q_in, qd_in, f_ext, C, float(dt), iterations, q_out, qd_out, nthreads);
  return -1;
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

int oracle_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
