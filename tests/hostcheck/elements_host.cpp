// Test infrastructure: compiles the product's element math (newton_chysx_b200/csrc/vbd_elements.cuh,
// which is __host__ __device__) for the host so that its formulas can be compared with the oracle
// on a machine without a GPU.
#include "../../newton_chysx_b200/csrc/vbd_elements.cuh"

using namespace vbd;

template <typename R>
static void run_membrane(int ord, const double* x, const double* xp, const double* pose, double area, double mu,
                         double lmbd, double damping, double dt, double* out) {
  vec3<R> X[3], XP[3];
  for (int i = 0; i < 3; ++i) {
    X[i] = {R(x[3 * i]), R(x[3 * i + 1]), R(x[3 * i + 2])};
    XP[i] = {R(xp[3 * i]), R(xp[3 * i + 1]), R(xp[3 * i + 2])};
  }
  R p[4] = {R(pose[0]), R(pose[1]), R(pose[2]), R(pose[3])};
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  membrane_add<R>(ord, X[0], X[1], X[2], p, R(mu), R(lmbd), R(damping), R(area), R(dt), XP, f, H);
  double o[12] = {f.x, f.y, f.z, H.xx, H.xy, H.xz, H.xy, H.yy, H.yz, H.xz, H.yz, H.zz};
  for (int i = 0; i < 12; ++i) out[i] = o[i];
}

template <typename R>
static void run_bending(int ord, const double* x, const double* xp, int boundary, double ra, double rl, double ke,
                        double kd, double dt, double* out) {
  vec3<R> X[4], XP[4];
  for (int i = 0; i < 4; ++i) {
    X[i] = {R(x[3 * i]), R(x[3 * i + 1]), R(x[3 * i + 2])};
    XP[i] = {R(xp[3 * i]), R(xp[3 * i + 1]), R(xp[3 * i + 2])};
  }
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  if (!boundary) bending_add<R>(ord, X, R(ra), R(rl), R(ke), R(kd), R(dt), XP, f, H);
  double o[12] = {f.x, f.y, f.z, H.xx, H.xy, H.xz, H.xy, H.yy, H.yz, H.xz, H.yz, H.zz};
  for (int i = 0; i < 12; ++i) out[i] = o[i];
}

template <typename R>
static void run_contact(double pen, const double* n, const double* rel, double ke, double kd, double mu, double eps,
                        double dt, double* out) {
  vec3<R> f = zero3<R>();
  sym3<R> H = szero<R>();
  contact_add<R>(R(pen), vec3<R>{R(n[0]), R(n[1]), R(n[2])}, vec3<R>{R(rel[0]), R(rel[1]), R(rel[2])}, R(ke), R(kd),
                 R(mu), R(eps), R(dt), f, H);
  double o[12] = {f.x, f.y, f.z, H.xx, H.xy, H.xz, H.xy, H.yy, H.yz, H.xz, H.yz, H.zz};
  for (int i = 0; i < 12; ++i) out[i] = o[i];
}

extern "C" {
void host_membrane(int prec, int ord, const double* x, const double* xp, const double* pose, double area, double mu,
                   double lmbd, double damping, double dt, double* out) {
  if (prec == 64) run_membrane<double>(ord, x, xp, pose, area, mu, lmbd, damping, dt, out);
  else run_membrane<float>(ord, x, xp, pose, area, mu, lmbd, damping, dt, out);
}
void host_bending(int prec, int ord, const double* x, const double* xp, int boundary, double ra, double rl, double ke,
                  double kd, double dt, double* out) {
  if (prec == 64) run_bending<double>(ord, x, xp, boundary, ra, rl, ke, kd, dt, out);
  else run_bending<float>(ord, x, xp, boundary, ra, rl, ke, kd, dt, out);
}
void host_contact(int prec, double pen, const double* n, const double* rel, double ke, double kd, double mu,
                  double eps, double dt, double* out) {
  if (prec == 64) run_contact<double>(pen, n, rel, ke, kd, mu, eps, dt, out);
  else run_contact<float>(pen, n, rel, ke, kd, mu, eps, dt, out);
}
}
