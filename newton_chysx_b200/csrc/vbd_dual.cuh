// Forward-mode dual numbers for the element Jacobians used by the VBD adjoint.
//
// The element routines of vbd_elements.cuh are templated on the real type. Instantiated with
// Dual<R, N>, where each of the N derivative slots is seeded with one input (a coordinate of a vertex
// or a material parameter), the same code returns the force and Hessian together with their
// derivatives with respect to those inputs. The adjoint contracts them with the output adjoints.
// Non-smooth operations take the derivative of the branch that is active (max, min, abs, the
// comparisons that select a formula), as reverse-mode differentiation of the same code would.
#pragma once
#include <type_traits>

#include "vbd_math.cuh"

namespace vbd {

template <typename R, int N>
struct Dual {
  R v;
  R d[N];
  __host__ __device__ __forceinline__ Dual() : v(R(0)) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = R(0);
  }
  // constants (any arithmetic type) promote implicitly, with zero derivative
  template <typename S, typename = typename std::enable_if<std::is_arithmetic<S>::value>::type>
  __host__ __device__ __forceinline__ Dual(S x) : v(R(x)) {  // NOLINT
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = R(0);
  }
  __host__ __device__ __forceinline__ static Dual seed(R x, int slot) {
    Dual r(x);
    r.d[slot] = R(1);
    return r;
  }
};

#define VBD_DUAL_T template <typename R, int N>
#define VBD_HD __host__ __device__ __forceinline__

VBD_DUAL_T VBD_HD Dual<R, N> operator+(const Dual<R, N>& a, const Dual<R, N>& b) {
  Dual<R, N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N> operator-(const Dual<R, N>& a, const Dual<R, N>& b) {
  Dual<R, N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N> operator-(const Dual<R, N>& a) {
  Dual<R, N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N> operator*(const Dual<R, N>& a, const Dual<R, N>& b) {
  Dual<R, N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N> operator/(const Dual<R, N>& a, const Dual<R, N>& b) {
  Dual<R, N> r;
  const R inv = R(1) / b.v;
  r.v = a.v * inv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N>& operator+=(Dual<R, N>& a, const Dual<R, N>& b) { return a = a + b; }
VBD_DUAL_T VBD_HD Dual<R, N>& operator-=(Dual<R, N>& a, const Dual<R, N>& b) { return a = a - b; }
VBD_DUAL_T VBD_HD bool operator<(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v < b.v; }
VBD_DUAL_T VBD_HD bool operator>(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v > b.v; }
VBD_DUAL_T VBD_HD bool operator>=(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v >= b.v; }
VBD_DUAL_T VBD_HD bool operator<=(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v <= b.v; }
VBD_DUAL_T VBD_HD bool operator==(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v == b.v; }
VBD_DUAL_T VBD_HD bool operator!=(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v != b.v; }

VBD_DUAL_T VBD_HD Dual<R, N> vsqrt(const Dual<R, N>& a) {
  Dual<R, N> r;
  r.v = vsqrt(a.v);
  const R k = R(0.5) / r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * k;
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N> vrsqrt(const Dual<R, N>& a) {
  Dual<R, N> r;
  r.v = vrsqrt(a.v);
  const R k = R(-0.5) * r.v / a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * k;
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N> vrcp(const Dual<R, N>& a) {
  Dual<R, N> r;
  r.v = vrcp(a.v);
  const R k = -r.v * r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * k;
  return r;
}
VBD_DUAL_T VBD_HD Dual<R, N> vatan2(const Dual<R, N>& y, const Dual<R, N>& x) {
  Dual<R, N> r;
  r.v = vatan2(y.v, x.v);
  const R inv = R(1) / (x.v * x.v + y.v * y.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) * inv;
  return r;
}

#undef VBD_DUAL_T
#undef VBD_HD

// dual-aware helpers used by the element routines (vabs, vmax, vmin are generic on operator<)
template <typename R, int N>
__host__ __device__ __forceinline__ R value(const Dual<R, N>& a) {
  return a.v;
}
template <typename R>
__host__ __device__ __forceinline__ R value(R a) {
  return a;
}

}  // namespace vbd
