// Small fixed-size vector algebra for the VBD kernels, templated on the real type.
// Symmetric 3x3 matrices are stored as 6 entries (xx, yy, zz, xy, xz, yz): every Hessian term on
// this path is a sum of outer products a a^T and scaled identities, so it is symmetric by
// construction, and keeping 6 instead of 9 entries saves registers and shuffles.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace vbd {

template <typename R>
struct vec3 {
  R x, y, z;
};

template <typename R>
struct sym3 {
  R xx, yy, zz, xy, xz, yz;
};

template <typename R> __host__ __device__ __forceinline__ vec3<R> mk(R a, R b, R c) { return {a, b, c}; }
template <typename R> __host__ __device__ __forceinline__ vec3<R> zero3() { return {R(0), R(0), R(0)}; }
template <typename R> __host__ __device__ __forceinline__ vec3<R> operator+(vec3<R> a, vec3<R> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename R> __host__ __device__ __forceinline__ vec3<R> operator-(vec3<R> a, vec3<R> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename R> __host__ __device__ __forceinline__ vec3<R> operator-(vec3<R> a) { return {-a.x, -a.y, -a.z}; }
template <typename R> __host__ __device__ __forceinline__ vec3<R> operator*(vec3<R> a, R s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <typename R> __host__ __device__ __forceinline__ vec3<R> operator*(R s, vec3<R> a) {
  return {a.x * s, a.y * s, a.z * s};
}
template <typename R> __host__ __device__ __forceinline__ R dot(vec3<R> a, vec3<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename R> __host__ __device__ __forceinline__ vec3<R> cross(vec3<R> a, vec3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ float vsqrt(float x) { return sqrtf(x); }
__host__ __device__ __forceinline__ double vsqrt(double x) { return sqrt(x); }
// FP32 atan2 on the device: the minimax polynomial of Abramowitz & Stegun 4.4.49 for atan on [0, 1]
// (|error| <= 4e-8 in exact arithmetic, ~1e-7 evaluated in FP32, the accuracy of the library atan2f),
// extended to all quadrants by atan(y/x) = pi/2 - atan(x/y) and the signs of x and y. The ratio uses the fast
// division (2 ulp). The host keeps atan2f.
__host__ __device__ __forceinline__ float vatan2(float y, float x) {
#ifdef __CUDA_ARCH__
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(fmaxf(ax, ay), 1.0e-30f), mn = fminf(ax, ay);
  const float t = __fdividef(mn, mx);
  const float t2 = t * t;
  float p = -0.0040540580f;
  p = fmaf(p, t2, 0.0218612288f);
  p = fmaf(p, t2, -0.0559098861f);
  p = fmaf(p, t2, 0.0964200441f);
  p = fmaf(p, t2, -0.1390853351f);
  p = fmaf(p, t2, 0.1994653599f);
  p = fmaf(p, t2, -0.3332985605f);
  p = fmaf(p, t2, 0.9999993329f);
  float r = p * t;
  if (ay > ax) r = 1.57079632679489662f - r;
  if (x < 0.f) r = 3.14159265358979324f - r;
  return copysignf(r, y);
#else
  return atan2f(y, x);
#endif
}
// reciprocal square root: the hardware approximation on the device for float, exact elsewhere
__host__ __device__ __forceinline__ float vrsqrt(float x) {
#ifdef __CUDA_ARCH__
  return rsqrtf(x);
#else
  return 1.0f / sqrtf(x);
#endif
}
__host__ __device__ __forceinline__ double vrsqrt(double x) { return 1.0 / sqrt(x); }
// reciprocal: the hardware approximation on the device for float (through the fast division), exact elsewhere
__host__ __device__ __forceinline__ float vrcp(float x) {
#ifdef __CUDA_ARCH__
  return __fdividef(1.0f, x);
#else
  return 1.0f / x;
#endif
}
__host__ __device__ __forceinline__ double vrcp(double x) { return 1.0 / x; }
// a / b for material ratios: the fast (2 ulp) division on the device for float, exact elsewhere
__host__ __device__ __forceinline__ float vdiv_fast(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdividef(a, b);
#else
  return a / b;
#endif
}
__host__ __device__ __forceinline__ double vdiv_fast(double a, double b) { return a / b; }
template <typename T> __host__ __device__ __forceinline__ T vdiv_fast(const T& a, const T& b) { return a / b; }
__host__ __device__ __forceinline__ double vatan2(double y, double x) { return atan2(y, x); }
template <typename R> __host__ __device__ __forceinline__ R vabs(R x) { return x < R(0) ? -x : x; }
template <typename R> __host__ __device__ __forceinline__ R vmax(R a, R b) { return a > b ? a : b; }
template <typename R> __host__ __device__ __forceinline__ R vmin(R a, R b) { return a < b ? a : b; }
template <typename R> __host__ __device__ __forceinline__ R length(vec3<R> a) { return vsqrt(dot(a, a)); }

template <typename R> __host__ __device__ __forceinline__ sym3<R> szero() { return {R(0), R(0), R(0), R(0), R(0), R(0)}; }
template <typename R> __host__ __device__ __forceinline__ sym3<R> sdiag(R d) { return {d, d, d, R(0), R(0), R(0)}; }
template <typename R> __host__ __device__ __forceinline__ sym3<R> operator+(sym3<R> a, sym3<R> b) {
  return {a.xx + b.xx, a.yy + b.yy, a.zz + b.zz, a.xy + b.xy, a.xz + b.xz, a.yz + b.yz};
}
template <typename R> __host__ __device__ __forceinline__ sym3<R> operator*(R s, sym3<R> a) {
  return {s * a.xx, s * a.yy, s * a.zz, s * a.xy, s * a.xz, s * a.yz};
}
// s * a a^T
template <typename R> __host__ __device__ __forceinline__ sym3<R> souter(vec3<R> a, R s) {
  vec3<R> b = a * s;
  return {a.x * b.x, a.y * b.y, a.z * b.z, a.x * b.y, a.x * b.z, a.y * b.z};
}
// acc += s * a a^T
template <typename R> __host__ __device__ __forceinline__ void souter_add(sym3<R>& acc, vec3<R> a, R s) {
  vec3<R> b = a * s;
  acc.xx += a.x * b.x;
  acc.yy += a.y * b.y;
  acc.zz += a.z * b.z;
  acc.xy += a.x * b.y;
  acc.xz += a.x * b.z;
  acc.yz += a.y * b.z;
}
template <typename R> __host__ __device__ __forceinline__ vec3<R> smul(const sym3<R>& a, vec3<R> v) {
  return {a.xx * v.x + a.xy * v.y + a.xz * v.z, a.xy * v.x + a.yy * v.y + a.yz * v.z,
          a.xz * v.x + a.yz * v.y + a.zz * v.z};
}
template <typename R> __host__ __device__ __forceinline__ R sdet(const sym3<R>& a) {
  return a.xx * (a.yy * a.zz - a.yz * a.yz) - a.xy * (a.xy * a.zz - a.yz * a.xz) + a.xz * (a.xy * a.yz - a.yy * a.xz);
}
// adj(a) * v  (adjugate of a symmetric matrix is symmetric)
template <typename R> __host__ __device__ __forceinline__ vec3<R> sadj_mul(const sym3<R>& a, vec3<R> v) {
  sym3<R> c;
  c.xx = a.yy * a.zz - a.yz * a.yz;
  c.yy = a.xx * a.zz - a.xz * a.xz;
  c.zz = a.xx * a.yy - a.xy * a.xy;
  c.xy = a.xz * a.yz - a.xy * a.zz;
  c.xz = a.xy * a.yz - a.xz * a.yy;
  c.yz = a.xy * a.xz - a.xx * a.yz;
  return smul(c, v);
}

template <typename R> __host__ __device__ __forceinline__ vec3<R> ld3(const float4& a) { return {R(a.x), R(a.y), R(a.z)}; }
template <typename R> __host__ __device__ __forceinline__ vec3<R> ld3(const double4& a) { return {R(a.x), R(a.y), R(a.z)}; }

// Internal position storage: float4 in FP32 mode, double4 in FP64 mode.
template <typename R> struct store4;
template <> struct store4<float> {
  using type = float4;
};
template <> struct store4<double> {
  using type = double4;
};
template <typename R> using pos4_t = typename store4<R>::type;

__host__ __device__ __forceinline__ float4 pk4(vec3<float> v, float w) { return make_float4(v.x, v.y, v.z, w); }
__host__ __device__ __forceinline__ double4 pk4(vec3<double> v, double w) { return make_double4(v.x, v.y, v.z, w); }

#ifdef __CUDACC__
// warp reduction of a partial (f, H) over groups of L adjacent lanes
template <int L, typename R> __device__ __forceinline__ R group_sum(R v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
#endif

}  // namespace vbd
