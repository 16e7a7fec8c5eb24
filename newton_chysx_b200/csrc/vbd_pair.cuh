// Paired FP32 arithmetic for the sweep: one thread solves two vertices of a color at once, the two vertices'
// values living in the two lanes of a float2, and every add, multiply and fused multiply-add is one paired
// instruction (sm_100 FADD2 / FMUL2 / FFMA2 through __fadd2_rn / __fmul2_rn / __ffma2_rn). Each lane is
// rounded exactly like the scalar instruction, so a lane computes what the scalar code computes up to the
// compiler's choice of where to fuse a multiply and an add. Square roots and divisions stay scalar per lane;
// atan2 evaluates the polynomial of vatan2 (vbd_math.cuh) in paired instructions. Only the FP32 sweep uses this.
#pragma once
#include <cuda_runtime.h>

#include "vbd_math.cuh"

namespace vbd {

struct pf {
  float2 v;
};

__device__ __forceinline__ pf pf2(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ pf pfs(float a) { return {make_float2(a, a)}; }
__device__ __forceinline__ pf operator+(pf a, pf b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ pf operator*(pf a, pf b) { return {__fmul2_rn(a.v, b.v)}; }
// a - b = b * (-1) + a: one rounding, as the scalar subtraction
__device__ __forceinline__ pf operator-(pf a, pf b) { return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ pf operator-(pf a) { return {make_float2(-a.v.x, -a.v.y)}; }
__device__ __forceinline__ pf pfma(pf a, pf b, pf c) { return {__ffma2_rn(a.v, b.v, c.v)}; }  // a * b + c
// c - a * b
__device__ __forceinline__ pf pfms(pf a, pf b, pf c) { return {__ffma2_rn(make_float2(-a.v.x, -a.v.y), b.v, c.v)}; }
__device__ __forceinline__ pf pmax(pf a, pf b) { return pf2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }
__device__ __forceinline__ pf prsqrt(pf a) { return pf2(rsqrtf(a.v.x), rsqrtf(a.v.y)); }
__device__ __forceinline__ pf pdiv(pf a, pf b) { return pf2(a.v.x / b.v.x, a.v.y / b.v.y); }
// vdiv_fast per lane
__device__ __forceinline__ pf pdiv_fast(pf a, pf b) { return pf2(__fdividef(a.v.x, b.v.x), __fdividef(a.v.y, b.v.y)); }
// vatan2 (vbd_math.cuh) with the polynomial in paired instructions
__device__ __forceinline__ pf patan2(pf y, pf x) {
  const float ax0 = fabsf(x.v.x), ay0 = fabsf(y.v.x), ax1 = fabsf(x.v.y), ay1 = fabsf(y.v.y);
  const pf t = pf2(__fdividef(fminf(ax0, ay0), fmaxf(fmaxf(ax0, ay0), 1.0e-30f)),
                   __fdividef(fminf(ax1, ay1), fmaxf(fmaxf(ax1, ay1), 1.0e-30f)));
  const pf t2 = t * t;
  pf p = pfma(pfs(-0.0040540580f), t2, pfs(0.0218612288f));
  p = pfma(p, t2, pfs(-0.0559098861f));
  p = pfma(p, t2, pfs(0.0964200441f));
  p = pfma(p, t2, pfs(-0.1390853351f));
  p = pfma(p, t2, pfs(0.1994653599f));
  p = pfma(p, t2, pfs(-0.3332985605f));
  p = pfma(p, t2, pfs(0.9999993329f));
  const pf r = p * t;
  float r0 = r.v.x, r1 = r.v.y;
  if (ay0 > ax0) r0 = 1.57079632679489662f - r0;
  if (ay1 > ax1) r1 = 1.57079632679489662f - r1;
  if (x.v.x < 0.f) r0 = 3.14159265358979324f - r0;
  if (x.v.y < 0.f) r1 = 3.14159265358979324f - r1;
  return pf2(copysignf(r0, y.v.x), copysignf(r1, y.v.y));
}

struct pv3 {
  pf x, y, z;
};
__device__ __forceinline__ pv3 operator+(pv3 a, pv3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ pv3 operator-(pv3 a, pv3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ pv3 operator*(pv3 a, pf s) { return {a.x * s, a.y * s, a.z * s}; }
// a * s + b
__device__ __forceinline__ pv3 pfma(pv3 a, pf s, pv3 b) { return {pfma(a.x, s, b.x), pfma(a.y, s, b.y), pfma(a.z, s, b.z)}; }
__device__ __forceinline__ pf pdot(pv3 a, pv3 b) { return pfma(a.z, b.z, pfma(a.y, b.y, a.x * b.x)); }
__device__ __forceinline__ pv3 pcross(pv3 a, pv3 b) {
  return {pfms(a.z, b.y, a.y * b.z), pfms(a.x, b.z, a.z * b.x), pfms(a.y, b.x, a.x * b.y)};
}
__device__ __forceinline__ pv3 pv3_of(vec3<float> a, vec3<float> b) { return {pf2(a.x, b.x), pf2(a.y, b.y), pf2(a.z, b.z)}; }
__device__ __forceinline__ vec3<float> lane0(pv3 a) { return {a.x.v.x, a.y.v.x, a.z.v.x}; }
__device__ __forceinline__ vec3<float> lane1(pv3 a) { return {a.x.v.y, a.y.v.y, a.z.v.y}; }

struct psym {
  pf xx, yy, zz, xy, xz, yz;
};
// acc += s a a^T
__device__ __forceinline__ void psouter_add(psym& h, pv3 a, pf s) {
  const pv3 sa = a * s;
  h.xx = pfma(sa.x, a.x, h.xx);
  h.yy = pfma(sa.y, a.y, h.yy);
  h.zz = pfma(sa.z, a.z, h.zz);
  h.xy = pfma(sa.x, a.y, h.xy);
  h.xz = pfma(sa.x, a.z, h.xz);
  h.yz = pfma(sa.y, a.z, h.yz);
}
__device__ __forceinline__ sym3<float> lane0(const psym& h) {
  return {h.xx.v.x, h.yy.v.x, h.zz.v.x, h.xy.v.x, h.xz.v.x, h.yz.v.x};
}
__device__ __forceinline__ sym3<float> lane1(const psym& h) {
  return {h.xx.v.y, h.yy.v.y, h.zz.v.y, h.xy.v.y, h.xz.v.y, h.yz.v.y};
}

// Membrane term, for both lanes, of a face whose solved vertex is vertex 0 (the 16-bit stencil form: x1, x2 the
// other two vertices, pose = D^-1 re-expressed for that vertex, mu and lambda already scaled by the area). The
// scalar form is membrane_add (vbd_elements.cuh) with ord = 0, area = 1 and no damping; a face with
// mu = lambda = 0 adds exactly zero.
__device__ __forceinline__ void pmembrane_add(pv3 x0, pv3 x1, pv3 x2, pf D00, pf D01, pf D10, pf D11, pf mu, pf lmbd,
                                              pv3& f, psym& H) {
  const pv3 x01 = x1 - x0, x02 = x2 - x0;
  const pv3 f0 = pfma(x01, D00, x02 * D10);
  const pv3 f1 = pfma(x01, D01, x02 * D11);
  const pf f00 = pdot(f0, f0), f11 = pdot(f1, f1), f01 = pdot(f0, f1);
  const pf Jsq = pmax(pfms(f01, f01, f00 * f11), pfs(1.0e-20f));
  const pf invJ = prsqrt(Jsq);
  const pf J = Jsq * invJ;
  const pf lnh = lmbd + mu;
  // mu and lambda come pre-multiplied by the area: no floor here (membrane_add with lnh_floor = 0); a lane with
  // mu = lambda = 0 divides by 1 and adds exactly zero
  const pf lsafe = pf2(lnh.v.x == 0.f ? 1.f : lnh.v.x, lnh.v.y == 0.f ? 1.f : lnh.v.y);
  const pf alpha = pfs(1.f) + pdiv_fast(mu, lsafe);
  const pv3 g0 = pfma(f0, f11, f1 * (-f01)) * invJ;
  const pv3 g1 = pfma(f1, f00, f0 * (-f01)) * invJ;
  const pf s = lnh * (J - alpha);
  const pf d0 = -(D00 + D10), d1 = -(D01 + D11);
  // force = -((mu f0 + s g0) d0 + (mu f1 + s g1) d1)
  const pv3 P0 = pfma(g0, s, f0 * mu), P1 = pfma(g1, s, f1 * mu);
  f = f - pfma(P0, d0, P1 * d1);
  const pf r = pmax(pfs(0.f), s) * invJ;
  const pv3 dJ = pfma(g0, d0, g1 * d1);
  const pv3 w = pfma(f1, d0, f0 * (-d1));
  const pf d00 = d0 * d0, d11 = d1 * d1, d01 = d0 * d1;
  const pf Ic = pfma(mu, d00 + d11, r * pfma(pfs(-2.f) * d01, f01, pfma(d00, f11, d11 * f00)));
  H.xx = H.xx + Ic;
  H.yy = H.yy + Ic;
  H.zz = H.zz + Ic;
  psouter_add(H, dJ, lnh - r);
  psouter_add(H, w, -r);
}

// Bending term, for both lanes, of a hinge (x0 opposite 0, x1 opposite 1, x2-x3 the edge) for the vertex whose
// role (0..3) is given per lane; k = ke * rest length (0 adds exactly zero). The scalar form is bending_add
// (vbd_elements.cuh) without damping; a degenerate hinge (|N1|, |N2| or |e| below 1e-6) adds nothing.
__device__ __forceinline__ void pbending_add(const pv3 x[4], pf rest_angle, pf k, int role0, int role1, pv3& f,
                                             psym& H) {
  const pv3 x02 = x[2] - x[0], x03 = x[3] - x[0], x13 = x[3] - x[1], x12 = x[2] - x[1], e = x[3] - x[2];
  const pv3 N1 = pcross(x02, x03), N2 = pcross(x13, x12);
  pf s1 = pdot(N1, N1), s2 = pdot(N2, N2), se = pdot(e, e);
  const float eps2 = 1.0e-12f;
  const bool bad0 = s1.v.x < eps2 || s2.v.x < eps2 || se.v.x < eps2;
  const bool bad1 = s1.v.y < eps2 || s2.v.y < eps2 || se.v.y < eps2;
  if (bad0 && bad1) return;
  // a degenerate lane gets finite stand-in lengths and zero stiffness: it adds +-0
  pf kk = k;
  if (bad0) s1.v.x = s2.v.x = se.v.x = 1.f, kk.v.x = 0.f;
  if (bad1) s1.v.y = s2.v.y = se.v.y = 1.f, kk.v.y = 0.f;
  const pf il1 = prsqrt(s1), il2 = prsqrt(s2), ile = prsqrt(se);
  // the angle from the unnormalised normals (atan2 ignores the common factor |N1| |N2|), as bending_add
  const pf theta = patan2(pdot(pcross(N1, N2), e) * ile, pdot(N1, N2));
  const pf dE = kk * (theta - rest_angle);
  const pf le = se * ile;
  // dtheta/dx_role = alpha n1 + beta n2 (bending_add): roles 0, 1: -|e| / |N_i| on their own normal; roles 2, 3:
  // the projections of the far edges on e
  const pf c0 = pf2(role0 == 0, role1 == 0), c1 = pf2(role0 == 1, role1 == 1);
  const pf c2 = pf2(role0 == 2, role1 == 2), c3 = pf2(role0 == 3, role1 == 3);
  const pv3 a1 = pfma(x03, c2, x02 * (-c3)), a2 = pfma(x13, c2, x12 * (-c3));
  // d = alpha n1 + beta n2 = a N1 + b N2 with a = alpha / |N1|, b = beta / |N2|
  const pf a = pfms(c0, le, pdot(a1, e) * ile) * (il1 * il1);
  const pf b = pfms(c1, le, pdot(a2, e) * ile) * (il2 * il2);
  const pv3 d = pfma(N1, a, N2 * b);
  f = pfma(d, -dE, f);
  psouter_add(H, d, kk);
}

}  // namespace vbd
