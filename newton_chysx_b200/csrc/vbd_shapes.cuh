// Signed distances and outward gradients of the analytic collision shapes, in the shape's local frame, for
// particle-shape contact generation (create_soft_contacts, geometry/kernels.py:1001-1140, with the SDFs of
// geometry/kernels.py:132-600). Capsules and cylinders run along local Z (the reference passes Axis.Z);
// cylinders are straight (equal top and bottom radius). Shape type codes are the reference's GeoType values.
#pragma once
#include "vbd_math.cuh"

namespace vbd {

enum GeoTypeCode { GEO_PLANE = 1, GEO_SPHERE = 3, GEO_CAPSULE = 4, GEO_ELLIPSOID = 5, GEO_CYLINDER = 6, GEO_BOX = 7 };

__device__ __forceinline__ float geo_sign(float x) { return x < 0.f ? -1.f : 1.f; }  // wp.sign

// d and n of point p for a shape of type `type` with scale sc (GeoType conventions: sphere (r), box (hx, hy, hz),
// capsule and cylinder (r, half height), ellipsoid (rx, ry, rz), plane (width, length; 0 = infinite)).
__device__ __forceinline__ void shape_sdf(int type, vec3<float> p, const float sc[3], float& d, vec3<float>& n) {
  d = 1.0e6f;
  n = {0.f, 0.f, 1.f};
  if (type == GEO_SPHERE) {  // :165-195
    const float l = length(p);
    d = l - sc[0];
    if (l > 1.0e-8f) n = p * (1.f / l);
  } else if (type == GEO_BOX) {  // :198-259
    const float qx = fabsf(p.x) - sc[0], qy = fabsf(p.y) - sc[1], qz = fabsf(p.z) - sc[2];
    const vec3<float> e = {fmaxf(qx, 0.f), fmaxf(qy, 0.f), fmaxf(qz, 0.f)};
    d = length(e) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.f);
    if (qx > 0.f || qy > 0.f || qz > 0.f) {
      const vec3<float> c = {fminf(fmaxf(p.x, -sc[0]), sc[0]), fminf(fmaxf(p.y, -sc[1]), sc[1]),
                             fminf(fmaxf(p.z, -sc[2]), sc[2])};
      const vec3<float> g = p - c;
      const float gl = length(g);
      n = gl > 0.f ? g * (1.f / gl) : g;
    } else if ((qx > qy && qx > qz) || (qy == 0.f && qz == 0.f)) {
      n = {geo_sign(p.x), 0.f, 0.f};
    } else if ((qy > qx && qy > qz) || (qx == 0.f && qz == 0.f)) {
      n = {0.f, geo_sign(p.y), 0.f};
    } else {
      n = {0.f, 0.f, geo_sign(p.z)};
    }
  } else if (type == GEO_CAPSULE) {  // :262-329
    const float hh = sc[1];
    vec3<float> v = {p.x, p.y, 0.f};
    vec3<float> g = {0.f, 0.f, 1.f};
    if (p.z > hh) {
      v.z = p.z - hh;
    } else if (p.z < -hh) {
      v.z = p.z + hh;
      g.z = -1.f;
    }
    const float l = length(v);
    d = l - sc[0];
    n = l > 1.0e-8f ? v * (1.f / l) : g;
  } else if (type == GEO_CYLINDER) {  // :332-446
    const vec3<float> v = {p.x, p.y, 0.f};
    const float vl = length(v);
    const float dx = vl - sc[0], dy = fabsf(p.z) - sc[1];
    const float ex = fmaxf(dx, 0.f), ey = fmaxf(dy, 0.f);
    d = fminf(fmaxf(dx, dy), 0.f) + sqrtf(ex * ex + ey * ey);
    const vec3<float> radial = vl > 1.0e-8f ? v * (1.f / vl) : vec3<float>{0.f, 0.f, 1.f};
    const vec3<float> axial = {0.f, 0.f, geo_sign(p.z)};
    if (dx > 0.f && dy > 0.f) {
      const vec3<float> g = radial * dx + axial * dy;
      const float gl = length(g);
      n = gl > 1.0e-8f ? g * (1.f / gl) : radial;
    } else {
      n = dx > dy ? radial : axial;
    }
  } else if (type == GEO_ELLIPSOID) {  // :449-512
    const float rx = fmaxf(fabsf(sc[0]), 1.0e-8f), ry = fmaxf(fabsf(sc[1]), 1.0e-8f), rz = fmaxf(fabsf(sc[2]), 1.0e-8f);
    const float ix = 1.f / rx, iy = 1.f / ry, iz = 1.f / rz;
    const vec3<float> q0 = {p.x * ix, p.y * iy, p.z * iz};
    const vec3<float> q1 = {p.x * (ix * ix), p.y * (iy * iy), p.z * (iz * iz)};
    const float k0 = length(q0), k1 = length(q1);
    d = k1 > 1.0e-8f ? k0 * (k0 - 1.f) / k1 : -fminf(fminf(rx, ry), rz);
    if (!(k1 < 1.0e-8f)) {
      const vec3<float> g = q1 * (k0 / k1);
      const float gl = length(g);
      if (gl > 1.0e-8f) n = g * (1.f / gl);
    }
  } else if (type == GEO_PLANE) {  // :568-589; the contact normal is local +Z
    const float w = sc[0] * 0.5f, l = sc[1] * 0.5f;
    d = (w > 0.f && l > 0.f) ? fmaxf(fmaxf(fabsf(p.x) - w, fabsf(p.y) - l), fabsf(p.z)) : p.z;
  }
}

}  // namespace vbd
