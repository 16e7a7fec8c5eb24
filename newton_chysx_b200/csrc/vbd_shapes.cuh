// Signed distances and outward gradients of the analytic collision shapes, in the shape's local frame, for
// particle-shape contact generation (create_soft_contacts, geometry/kernels.py:1001-1140, with the SDFs of
// geometry/kernels.py:132-600). Capsules and cylinders run along local Z (the reference passes Axis.Z);
// cylinders are straight (equal top and bottom radius). Shape type codes are the reference's GeoType values.
#pragma once
#include "vbd_math.cuh"

namespace vbd {

enum GeoTypeCode {
  GEO_PLANE = 1,
  GEO_HFIELD = 2,
  GEO_SPHERE = 3,
  GEO_CAPSULE = 4,
  GEO_ELLIPSOID = 5,
  GEO_CYLINDER = 6,
  GEO_BOX = 7,
  GEO_MESH = 8,
  GEO_CONE = 9,
  GEO_CONVEX_MESH = 10
};

__device__ __forceinline__ float geo_sign(float x) { return x < 0.f ? -1.f : 1.f; }  // wp.sign
// clamp that maps NaN to lo, so that an index derived from it stays in range
__device__ __forceinline__ float geo_clamp(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ vec3<float> geo_normalize(vec3<float> a) {  // wp.normalize: zero stays zero
  const float l = length(a);
  return l > 0.f ? a * (1.f / l) : a;
}

// d and n of point p for a shape of type `type` with scale sc (GeoType conventions: sphere (r), box (hx, hy, hz),
// capsule, cylinder and cone (r, half height), ellipsoid (rx, ry, rz), plane (width, length; 0 = infinite)).
// Heightfields go through heightfield_sdf.
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
  } else if (type == GEO_CONE) {  // :141-161 with top radius 0, :515-564; base at z = -hh, apex at z = +hh
    const float r = sc[0], hh = sc[1];
    const float qx = sqrtf(p.x * p.x + p.y * p.y), qy = p.z;
    const float k2x = -r, k2y = 2.f * hh;
    const float cax = qx - fminf(qx, qy < 0.f ? r : 0.f), cay = fabsf(qy) - hh;
    const float den = k2x * k2x + k2y * k2y;
    const float t = den > 0.f ? fminf(fmaxf(((0.f - qx) * k2x + (hh - qy) * k2y) / den, 0.f), 1.f) : 0.f;
    const float cbx = qx + k2x * t, cby = qy - hh + k2y * t;
    const float sg = (cbx < 0.f && cay < 0.f) ? -1.f : 1.f;
    d = sg * sqrtf(fminf(cax * cax + cay * cay, cbx * cbx + cby * cby));
    if (hh <= 0.f) {
      n = {0.f, 0.f, geo_sign(p.z)};
    } else {
      const float dx = qx - r * (hh - p.z) / (2.f * hh), dy = fabsf(p.z) - hh;
      if (dx > dy)
        n = qx > 0.f ? geo_normalize(vec3<float>{p.x / qx, p.y / qx, r / (2.f * hh)}) : vec3<float>{0.f, 0.f, 1.f};
      else
        n = {0.f, 0.f, geo_sign(p.z)};
    }
  } else if (type == GEO_PLANE) {  // :568-589; the contact normal is local +Z
    const float w = sc[0] * 0.5f, l = sc[1] * 0.5f;
    d = (w > 0.f && l > 0.f) ? fmaxf(fmaxf(fabsf(p.x) - w, fabsf(p.y) - l), fabsf(p.z)) : p.z;
  }
}

// Signed distance and gradient of a heightfield (sample_sdf_grad_heightfield, utils/heightfield.py:94-205): grid
// `g` = (data_offset, nrow, ncol), extents `e` = (hx, hy, min_z, max_z) with the shape's scale applied, normalized
// elevations `elev` (z = min_z + e (max_z - min_z)). The point is clamped to the footprint; the cell's triangle
// (split along the diagonal from (col, row) to (col + 1, row + 1)) gives the plane distance and normal; outside
// the footprint the lateral gap is folded into the distance. Reads stay inside the grid for any input,
// NaN included (geo_clamp).
__device__ __forceinline__ void heightfield_sdf(int4 g, float4 e, const float* __restrict__ elev, vec3<float> p,
                                                float& d, vec3<float>& n) {
  const int nrow = g.y, ncol = g.z;
  if (nrow <= 1 || ncol <= 1) {
    d = 1.0e10f;
    n = {0.f, 0.f, 1.f};
    return;
  }
  const float hx = e.x, hy = e.y, zmin = e.z, zr = e.w - e.z;
  const float dx = 2.f * hx / float(ncol - 1), dy = 2.f * hy / float(nrow - 1);
  const float cx = geo_clamp(p.x, -hx, hx), cy = geo_clamp(p.y, -hy, hy);
  const float ox = p.x - cx, oy = p.y - cy;
  const float lat = ox * ox + oy * oy;
  const float colf = geo_clamp((cx + hx) / dx, 0.f, float(ncol - 1));
  const float rowf = geo_clamp((cy + hy) / dy, 0.f, float(nrow - 1));
  const int col = min(int(colf), ncol - 2), row = min(int(rowf), nrow - 2);
  const float fx = colf - float(col), fy = rowf - float(row);
  const float* z = elev + g.x + long(row) * ncol + col;
  const float h00 = zmin + __ldg(z) * zr, h10 = zmin + __ldg(z + 1) * zr;
  const float h01 = zmin + __ldg(z + ncol) * zr, h11 = zmin + __ldg(z + ncol + 1) * zr;
  const vec3<float> v0 = {-hx + float(col) * dx, -hy + float(row) * dy, h00};
  vec3<float> e1, e2;
  if (fx >= fy) {
    e1 = {dx, 0.f, h10 - h00};
    e2 = {dx, dy, h11 - h00};
  } else {
    e1 = {dx, dy, h11 - h00};
    e2 = {0.f, dy, h01 - h00};
  }
  const vec3<float> nrm = geo_normalize(cross(e1, e2));
  const float dp = dot(p - v0, nrm);
  if (lat > 0.f) {
    d = sqrtf(lat + dp * dp);
    const vec3<float> raw = vec3<float>{ox, oy, 0.f} + nrm * dp;
    n = dot(raw, raw) > 1.0e-20f ? geo_normalize(raw) : vec3<float>{0.f, 0.f, 1.f};
  } else {
    d = dp;
    n = nrm;
  }
}

}  // namespace vbd
