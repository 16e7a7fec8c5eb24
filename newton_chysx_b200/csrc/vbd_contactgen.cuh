// One particle against one shape, as create_soft_contacts does it (geometry/kernels.py:1001-1140): the shape's
// world frame X_ws = body_q[body] X_bs (X_bs alone for a static shape, body -1), the particle in the shape frame,
// the shape's signed distance and outward normal (analytic SDFs, heightfield query, mesh query), and for
// d < margin + radius a contact at the closest surface point x_local - n d mapped to the body frame by X_bs, with
// the normal mapped to world by X_ws, in a slot taken from an atomic counter. Shared by the kernel-parameter path
// (at most kMaxContactShapes shapes per call) and the device-resident shape sets (any number of shapes and worlds).
#pragma once
#include <cmath>

#include "vbd_b200.h"
#include "vbd_mesh.cuh"
#include "vbd_shapes.cuh"

namespace vbd {

// A shape: transform in its body's frame (p, q xyzw; the world frame for a static shape), scale, and the data of
// its kind.
struct ShapeRec {
  float4 p;
  float4 q;    // unit quaternion (x, y, z, w)
  float4 sc;   // scale
  int4 hf;     // heightfield grid (data_offset, nrow, ncol, 0)
  float4 hfe;  // heightfield extents (hx, hy, min_z, max_z), scale applied
  MeshView mesh;
  int type;   // GeoType
  int world;  // -1 = global
  int id;     // index in the model
  int body;   // -1 = static (geometry/kernels.py:1045-1049)
};

__host__ __device__ __forceinline__ vec3<float> rot_q(float4 q, vec3<float> v) {
  const vec3<float> u = {q.x, q.y, q.z};
  return v * (2.f * q.w * q.w - 1.f) + cross(u, v) * (2.f * q.w) + u * (2.f * dot(u, v));
}

// Hamilton product a b of quaternions (x, y, z, w): the rotation b followed by a.
__host__ __device__ __forceinline__ float4 mul_q(float4 a, float4 b) {
  return make_float4(a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y, a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z,
                     a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}

// body_q: [bodies, 7] body transforms (p, q xyzw) of this call; read only for a shape on a body. BODIES = false
// compiles the body frame out (every shape of the launch is static).
template <bool BODIES>
__device__ __forceinline__ void soft_contact_shape(const ShapeRec& sh, const float* __restrict__ elev,
                                                   const float* __restrict__ body_q, vec3<float> x, float r,
                                                   float margin, int i, int cmax, int* count, int* particle,
                                                   int* shape, float* body_pos, float* body_vel, float* normal) {
  const float4 P = sh.p, Q = sh.q, SC = sh.sc;
  float4 Pw = P, Qw = Q;  // X_ws
  if (BODIES && sh.body >= 0) {
    const float* X = body_q + 7 * sh.body;
    const float4 Qb = make_float4(X[3], X[4], X[5], X[6]);
    const vec3<float> pw = rot_q(Qb, vec3<float>{P.x, P.y, P.z});
    Pw = make_float4(X[0] + pw.x, X[1] + pw.y, X[2] + pw.z, 0.f);
    Qw = mul_q(Qb, Q);
  }
  const float4 Qi = make_float4(-Qw.x, -Qw.y, -Qw.z, Qw.w);
  const vec3<float> xl = rot_q(Qi, vec3<float>{x.x - Pw.x, x.y - Pw.y, x.z - Pw.z});
  const float sc[3] = {SC.x, SC.y, SC.z};
  float d;
  vec3<float> nn;
  const int type = sh.type;
  if (type == GEO_HFIELD) {
    heightfield_sdf(sh.hf, sh.hfe, elev, xl, d, nn);
  } else if (type == GEO_MESH || type == GEO_CONVEX_MESH) {  // geometry/kernels.py:1091-1113
    d = 1.0e6f;
    nn = {0.f, 0.f, 0.f};
    const float ms = fminf(fminf(fabsf(sc[0]), fabsf(sc[1])), fabsf(sc[2]));
    const vec3<float> xs = {xl.x / sc[0], xl.y / sc[1], xl.z / sc[2]};
    vec3<float> cp;
    float sg;
    int face;
    if (mesh_query_point_sign(sh.mesh, xs, margin + r / ms, cp, sg, face)) {
      const vec3<float> delta = xl - vec3<float>{cp.x * sc[0], cp.y * sc[1], cp.z * sc[2]};
      d = length(delta) * sg;
      nn = geo_normalize(delta) * sg;
    }
  } else {
    shape_sdf(type, xl, sc, d, nn);
  }
  if (d < margin + r) {
    const int k = atomicAdd(count, 1);
    if (k < cmax) {
      const vec3<float> bp = rot_q(Q, xl - nn * d) + vec3<float>{P.x, P.y, P.z};  // body frame
      const vec3<float> wn = rot_q(Qw, nn);
      particle[k] = i;
      shape[k] = sh.id;
      body_pos[3 * k] = bp.x, body_pos[3 * k + 1] = bp.y, body_pos[3 * k + 2] = bp.z;
      body_vel[3 * k] = body_vel[3 * k + 1] = body_vel[3 * k + 2] = 0.f;
      normal[3 * k] = wn.x, normal[3 * k + 1] = wn.y, normal[3 * k + 2] = wn.z;
    }
  }
}

// The shapes of one launch passed by value as a kernel parameter (read through the constant bank).
constexpr int kParamTableShapes = 16;
struct ShapeParamTable {
  ShapeRec rec[kParamTableShapes];
};

// create_soft_contacts (geometry/kernels.py:1001-1140) over a parameter table: one thread per particle, looping over
// the shapes (the reference launches one thread per (particle, shape); here the shape, hence the branch taken, is
// the same across a warp). WORLDS: some shape belongs to a world (else the world filter can never apply and is
// compiled out); BODIES: some shape is on a body. Four 256-thread CTAs per SM: the loop is latency-bound, and 4
// resident CTAs ran faster than 3.
template <bool WORLDS, bool BODIES>
__global__ void __launch_bounds__(256, 4)
    k_soft_contacts_shapes(int n, const float* __restrict__ q, const float* __restrict__ radius,
                           const int* __restrict__ flags, int S, const ShapeParamTable shapes,
                           const float* __restrict__ elev, const int* __restrict__ particle_world,
                           const float* __restrict__ body_q, float margin, int cmax, int* count, int* particle,
                           int* shape, float* body_pos, float* body_vel, float* normal) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !(flags[i] & 1)) return;
  const vec3<float> x = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};
  const float r = radius[i];
  const int pw = WORLDS && particle_world ? particle_world[i] : -1;
  for (int s = 0; s < S; ++s) {
    if (WORLDS) {  // other world (geometry/kernels.py:1036-1043)
      const int sw = shapes.rec[s].world;
      if (pw != -1 && sw != -1 && pw != sw) continue;
    }
    soft_contact_shape<BODIES>(shapes.rec[s], elev, body_q, x, r, margin, i, cmax, count, particle, shape, body_pos,
                               body_vel, normal);
  }
}

// Host: fills the record of model shape s0 from a VbdShapeTable and checks it, so that every device read the
// record leads to stays in bounds. Returns VBD_OK, VBD_ERR_INVALID_ARGUMENT or VBD_ERR_UNSUPPORTED.
inline int fill_shape_rec(const VbdShapeTable* tb, int s0, ShapeRec& rec) {
  const int t = tb->shape_type_host[s0];
  if (t != GEO_PLANE && t != GEO_SPHERE && t != GEO_CAPSULE && t != GEO_ELLIPSOID && t != GEO_CYLINDER &&
      t != GEO_BOX && t != GEO_CONE && t != GEO_HFIELD && t != GEO_MESH && t != GEO_CONVEX_MESH)
    return VBD_ERR_UNSUPPORTED;
  const float* X = tb->shape_transform_host + 7 * s0;
  const float* sc = tb->shape_scale_host + 3 * s0;
  const float ql = std::sqrt(X[3] * X[3] + X[4] * X[4] + X[5] * X[5] + X[6] * X[6]);
  if (!(ql > 0.f)) return VBD_ERR_INVALID_ARGUMENT;
  rec = ShapeRec();
  rec.type = t;
  rec.id = s0;
  rec.world = tb->shape_world_host ? tb->shape_world_host[s0] : -1;
  rec.body = tb->shape_body_host ? tb->shape_body_host[s0] : -1;
  if (rec.body < -1 || (rec.body >= 0 && rec.body >= tb->body_count)) return VBD_ERR_INVALID_ARGUMENT;
  rec.p = make_float4(X[0], X[1], X[2], 0.f);
  rec.q = make_float4(X[3] / ql, X[4] / ql, X[5] / ql, X[6] / ql);
  rec.sc = make_float4(sc[0], sc[1], sc[2], 0.f);
  if (t == GEO_HFIELD) {  // every grid read of heightfield_sdf stays inside [data_offset, data_offset + nrow ncol)
    if (!tb->shape_heightfield_index_host || !tb->heightfields_host) return VBD_ERR_INVALID_ARGUMENT;
    const int k = tb->shape_heightfield_index_host[s0];
    if (k < 0 || k >= tb->heightfield_count) return VBD_ERR_INVALID_ARGUMENT;
    const VbdHeightfield& h = tb->heightfields_host[k];
    if (h.nrow < 0 || h.ncol < 0 || h.data_offset < 0) return VBD_ERR_INVALID_ARGUMENT;
    if (h.nrow > 1 && h.ncol > 1) {
      if (!tb->elevations_dev || int64_t(h.data_offset) + int64_t(h.nrow) * h.ncol > tb->elevation_count ||
          !(h.hx > 0.f) || !(h.hy > 0.f) || !std::isfinite(h.hx) || !std::isfinite(h.hy))
        return VBD_ERR_INVALID_ARGUMENT;
    }
    rec.hf = make_int4(h.data_offset, h.nrow, h.ncol, 0);
    rec.hfe = make_float4(h.hx, h.hy, h.min_z, h.max_z);
  }
  if (t == GEO_MESH || t == GEO_CONVEX_MESH) {
    if (!tb->shape_mesh_host || !tb->shape_mesh_host[s0]) return VBD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 3; ++k)
      if (!(sc[k] != 0.f) || !std::isfinite(sc[k])) return VBD_ERR_INVALID_ARGUMENT;
    rec.mesh = tb->shape_mesh_host[s0]->view;
  }
  return VBD_OK;
}

}  // namespace vbd
