// Device math of particle self-contact (vertex-triangle and edge-edge), templated on the real type.
//
// Reference (newton/_src/solvers/vbd/particle_vbd_kernels.py unless noted):
//   barrier               evaluate_self_contact_force_norm :1193-1222
//   damping               damp_collision :1225-1238
//   edge-edge term        evaluate_edge_edge_contact_2_vertices :1371-1506
//   vertex-triangle term  evaluate_vertex_triangle_collision_force_hessian_4_vertices :1599-1745
//   friction              compute_friction :1748-1779, math/__init__.py orthonormal_basis
//   division planes       segment_plane_intersects, create_vertex_triangle_division_plane_closest_pt,
//                         robust_edge_pair_normal, create_edge_edge_division_plane_closest_pt,
//                         planar_truncation_t :2475-2741
//   closest points        geometry/kernels.py triangle_closest_point :64-128; the edge-edge closest points
//                         come from Warp's native closest_point_edge_edge, which is not in the reference tree:
//                         restated here from the published segment-segment method (C. Ericson, Real-Time
//                         Collision Detection, 2005, sec. 5.1.9), eps bounding squared lengths of degenerate
//                         segments, exactly parallel segments taking s = 0.
//
// The reference evaluates a pair once and scatters its four (or two) vertex terms with atomics. Here
// the solve of each vertex gathers the pairs it belongs to and evaluates the term of its own slot in
// the pair, so a vertex's sum has a fixed order and no atomics are needed.
#pragma once
#include "vbd_math.cuh"

namespace vbd {

template <typename R> __host__ __device__ __forceinline__ R vclamp(R x, R lo, R hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Closest point on triangle (a, b, c) to p and its barycentric weights, with the reference's branch order
// (vertex regions A, B, C, then edges AB, AC, BC, then the interior).
template <typename R>
__host__ __device__ __forceinline__ vec3<R> tri_closest(vec3<R> a, vec3<R> b, vec3<R> c, vec3<R> p, R bary[3]) {
  const vec3<R> ab = b - a, ac = c - a, ap = p - a;
  const R d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= R(0) && d2 <= R(0)) {
    bary[0] = R(1), bary[1] = R(0), bary[2] = R(0);
    return a;
  }
  const vec3<R> bp = p - b;
  const R d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= R(0) && d4 <= d3) {
    bary[0] = R(0), bary[1] = R(1), bary[2] = R(0);
    return b;
  }
  const vec3<R> cp = p - c;
  const R d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= R(0) && d5 <= d6) {
    bary[0] = R(0), bary[1] = R(0), bary[2] = R(1);
    return c;
  }
  const R vc = d1 * d4 - d3 * d2;
  if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) {
    const R v = d1 / (d1 - d3);
    bary[0] = R(1) - v, bary[1] = v, bary[2] = R(0);
    return a + v * ab;
  }
  const R vb = d5 * d2 - d1 * d6;
  if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) {
    const R v = d2 / (d2 - d6);
    bary[0] = R(1) - v, bary[1] = R(0), bary[2] = v;
    return a + v * ac;
  }
  const R va = d3 * d6 - d5 * d4;
  if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) {
    const R v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    bary[0] = R(0), bary[1] = R(1) - v, bary[2] = v;
    return b + v * (c - b);
  }
  const R denom = R(1) / (va + vb + vc);
  const R v = vb * denom, w = vc * denom;
  bary[0] = R(1) - v - w, bary[1] = v, bary[2] = w;
  return a + v * ab + w * ac;
}

// Closest points of segments p1-q1 and p2-q2: parameters s, t and the distance.
template <typename R>
__host__ __device__ __forceinline__ void edge_closest(vec3<R> p1, vec3<R> q1, vec3<R> p2, vec3<R> q2, R eps, R& s, R& t,
                                                      R& dist) {
  const vec3<R> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
  const R a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  if (a <= eps && e <= eps) {
    s = t = R(0);
  } else if (a <= eps) {
    s = R(0);
    t = vclamp(f / e, R(0), R(1));
  } else {
    const R c = dot(d1, r);
    if (e <= eps) {
      t = R(0);
      s = vclamp(-c / a, R(0), R(1));
    } else {
      const R b = dot(d1, d2);
      const R denom = a * e - b * b;
      s = denom != R(0) ? vclamp((b * f - c * e) / denom, R(0), R(1)) : R(0);
      t = (b * s + f) / e;
      if (t < R(0)) {
        t = R(0);
        s = vclamp(-c / a, R(0), R(1));
      } else if (t > R(1)) {
        t = R(1);
        s = vclamp((b - c) / a, R(0), R(1));
      }
    }
  }
  dist = length((p1 + d1 * s) - (p2 + d2 * t));
}

// Tangent basis of a unit normal (orthonormal_basis).
template <typename R>
__host__ __device__ __forceinline__ void onb(vec3<R> n, vec3<R>& b1, vec3<R>& b2) {
  if (n.z < R(0)) {
    const R a = R(1) / (R(1) - n.z), b = n.x * n.y * a;
    b1 = {R(1) - n.x * n.x * a, -b, n.x};
    b2 = {b, n.y * n.y * a - R(1), -n.y};
  } else {
    const R a = R(1) / (R(1) + n.z), b = -n.x * n.y * a;
    b1 = {R(1) - n.x * n.x * a, b, -n.x};
    b2 = {b, R(1) - n.y * n.y * a, -n.y};
  }
}

// dE/dd and d2E/dd2 of the barrier: linear k (r - d) for d >= r/2, log barrier below, quadratic below 1e-5.
template <typename R>
__host__ __device__ __forceinline__ void sc_norm(R dis, R radius, R k, R& dEdD, R& d2E) {
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

// Force and Hessian of one slot of a contact: normal barrier scaled by the slot's weight w, damping when
// the slot moved towards the other side since the start of the step (disp . (sgn n) > 0), and w times
// the tangential friction (ff, fH). Adds to (f, H).
template <typename R>
__host__ __device__ __forceinline__ void sc_slot_add(R w, R sgn, vec3<R> n, R dEdD, R d2E, vec3<R> disp, vec3<R> ff,
                                                     const sym3<R>& fH, R kd_over_dt, vec3<R>& f, sym3<R>& H) {
  const R hn = d2E * w * w;
  vec3<R> fk = (-dEdD * n) * w;
  sym3<R> Hk = souter(n, hn);
  if (dot(disp, n * sgn) > R(0)) {
    const R dn = kd_over_dt * hn * dot(n, disp);  // (kd/dt) H_k disp with H_k = hn n n^T
    fk = fk + n * dn;
    Hk = Hk + kd_over_dt * Hk;
  }
  f = f + fk + ff * w;
  H = H + Hk + (w * w) * fH;
}

// IPC-regularised friction of a contact with unit normal n, normal force fn and relative tangential
// displacement dx (compute_friction with T = [b1 b2]).
template <typename R>
__host__ __device__ __forceinline__ void sc_friction(R mu, R fn, vec3<R> n, vec3<R> dx, R eps_u, vec3<R>& ff, sym3<R>& fH) {
  vec3<R> b1, b2;
  onb(n, b1, b2);
  const R u0 = dot(b1, dx), u1 = dot(b2, dx);
  const R un = vsqrt(u0 * u0 + u1 * u1);
  if (un > R(0)) {
    const R f1 = un > eps_u ? R(1) / un : (-un / eps_u + R(2)) / eps_u;
    ff = (-mu * fn) * ((f1 * u0) * b1 + (f1 * u1) * b2);
    const R s = mu * fn * f1;
    fH = souter(b1, s);
    souter_add(fH, b2, s);
  } else {
    ff = zero3<R>();
    fH = szero<R>();
  }
}

// Vertex-triangle pair, x = (a, b, c, p) current and xa at the start of the step. Adds the term of slot
// `order` (0..2: triangle vertex, 3: the colliding vertex). Returns false when the pair is not in contact.
template <typename R>
__device__ __forceinline__ bool sc_vt_add(int order, const vec3<R> x[4], const vec3<R> xa[4], R radius, R ke, R kd, R mu,
                                          R eps_u, R dt, vec3<R>& f, sym3<R>& H) {
  R bary[3];
  const vec3<R> cp = tri_closest(x[0], x[1], x[2], x[3], bary);
  const vec3<R> diff = x[3] - cp;
  const R dis = length(diff);
  if (!(R(0) < dis && dis < radius)) return false;
  const vec3<R> n = diff * (R(1) / dis);
  R dEdD, d2E;
  sc_norm(dis, radius, ke, dEdD, d2E);
  const vec3<R> cpp = bary[0] * xa[0] + bary[1] * xa[1] + bary[2] * xa[2];
  const vec3<R> dx = (x[3] - xa[3]) - (cp - cpp);
  vec3<R> ff;
  sym3<R> fH;
  sc_friction(mu, -dEdD, n, dx, eps_u, ff, fH);
  // the slot's weight and displacement picked with selects (no dynamic indexing of local arrays)
  const R w = order == 3 ? R(1) : -(order == 0 ? bary[0] : (order == 1 ? bary[1] : bary[2]));
  const R sgn = order == 3 ? R(1) : R(-1);
  const vec3<R> disp = order == 0 ? xa[0] - x[0] : (order == 1 ? xa[1] - x[1] : (order == 2 ? xa[2] - x[2] : xa[3] - x[3]));
  sc_slot_add(w, sgn, n, dEdD, d2E, disp, ff, fH, kd / dt, f, H);
  return true;
}

// Edge-edge pair, x = (e1.v0, e1.v1, e2.v0, e2.v1). Adds the term of e1's vertex `order` (0 or 1).
template <typename R>
__device__ __forceinline__ bool sc_ee_add(int order, const vec3<R> x[4], const vec3<R> xa[4], R radius, R ke, R kd, R mu,
                                          R eps_u, R dt, R ee_eps, vec3<R>& f, sym3<R>& H) {
  R s, t, dis;
  edge_closest(x[0], x[1], x[2], x[3], ee_eps, s, t, dis);
  if (!(R(0) < dis && dis < radius)) return false;
  const vec3<R> c1 = x[0] + (x[1] - x[0]) * s, c2 = x[2] + (x[3] - x[2]) * t;
  const vec3<R> n = (c1 - c2) * (R(1) / dis);
  R dEdD, d2E;
  sc_norm(dis, radius, ke, dEdD, d2E);
  const vec3<R> c1p = xa[0] + (xa[1] - xa[0]) * s, c2p = xa[2] + (xa[3] - xa[2]) * t;
  const vec3<R> dx = (c1 - c1p) - (c2 - c2p);
  vec3<R> ff;
  sym3<R> fH;
  sc_friction(mu, -dEdD, n, dx, eps_u, ff, fH);
  const R w = order == 0 ? R(1) - s : s;
  const vec3<R> disp = order == 0 ? xa[0] - x[0] : xa[1] - x[1];
  sc_slot_add(w, R(1), n, dEdD, d2E, disp, ff, fH, kd / dt, f, H);
  return true;
}

// ------------------------------------------------------------------------------- division planes
template <typename R>
__host__ __device__ __forceinline__ bool seg_plane(vec3<R> v, vec3<R> dv, vec3<R> n, vec3<R> d, R eps_par, R near, R far) {
  const R nv = dot(n, dv), num = -dot(n, v - d);
  if (vabs(nv) < eps_par) return false;  // coplanar segments do not count here
  const R t = num / nv;
  return t >= near && t <= R(1) + far;
}

template <typename R> __host__ __device__ __forceinline__ vec3<R> vnormalize(vec3<R> a) {
  const R l = length(a);
  return l > R(0) ? a * (R(1) / l) : zero3<R>();
}

// Plane between a vertex and a triangle: x = (v, t1, t2, t3), dx their displacements since the last
// detection. cut[k] = the plane bounds vertex k's step.
template <typename R>
__host__ __device__ __forceinline__ void vt_plane(const vec3<R> x[4], const vec3<R> dx[4], bool cut[4], vec3<R>& n,
                                                  vec3<R>& d) {
  R bary[3];
  const vec3<R> cp = tri_closest(x[1], x[2], x[3], x[0], bary);
  const vec3<R> nh = x[0] - cp;
  if (length(nh) < R(1e-12)) {
    for (int k = 0; k < 4; ++k) cut[k] = true;  // zero normal: the step fraction comes out as 1
    n = zero3<R>();
    d = x[0];
    return;
  }
  n = vnormalize(nh);
  const R dvn = vmax(-dot(n, dx[0]), R(0));
  const R dtn = vmax(vmax(dot(n, dx[1]), dot(n, dx[2])), vmax(dot(n, dx[3]), R(0)));
  if (dtn + dvn == R(0)) {
    d = cp + R(0.5) * nh;
  } else {
    const R l = vclamp(dtn / (dtn + dvn), R(0.05), R(0.95));
    d = cp + l * nh;
  }
  cut[0] = dvn == R(0) ? false : seg_plane(x[0], dx[0], n, d, R(1e-6), R(-1e-8), R(1e-8));
  for (int k = 1; k < 4; ++k) cut[k] = dtn == R(0) ? false : seg_plane(x[k], dx[k], n, d, R(1e-6), R(-1e-8), R(1e-8));
}

template <typename R>
__host__ __device__ __forceinline__ vec3<R> robust_pair_normal(vec3<R> a0, vec3<R> a1, vec3<R> b0, vec3<R> b1) {
  const R eps = R(1e-6);
  vec3<R> d0 = a1 - a0, d1 = b1 - b0;
  const R l0 = length(d0), l1 = length(d1);
  d0 = l0 > eps ? d0 * (R(1) / l0) : zero3<R>();
  d1 = l1 > eps ? d1 * (R(1) / l1) : zero3<R>();
  vec3<R> n = cross(d0, d1);
  R ln = length(n);
  if (ln > eps) return n * (R(1) / ln);
  vec3<R> ref = d0;
  if (length(ref) <= eps) ref = d1;
  if (length(ref) <= eps) return {R(1), R(0), R(0)};
  const vec3<R> bridge = R(0.5) * ((b0 + b1) - (a0 + a1));
  const R bl = length(bridge);
  if (bl > eps) {
    n = cross(ref, bridge * (R(1) / bl));
    ln = length(n);
    if (ln > eps) return n * (R(1) / ln);
  }
  vec3<R> axis = {R(1), R(0), R(0)};
  if (vabs(dot(ref, axis)) > R(0.9)) axis = {R(0), R(1), R(0)};
  n = cross(ref, axis);
  ln = length(n);
  if (ln > eps) return n * (R(1) / ln);
  n = cross(ref, vec3<R>{R(0), R(0), R(1)});
  ln = length(n);
  if (ln > eps) return n * (R(1) / ln);
  return {R(1), R(0), R(0)};
}

// Plane between two edges: x = (e0.v0, e0.v1, e1.v0, e1.v1).
template <typename R>
__host__ __device__ __forceinline__ void ee_plane(const vec3<R> x[4], const vec3<R> dx[4], bool cut[4], vec3<R>& n,
                                                  vec3<R>& d) {
  R s, t, dist;
  edge_closest(x[0], x[1], x[2], x[3], R(1e-6), s, t, dist);
  const vec3<R> c1 = x[0] + (x[1] - x[0]) * s, c2 = x[2] + (x[3] - x[2]) * t;
  const vec3<R> nh = c1 - c2;
  if (length(nh) < R(1e-12)) {
    for (int k = 0; k < 4; ++k) cut[k] = true;
    n = robust_pair_normal(x[0], x[1], x[2], x[3]);
    d = c1 * R(0.5) + c2 * R(0.5);
    return;
  }
  n = vnormalize(nh);
  const R de0 = vmax(vmax(-dot(n, dx[0]), -dot(n, dx[1])), R(0));
  const R de1 = vmax(vmax(dot(n, dx[2]), dot(n, dx[3])), R(0));
  if (de0 + de1 == R(0)) {
    d = c2 + R(0.5) * nh;
  } else {
    const R l = vclamp(de1 / (de1 + de0), R(0.05), R(0.95));
    d = c2 + l * nh;
  }
  for (int k = 0; k < 2; ++k) cut[k] = de0 == R(0) ? false : seg_plane(x[k], dx[k], n, d, R(1e-6), R(-1e-8), R(1e-6));
  for (int k = 2; k < 4; ++k) cut[k] = de1 == R(0) ? false : seg_plane(x[k], dx[k], n, d, R(1e-6), R(-1e-8), R(1e-6));
}

// Fraction of the step dv from v that stays gamma short of the plane (n, d); 1 when the step does not
// cross it.
template <typename R>
__host__ __device__ __forceinline__ R plane_t(vec3<R> v, vec3<R> dv, vec3<R> n, vec3<R> d, R eps, R gamma) {
  const R den = dot(n, dv);
  if (vabs(den) < eps) return R(1);
  const R t = dot(n, d - v) / den;
  if (t < R(0)) return R(1);
  return vclamp(vmin(t * gamma, t - R(1e-3)), R(0), R(1));
}

}  // namespace vbd
