// Triangle-mesh shapes for particle contacts: the closest point on a static mesh within a search radius and the
// inside/outside sign, as create_soft_contacts asks of wp.mesh_query_point_sign_normal for GeoType.MESH and
// CONVEX_MESH (geometry/kernels.py:1091-1113). Warp's mesh query is native code outside the reference tree; this
// restates its documented behaviour: the closest point over all triangles, found through a bounding-volume
// hierarchy, and the sign from the angle-weighted pseudo-normal of the closest feature (J. A. Baerentzen and
// H. Aanaes, "Signed distance computation using the angle weighted pseudonormal", IEEE TVCG 11(3), 2005): the
// face normal inside a triangle, the sum of the adjacent face normals on an edge, the incident face normals
// weighted by their angles at a vertex.
#pragma once
#include "vbd_selfcontact.cuh"

namespace vbd {

// Internal node of the hierarchy: the boxes of both children, so that one node read decides both descents.
// child >= 0 is another internal node, child < 0 the leaf triangle ~child.
struct MeshBvhNode {
  float4 lo[2];
  float4 hi[2];
  int child[2];
  int pad[2];
};

struct MeshView {
  const MeshBvhNode* nodes;  // tri_count - 1 internal nodes, root 0 (none for a single triangle)
  const float4* pts;         // vertices (x, y, z, 0), mesh frame, unscaled
  const int4* tris;          // (i, j, k, 0)
  const float4* fn;          // unit face normals
  const float4* en;          // per triangle, pseudo-normals of its edges AB, AC, BC
  const float4* vn;          // angle-weighted vertex pseudo-normals
  int tri_count;
  int pad;
};

constexpr int kMeshStack = 64;  // the hierarchy is split at the median: depth <= ceil(log2 tri_count) < 32

__device__ __forceinline__ vec3<float> f3(float4 a) { return {a.x, a.y, a.z}; }

__device__ __forceinline__ float box_dist2(float4 lo, float4 hi, vec3<float> p) {
  const float dx = fmaxf(fmaxf(lo.x - p.x, p.x - hi.x), 0.f);
  const float dy = fmaxf(fmaxf(lo.y - p.y, p.y - hi.y), 0.f);
  const float dz = fmaxf(fmaxf(lo.z - p.z, p.z - hi.z), 0.f);
  return dx * dx + dy * dy + dz * dz;
}

// Closest point of mesh m to p closer than max_dist: returns false when there is none. On success cp is the
// closest point, sign -1 inside and +1 outside (the pseudo-normal test), face the triangle. A push beyond
// kMeshStack entries is dropped rather than written out of bounds; a median-split hierarchy never needs one.
__device__ __forceinline__ bool mesh_query_point_sign(const MeshView& m, vec3<float> p, float max_dist,
                                                      vec3<float>& cp, float& sign, int& face) {
  float best = max_dist * max_dist;
  int bt = -1;
  float bb[3] = {0.f, 0.f, 0.f};
  auto leaf = [&](int t) {
    const int4 f = __ldg(&m.tris[t]);
    float w[3];
    const vec3<float> c = tri_closest(f3(__ldg(&m.pts[f.x])), f3(__ldg(&m.pts[f.y])), f3(__ldg(&m.pts[f.z])), p, w);
    const vec3<float> d = c - p;
    const float d2 = dot(d, d);
    if (d2 < best) {
      best = d2, bt = t, cp = c;
      bb[0] = w[0], bb[1] = w[1], bb[2] = w[2];
    }
  };
  if (m.tri_count == 1) {
    leaf(0);
  } else if (m.tri_count > 1) {
    int stack[kMeshStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const MeshBvhNode& nd = m.nodes[stack[--sp]];
      const float d0 = box_dist2(nd.lo[0], nd.hi[0], p), d1 = box_dist2(nd.lo[1], nd.hi[1], p);
      const int near = d1 < d0 ? 1 : 0;
      const float dn = near ? d1 : d0, df = near ? d0 : d1;
      const int cn = nd.child[near], cf = nd.child[1 - near];
      // leaves are evaluated at once (nearer first); internal children are pushed farther first
      if (dn < best && cn < 0) leaf(~cn);
      if (df < best && cf < 0) leaf(~cf);
      if (df < best && cf >= 0 && sp < kMeshStack) stack[sp++] = cf;
      if (dn < best && cn >= 0 && sp < kMeshStack) stack[sp++] = cn;
    }
  }
  if (bt < 0) return false;
  // the closest feature from the barycentric weights: two zero weights = a vertex, one = an edge
  vec3<float> pn;
  const int4 f = __ldg(&m.tris[bt]);
  const int zeros = (bb[0] == 0.f) + (bb[1] == 0.f) + (bb[2] == 0.f);
  if (zeros >= 2) {
    pn = f3(__ldg(&m.vn[bb[0] != 0.f ? f.x : (bb[1] != 0.f ? f.y : f.z)]));
  } else if (zeros == 1) {
    pn = f3(__ldg(&m.en[3 * bt + (bb[2] == 0.f ? 0 : (bb[1] == 0.f ? 1 : 2))]));
  } else {
    pn = f3(__ldg(&m.fn[bt]));
  }
  sign = dot(p - cp, pn) < 0.f ? -1.f : 1.f;
  face = bt;
  return true;
}

}  // namespace vbd

// A static triangle mesh on the device (the handle behind VbdMeshHandle): one allocation holding the hierarchy,
// vertices, triangles and pseudo-normals that `view` points into.
struct VbdMeshImpl {
  vbd::MeshView view;
  void* buffer;
  int point_count;
};
