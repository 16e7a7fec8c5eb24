// vbd_step_noalloc: a cloth VBD step that allocates nothing.
//
// Who needs it: callers that may not call cudaMalloc at all. Examples are a host application
// (engine, simulator, plug-in host) that owns every device allocation through its own pool and
// forbids plug-ins from allocating, and code that steps the cloth while it captures a larger CUDA
// graph, where an allocation inside the captured region would break the capture. vbd_create
// allocates the solver's scratch and packed model, so those callers cannot use it.
//
// This entry point runs the per-color step on the model arrays exactly as the caller holds them
// (the reference layout, plus the reference-layout vertex adjacency that vbd_build_adjacency writes
// into caller-owned buffers). Its per-particle scratch (positions, previous positions, inertial
// targets, contact slots) and an error word live in one file-scope __device__ array, g_noalloc_scratch,
// of fixed size: VBD_NOALLOC_MAX_PARTICLES (32768) particles, 2,097,408 bytes. Every GPU that loads the
// library holds that array until the process exits. The host code gets the array's device address once
// per device with cudaGetSymbolAddress. It does that on the first call made with that device current, so
// make the first call before any stream capture.
//
// All calls on a device share the one array and it keeps the last call's contents. The kernels
// rewrite everything they read before reading it; the contact slots and the error word are cleared at
// the start of every call. Two calls whose kernels overlap on the GPU (different streams, or different
// host threads on the same device) race on the array; serialise them.
//
// Contacts: each particle keeps its VBD_NOALLOC_MAX_CONTACT_SLOTS contacts of lowest index in the
// contact list (a sorted insertion with atomicMin, so the kept set and its order do not depend on
// thread timing); a particle with more sets VBD_DEVERR_CONTACT_OVERFLOW in the error word, which
// vbd_step_noalloc_error reads back, together with the solve's VBD_DEVERR_* bits.
//
// Limits: FP32 only; at most VBD_NOALLOC_MAX_PARTICLES particles; particle-shape contacts on static
// shapes with a fixed penalty (the AVBD ramp rigid_avbd_linear_beta = 0, the reference default). Larger
// models return VBD_ERR_TOO_LARGE before any GPU work.
#include <climits>
#include <mutex>

#include "vbd_b200.h"
#include "vbd_elements.cuh"

using namespace vbd;

namespace {

constexpr int kMaxP = VBD_NOALLOC_MAX_PARTICLES;
constexpr int kSlots = VBD_NOALLOC_MAX_CONTACT_SLOTS;

constexpr int kEmpty = INT_MAX;  // an unused contact slot

struct NoAllocScratch {
  float4 pos[kMaxP];
  float4 qprev[kMaxP];
  float4 inertia[kMaxP];      // w = mass, or 0 for a fixed particle
  int slots[kMaxP * kSlots];  // per particle its kept contact indices in increasing order, kEmpty after
  int err;                    // VBD_DEVERR_* bits of the last call
  int pad_[63];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;
static_assert(sizeof(NoAllocScratch) == 2097408, "scratch size stated in the header");

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_addr[kMaxDevices] = {};

struct NaCtx {
  NoAllocScratch* s;
  int V, S;
  // model, reference layout
  const float* mass;
  const float* inv_mass;
  const int* flags;
  const float* radius;
  const int* tri_indices;
  const float* tri_poses;
  const float* tri_materials;
  const float* tri_areas;
  const int* edge_indices;
  const float* edge_rest_angle;
  const float* edge_rest_length;
  const float* edge_bending;
  const int* face_off;  // two ints per entry
  const int* faces;
  const int* edge_off;
  const int* edges;
  const float* gravity;
  // state
  float* q_in;
  float* q_out;
  const float* qd_in;
  float* qd_out;
  const float* f_ext;
  // contacts
  const int* c_count;
  int c_max;
  const int* c_particle;
  const int* c_shape;
  const float* c_body_pos;
  const float* c_body_vel;
  const float* c_normal;
  float soft_ke, soft_kd, soft_mu;
  const float* shape_ke;
  const float* shape_kd;
  const float* shape_mu;
  float dt, dt2r, fric_eps;
};

__device__ __forceinline__ vec3<float> p3(const float4& a) { return {a.x, a.y, a.z}; }

__global__ void k_na_forward(NaCtx c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.V) return;
  const vec3<float> q = {c.q_in[3 * i], c.q_in[3 * i + 1], c.q_in[3 * i + 2]};
  const int fl = c.flags[i];
  const float m = c.mass[i], im = c.inv_mass[i];
  const float ms = ((fl & 1) && m != 0.f) ? m : 0.f;
  c.s->qprev[i] = make_float4(q.x, q.y, q.z, 0.f);
  static_assert(kSlots == 4, "one int4 store clears a particle's slots");
  reinterpret_cast<int4*>(c.s->slots)[i] = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
  if (i == 0) c.s->err = 0;
  vec3<float> x = q;
  if ((fl & 1) && im != 0.f) {
    vec3<float> fe = {0.f, 0.f, 0.f};
    if (c.f_ext) fe = {c.f_ext[3 * i], c.f_ext[3 * i + 1], c.f_ext[3 * i + 2]};
    const vec3<float> g = {c.gravity[0], c.gravity[1], c.gravity[2]};
    const vec3<float> v = vec3<float>{c.qd_in[3 * i], c.qd_in[3 * i + 1], c.qd_in[3 * i + 2]} + (g + fe * im) * c.dt;
    x = q + v * c.dt;
  }
  c.s->inertia[i] = make_float4(x.x, x.y, x.z, ms);
  c.s->pos[i] = make_float4(x.x, x.y, x.z, 0.f);
}

__global__ void k_na_contacts(NaCtx c) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int count = *c.c_count;
  if (count > c.c_max) count = c.c_max;
  if (t >= count) return;
  const int p = c.c_particle[t], s = c.c_shape[t];
  if (p < 0 || p >= c.V || s < 0 || s >= c.S) {
    atomicOr(&c.s->err, VBD_DEVERR_BAD_CONTACT);
    return;
  }
  // sorted insertion: slot j ends with the smallest index of those that reach it, and the larger one of each
  // exchange moves on to slot j + 1, so the slots end with the kSlots smallest indices in increasing order
  int* slot = c.s->slots + p * kSlots;
  int val = t;
  for (int j = 0; j < kSlots; ++j) {
    const int old = atomicMin(slot + j, val);
    if (old == kEmpty) return;
    val = max(old, val);
  }
  atomicOr(&c.s->err, VBD_DEVERR_CONTACT_OVERFLOW);  // `val` is dropped: the largest index seen here
}

// one thread per vertex of the color; the element math is shared with the main kernels
__global__ void k_na_color(NaCtx c, const int* __restrict__ verts, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int v = verts[k];
  const float4 in4 = c.s->inertia[v];
  const float m = in4.w;
  if (m == 0.f) return;
  vec3<float> f = {0.f, 0.f, 0.f};
  sym3<float> H = szero<float>();
  for (int a = c.face_off[v]; a < c.face_off[v + 1]; a += 2) {
    const int t = c.faces[a], ord = c.faces[a + 1];
    const float mu = c.tri_materials[5 * t], lm = c.tri_materials[5 * t + 1], kd = c.tri_materials[5 * t + 2];
    if (!(mu > 0.f || lm > 0.f)) continue;
    const int* ti = c.tri_indices + 3 * t;
    const float pose[4] = {c.tri_poses[4 * t], c.tri_poses[4 * t + 1], c.tri_poses[4 * t + 2], c.tri_poses[4 * t + 3]};
    vec3<float> xp[3];
    if (kd > 0.f)
      for (int j = 0; j < 3; ++j) xp[j] = p3(c.s->qprev[ti[j]]);
    membrane_add<float>(ord, p3(c.s->pos[ti[0]]), p3(c.s->pos[ti[1]]), p3(c.s->pos[ti[2]]), pose, mu, lm, kd,
                        c.tri_areas[t], c.dt, xp, f, H);
  }
  for (int a = c.edge_off[v]; a < c.edge_off[v + 1]; a += 2) {
    const int e = c.edges[a], ord = c.edges[a + 1];
    const float ke = c.edge_bending[2 * e], kd = c.edge_bending[2 * e + 1];
    if (!(ke > 0.f)) continue;
    const int* ei = c.edge_indices + 4 * e;
    if (ei[0] < 0 || ei[1] < 0) continue;  // boundary hinge: no bending term
    vec3<float> x[4], xp[4];
    for (int j = 0; j < 4; ++j) {
      x[j] = p3(c.s->pos[ei[j]]);
      if (kd > 0.f) xp[j] = p3(c.s->qprev[ei[j]]);
    }
    bending_add<float>(ord, x, c.edge_rest_angle[e], c.edge_rest_length[e], ke, kd, c.dt, xp, f, H);
  }
  const vec3<float> x = p3(c.s->pos[v]);
  const float md = m * c.dt2r;
  f = f + md * (p3(in4) - x);
  H.xx += md;
  H.yy += md;
  H.zz += md;
  const int4 kept = reinterpret_cast<const int4*>(c.s->slots)[v];  // contact index order
  const int ids[kSlots] = {kept.x, kept.y, kept.z, kept.w};
  for (int j = 0; j < kSlots && ids[j] != kEmpty; ++j) {
    const int t = ids[j], s = c.c_shape[t];
    const vec3<float> bx = {c.c_body_pos[3 * t], c.c_body_pos[3 * t + 1], c.c_body_pos[3 * t + 2]};
    const vec3<float> nn = {c.c_normal[3 * t], c.c_normal[3 * t + 1], c.c_normal[3 * t + 2]};
    const float pen = -(dot(nn, x - bx) - c.radius[v]);
    if (pen > 0.f) {
      const vec3<float> bv = {c.c_body_vel[3 * t], c.c_body_vel[3 * t + 1], c.c_body_vel[3 * t + 2]};
      const vec3<float> rel = (x - p3(c.s->qprev[v])) - bv * c.dt;
      const float ke = 0.5f * (c.soft_ke + c.shape_ke[s]);
      const float kd = 0.5f * (c.soft_kd + c.shape_kd[s]);
      const float mu = sqrtf(c.soft_mu * c.shape_mu[s]);
      contact_add<float>(pen, nn, rel, ke, kd, mu, c.fric_eps, c.dt, f, H);
    }
  }
  const float d = sdet(H);
  if (!isfinite(d)) {
    atomicOr(&c.s->err, VBD_DEVERR_NONFINITE);
    return;
  }
  if (!(fabsf(d) > 1e-8f)) {  // the reference skips the update
    atomicOr(&c.s->err, VBD_DEVERR_SINGULAR_SKIPPED);
    return;
  }
  const vec3<float> xn = x + sadj_mul(H, f) * (1.f / d);
  if (isfinite(xn.x) && isfinite(xn.y) && isfinite(xn.z))
    c.s->pos[v] = make_float4(xn.x, xn.y, xn.z, 0.f);
  else
    atomicOr(&c.s->err, VBD_DEVERR_NONFINITE);
}

__global__ void k_na_finalize(NaCtx c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.V) return;
  const vec3<float> p = p3(c.s->pos[i]);
  const vec3<float> v = (p - p3(c.s->qprev[i])) * (1.f / c.dt);
  c.q_in[3 * i] = p.x, c.q_in[3 * i + 1] = p.y, c.q_in[3 * i + 2] = p.z;
  c.q_out[3 * i] = p.x, c.q_out[3 * i + 1] = p.y, c.q_out[3 * i + 2] = p.z;
  c.qd_out[3 * i] = v.x, c.qd_out[3 * i + 1] = v.y, c.qd_out[3 * i + 2] = v.z;
}

// Device address of the scratch array for the current device (cached per device).
int scratch_for_current_device(NoAllocScratch** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return VBD_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return VBD_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return VBD_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<NoAllocScratch*>(p);
  }
  *out = g_scratch_addr[dev];
  return VBD_OK;
}

}  // namespace

extern "C" int vbd_step_noalloc(const VbdModelDesc* m, const VbdRefAdjacency* adj, int32_t iterations,
                                float friction_epsilon, float* q_in, float* q_out, const float* qd_in,
                                float* qd_out, const float* particle_f, const VbdContactsDesc* contacts, float dt,
                                void* stream) {
  if (!m || !adj || !q_in || !q_out || !qd_in || !qd_out || !(dt > 0.f) || iterations < 0)
    return VBD_ERR_INVALID_ARGUMENT;
  if (m->particle_count <= 0 || m->color_count <= 0 || !m->color_offsets_host || !m->color_particles_dev)
    return VBD_ERR_INVALID_ARGUMENT;
  if (m->spring_count != 0 || m->tet_count != 0) return VBD_ERR_UNSUPPORTED;
  if (m->particle_count > kMaxP) return VBD_ERR_TOO_LARGE;
  if (!adj->face_offsets_dev || !adj->edge_offsets_dev || (m->tri_count > 0 && !adj->faces_dev) ||
      (m->edge_count > 0 && !adj->edges_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  if (m->color_offsets_host[0] != 0 || m->color_offsets_host[m->color_count] != m->particle_count)
    return VBD_ERR_INVALID_ARGUMENT;
  const bool has_c = contacts && contacts->soft_contact_max > 0 && contacts->soft_contact_count_dev &&
                     m->shape_count > 0;
  if (has_c && (!m->shape_material_ke_dev || !m->shape_material_kd_dev || !m->shape_material_mu_dev ||
                !contacts->soft_contact_particle_dev || !contacts->soft_contact_shape_dev ||
                !contacts->soft_contact_body_pos_dev || !contacts->soft_contact_body_vel_dev ||
                !contacts->soft_contact_normal_dev))
    return VBD_ERR_INVALID_ARGUMENT;
  NoAllocScratch* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != VBD_OK) return rc;
  NaCtx c{};
  c.s = scratch;
  c.V = m->particle_count;
  c.S = m->shape_count;
  c.mass = m->particle_mass_dev;
  c.inv_mass = m->particle_inv_mass_dev;
  c.flags = m->particle_flags_dev;
  c.radius = m->particle_radius_dev;
  c.tri_indices = m->tri_indices_dev;
  c.tri_poses = m->tri_poses_dev;
  c.tri_materials = m->tri_materials_dev;
  c.tri_areas = m->tri_areas_dev;
  c.edge_indices = m->edge_indices_dev;
  c.edge_rest_angle = m->edge_rest_angle_dev;
  c.edge_rest_length = m->edge_rest_length_dev;
  c.edge_bending = m->edge_bending_properties_dev;
  c.face_off = adj->face_offsets_dev;
  c.faces = adj->faces_dev;
  c.edge_off = adj->edge_offsets_dev;
  c.edges = adj->edges_dev;
  c.gravity = m->gravity_dev;
  c.q_in = q_in;
  c.q_out = q_out;
  c.qd_in = qd_in;
  c.qd_out = qd_out;
  c.f_ext = particle_f;
  c.soft_ke = m->soft_contact_ke;
  c.soft_kd = m->soft_contact_kd;
  c.soft_mu = m->soft_contact_mu;
  c.shape_ke = m->shape_material_ke_dev;
  c.shape_kd = m->shape_material_kd_dev;
  c.shape_mu = m->shape_material_mu_dev;
  c.dt = dt;
  c.dt2r = 1.f / (dt * dt);
  c.fric_eps = friction_epsilon;
  if (has_c) {
    c.c_count = contacts->soft_contact_count_dev;
    c.c_max = contacts->soft_contact_max;
    c.c_particle = contacts->soft_contact_particle_dev;
    c.c_shape = contacts->soft_contact_shape_dev;
    c.c_body_pos = contacts->soft_contact_body_pos_dev;
    c.c_body_vel = contacts->soft_contact_body_vel_dev;
    c.c_normal = contacts->soft_contact_normal_dev;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int V = c.V;
  k_na_forward<<<(V + 255) / 256, 256, 0, st>>>(c);  // also clears the contact slots and the error word
  if (has_c) k_na_contacts<<<(c.c_max + 255) / 256, 256, 0, st>>>(c);
  for (int it = 0; it < iterations; ++it)
    for (int col = 0; col < m->color_count; ++col) {
      const int a = m->color_offsets_host[col], b = m->color_offsets_host[col + 1];
      if (b > a) k_na_color<<<(b - a + 127) / 128, 128, 0, st>>>(c, m->color_particles_dev + a, b - a);
    }
  k_na_finalize<<<(V + 255) / 256, 256, 0, st>>>(c);
  return cudaGetLastError() == cudaSuccess ? VBD_OK : VBD_ERR_CUDA;
}

extern "C" int vbd_step_noalloc_error(int32_t* bits, void* stream) {
  if (!bits) return VBD_ERR_INVALID_ARGUMENT;
  NoAllocScratch* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != VBD_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int value = 0;
  if (cudaMemcpyAsync(&value, &scratch->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return VBD_ERR_CUDA;
  *bits = value;
  return VBD_OK;
}
