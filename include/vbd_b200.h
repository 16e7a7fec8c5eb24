/* C ABI of the B200 cloth Vertex Block Descent library (libvbd_b200.so).
 *
 * Drop-in boundary for the particle path of newton.solvers.SolverVBD (reference project
 * caixiao-0725/newton-ChysX). Every pointer named *_dev is CUDA device memory in the reference's
 * Model / State / Contacts layout (float32 vec3 = 3 packed floats, int32 indices); *_host is host
 * memory. Functions return VBD_OK (0) or a negative VBD_ERR_* code and never abort the process.
 * No function allocates device memory after vbd_create returns, so vbd_step can be captured in a
 * CUDA graph on the caller's stream.
 */
#ifndef VBD_B200_H
#define VBD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VBD_OK 0
#define VBD_ERR_INVALID_ARGUMENT -1
#define VBD_ERR_CUDA -2
#define VBD_ERR_OUT_OF_MEMORY -3
#define VBD_ERR_UNSUPPORTED -4
#define VBD_ERR_EMPTY_COLORING -5
#define VBD_ERR_TOO_LARGE -6 /* vbd_step_noalloc: the model exceeds its fixed scratch */

/* Bits of the device-side error word (vbd_get_error). Kernels set bits instead of trapping. */
#define VBD_DEVERR_NONFINITE 1          /* a solved displacement was NaN/Inf (position left unchanged) */
#define VBD_DEVERR_CONTACT_OVERFLOW 2   /* more contacts on one particle than contact slots */
#define VBD_DEVERR_SINGULAR_SKIPPED 4   /* |det H| <= 1e-8: update skipped, as the reference does */
#define VBD_DEVERR_BAD_CONTACT 8        /* a contact names a particle or shape out of range (ignored) */

/* Arithmetic of vbd_step. */
#define VBD_PRECISION_FP32 0   /* FP32 throughout: the reference's arithmetic */
#define VBD_PRECISION_MIXED 1  /* FP32 element math, FP64 3x3 solve below a conditioning threshold,
                                  FP64 residual reductions */
#define VBD_PRECISION_FP64 2   /* FP64 throughout (state in float64): the FP64 reference run */

/* Scheduling of the per-color sweep. */
#define VBD_SCHEDULE_AUTO 0
#define VBD_SCHEDULE_PER_COLOR 1   /* one grid launch per color per iteration (large single cloth) */
#define VBD_SCHEDULE_PERSISTENT 2  /* one launch per substep; one CTA owns one instance (world) at a time */

/* Element data layout read by the sweep. */
#define VBD_LAYOUT_AUTO 0
#define VBD_LAYOUT_CSR 1  /* vertex -> element adjacency, element records gathered by id (any lanes/vertex) */
#define VBD_LAYOUT_ELL 2  /* per-incidence stencil records in sweep order, slot-major (one lane/vertex) */
#define VBD_LAYOUT_ELL16 3 /* the same with 16-bit instance-local vertex ids: 32-byte face and 16-byte hinge
                              records (persistent schedule, instances below 65536 particles); hinge damping,
                              when the model has some, in a side array read by a kernel variant of its own */
#define VBD_LAYOUT_RING 4  /* one-ring fan records (16-bit instance-local ids): each vertex walks its fan once,
                              sharing every incident face normal between the membrane, the two spoke hinges and
                              the rim hinge of that face (persistent schedule, instances below 65536 particles,
                              manifold fans of at most 8 triangles); a damped hinge is evaluated on its own */

typedef struct VbdModelDesc {
  int32_t particle_count; /* V */
  int32_t tri_count;      /* T */
  int32_t edge_count;     /* E */
  int32_t shape_count;    /* S */
  /* particles (Model.particle_*) */
  const float* particle_mass_dev;     /* [V] */
  const float* particle_inv_mass_dev; /* [V] */
  const int32_t* particle_flags_dev;  /* [V], bit 0 = ParticleFlags.ACTIVE */
  const float* particle_radius_dev;   /* [V] */
  /* triangles (Model.tri_*) */
  const int32_t* tri_indices_dev;  /* [T,3] */
  const float* tri_poses_dev;      /* [T,2,2] rest D^-1, row-major */
  const float* tri_materials_dev;  /* [T,5]: mu, lambda, damping, drag, lift (first three read) */
  const float* tri_areas_dev;      /* [T] */
  /* bending hinges (Model.edge_*) */
  const int32_t* edge_indices_dev;         /* [E,4]: o0, o1, v0, v1 (-1 = no opposite vertex) */
  const float* edge_rest_angle_dev;        /* [E] */
  const float* edge_rest_length_dev;       /* [E] */
  const float* edge_bending_properties_dev;/* [E,2]: ke, kd */
  /* coloring (Model.particle_color_groups, concatenated in sweep order) */
  int32_t color_count;
  const int32_t* color_offsets_host;   /* [color_count+1] */
  const int32_t* color_particles_dev;  /* [V] */
  /* worlds: particles of world w are [world_particle_start_host[w], world_particle_start_host[w+1]).
     world_count <= 1 means one instance. Instances must not share triangles or hinges. */
  int32_t world_count;
  const int32_t* world_particle_start_host; /* [world_count+1] or NULL */
  /* gravity: Model.gravity[0] (the reference VBD reads world 0 only) */
  const float* gravity_dev; /* [3] */
  /* particle-shape contact materials */
  float soft_contact_ke, soft_contact_kd, soft_contact_mu; /* Model.soft_contact_* */
  const float* shape_material_ke_dev; /* [S] */
  const float* shape_material_kd_dev; /* [S] */
  const float* shape_material_mu_dev; /* [S] */
  const int32_t* shape_body_dev;      /* [S], -1 = static */
  const float* body_com_dev;          /* [B,3] or NULL */
  /* springs (Model.spring_*; spring_count 0 = none). Forces on both ends, as
     evaluate_spring_force_and_hessian_both_vertices (particle_vbd_kernels.py:2299-2343). The reference's
     coloring leaves springs out: a spring whose ends share a color is summed before that color's solve from
     the positions before it (accumulate_spring_force_and_hessian, :2347-2397), as the reference does. */
  int32_t spring_count;
  const int32_t* spring_indices_dev;   /* [2*spring_count]: end 0, end 1 */
  const float* spring_rest_length_dev; /* [spring_count] */
  const float* spring_stiffness_dev;   /* [spring_count] */
  const float* spring_damping_dev;     /* [spring_count] */
  /* tetrahedra (Model.tet_*; tet_count 0 = none): volumetric stable Neo-Hookean
     (evaluate_volumetric_neo_hookean_force_and_hessian, particle_vbd_kernels.py:335-473) */
  int32_t tet_count;
  const int32_t* tet_indices_dev;   /* [N,4] */
  const float* tet_poses_dev;       /* [N,3,3] rest D^-1, row-major */
  const float* tet_materials_dev;   /* [N,3]: mu, lambda, damping */
} VbdModelDesc;

typedef struct VbdSolverParams {
  int32_t iterations;           /* SolverVBD(iterations=10) */
  float friction_epsilon;       /* SolverVBD(friction_epsilon=1e-2) */
  float avbd_linear_beta;       /* rigid_avbd_linear_beta (0 = fixed penalty k) */
  float contact_k_start;        /* rigid_contact_k_start (seed when beta > 0) */
  int32_t precision;            /* VBD_PRECISION_* */
  float fp64_solve_threshold;   /* MIXED: FP64 solve when |det H| < thr * max|H_ij|^3 */
  int32_t schedule;             /* VBD_SCHEDULE_* */
  int32_t lanes_per_vertex;     /* 1,2,4,8,16,32; 0 = choose */
  int32_t block_size;           /* threads per CTA; 0 = choose */
  int32_t contact_slots;        /* contacts kept per particle; 0 = max(shape_count, 1) */
  int32_t positions_in_shared;  /* persistent schedule, FP32/MIXED: keep each instance's positions in
                                   shared memory during the sweep. 0 = when they fit, 1 = never,
                                   2 = required (VBD_ERR_UNSUPPORTED if they do not fit) */
  int32_t layout;               /* VBD_LAYOUT_*; AUTO = ELL16 where it applies, else ELL when lanes_per_vertex is 1 */
  int32_t min_blocks_per_sm;    /* ELL + persistent, FP32/MIXED: 2..4 compiles the kernel for that many
                                   resident CTAs of 256 threads per SM (fewer registers); 0 = none */
  int32_t pair_vertices;        /* ELL16 + persistent, FP32: 1 = each thread solves two vertices of a color at
                                   once, one per lane of the paired FP32 instructions (FFMA2/FADD2/FMUL2);
                                   0 = one vertex per thread */
  int32_t instance_per_warp;    /* persistent schedule, CSR layout, lanes_per_vertex 1..8: 1 = each warp takes
                                   instances from the work queue on its own (colors separated by __syncwarp, eight
                                   instances side by side in a CTA of 256; positions in shared memory per warp when
                                   they fit), for batches of small instances; 0 = one instance per CTA */
} VbdSolverParams;

typedef struct VbdContactsDesc {
  const int32_t* soft_contact_count_dev; /* [1] */
  int32_t soft_contact_max;
  const int32_t* soft_contact_particle_dev; /* [max] */
  const int32_t* soft_contact_shape_dev;    /* [max] */
  const float* soft_contact_body_pos_dev;   /* [max,3] */
  const float* soft_contact_body_vel_dev;   /* [max,3] */
  const float* soft_contact_normal_dev;     /* [max,3] */
} VbdContactsDesc;

typedef struct VbdBodyState {
  /* rigid body poses for particle-shape contacts on bodies (NULL when every shape is static).
     body_q: [B,7] (p, quat xyzw); body_qd: [B,6] (linear, angular); body_q_prev: [B,7] or NULL. */
  const float* body_q_dev;
  const float* body_q_prev_dev;
  const float* body_qd_dev;
} VbdBodyState;

typedef struct VbdSolver* VbdHandle;

/* Replaces SolverVBD.__init__ (solver_vbd.py:196-541): builds the vertex->element adjacency
   (particle_vbd_kernels.py:639-738 fill order, solver_vbd.py:1177-1337), packs the model for the
   kernels and allocates all solver scratch. Returns VBD_ERR_EMPTY_COLORING like the reference's
   ValueError (solver_vbd.py:533-537). Models with springs or tetrahedra run on the CSR layout (AUTO picks
   it; ELL, ELL16 and RING return VBD_ERR_UNSUPPORTED); like triangles and hinges, springs and tetrahedra
   must not span instances (worlds). */
int vbd_create(const VbdModelDesc* model, const VbdSolverParams* params, VbdHandle* out);

/* Re-reads the model arrays given to vbd_create (materials, rest state, masses, flags) after the
   caller changed them in place; replaces SolverVBD.notify_model_changed (solver_vbd.py:779-782). */
int vbd_refresh_model(VbdHandle h, void* stream);

/* Replaces SolverVBD.step(state_in, state_out, control, contacts, dt) for particles
   (solver_vbd.py:1575-1622): forward step, `iterations` colored VBD sweeps, velocity update.
   Side effects as in the reference: q_in_dev is overwritten with the solution, q_out_dev holds the
   same positions, qd_out_dev = (q - q_prev) / dt; qd_in_dev and particle_f_dev are read only.
   contacts / bodies may be NULL. Launches on `stream` (a cudaStream_t), never synchronizes. */
int vbd_step(VbdHandle h, float* q_in_dev, float* q_out_dev, const float* qd_in_dev, float* qd_out_dev,
             const float* particle_f_dev, const VbdContactsDesc* contacts, const VbdBodyState* bodies, float dt,
             void* stream);

/* The same step on float64 state arrays (VBD_PRECISION_FP64 solvers only). */
int vbd_step_f64(VbdHandle h, double* q_in_dev, double* q_out_dev, const double* qd_in_dev, double* qd_out_dev,
                 const double* particle_f_dev, const VbdContactsDesc* contacts, const VbdBodyState* bodies, double dt,
                 void* stream);

/* ---------------------------------------------------------------- differentiation (no reference
   counterpart: the reference VBD kernels are built with enable_backward=False,
   particle_vbd_kernels.py:27-28) */

/* The forward substep of vbd_step (per-color sweep) that also records what its adjoint needs: y [V,3] the
   inertial targets and checkpoints [(iterations+1),V,3] the positions at the start of every iteration and at
   the end. Arrays are float32, or float64 for a VBD_PRECISION_FP64 solver. q_out/qd_out receive the step's
   result (q_in is not modified). contacts: this substep's particle-shape contacts against static shapes, or
   NULL; the adjoint must be given the same arrays. Membranes, hinges, tetrahedra and springs with their damping
   take part. VBD_ERR_UNSUPPORTED for contacts with the AVBD penalty ramp on (rigid_avbd_beta > 0). */
int vbd_record_step(VbdHandle h, const void* q_in_dev, const void* qd_in_dev, const void* particle_f_dev,
                    const VbdContactsDesc* contacts, double dt, void* y_dev, void* checkpoints_dev, void* q_out_dev,
                    void* qd_out_dev, void* stream);

/* Reverse of that substep: from dL/dq_out and dL/dqd_out (either may be NULL = 0), writes dL/dq_in
   and dL/dqd_in and ADDS the triangles' dL/dmu and dL/dlambda (Model.tri_materials columns 0 and 1)
   into adj_tri_mu / adj_tri_lambda [T] (either may be NULL). contacts: the arrays the forward substep was
   given; their contact set, points, normals and stiffness are held fixed (the derivative of the step for
   those contacts). The first call allocates (colors + 3) x V x 3 work values; it returns
   VBD_ERR_UNSUPPORTED if that happens during a capture. */
int vbd_adjoint_step(VbdHandle h, const void* q_in_dev, const void* y_dev, const void* checkpoints_dev,
                     const VbdContactsDesc* contacts, double dt, const void* adj_q_out_dev,
                     const void* adj_qd_out_dev, void* adj_q_in_dev, void* adj_qd_in_dev, void* adj_tri_mu_dev,
                     void* adj_tri_lambda_dev, void* stream);

/* Reads and clears the device error word (VBD_DEVERR_* bits). Synchronizes `stream`. */
int vbd_get_error(VbdHandle h, int32_t* bits, void* stream);

/* MIXED precision: FP64 sum over particles of |f|^2 at each iteration of the last step (the force
   residual the block solve removes). n = iterations. Synchronizes `stream`. */
int vbd_get_residuals(VbdHandle h, double* out_host, int32_t n, void* stream);

/* Number of kernel launches one vbd_step issues (for accounting). */
int vbd_launches_per_step(VbdHandle h, int32_t* out);

/* Scheduling actually chosen (VBD_SCHEDULE_*, lanes per vertex, block size, dynamic shared memory
   per CTA of the persistent kernel (0 = positions in global memory), VBD_LAYOUT_*). Any pointer may
   be NULL. */
int vbd_get_config(VbdHandle h, int32_t* schedule, int32_t* lanes_per_vertex, int32_t* block_size,
                   int32_t* shared_bytes, int32_t* layout);

int vbd_destroy(VbdHandle h);

/* Diagnostics: vbd_eval_atan2 writes out[i] = the step's FP32 device atan2 of (y[i], x[i]) (the Abramowitz &
   Stegun 4.4.49 polynomial with the quadrant fix-up that the bending term uses in place of atan2f), for tests
   against the library atan2f. Device arrays of n floats. */
int vbd_eval_atan2(int32_t n, const float* y_dev, const float* x_dev, float* out_dev, void* stream);

/* ---------------------------------------------------------------- step without allocation */

/* Vertex -> element adjacency in the reference layout, as vbd_build_adjacency writes it (offsets
   count two ints per entry; entries are (element, order) pairs), copied to device memory. */
typedef struct VbdRefAdjacency {
  const int32_t* face_offsets_dev; /* [V+1] */
  const int32_t* faces_dev;
  const int32_t* edge_offsets_dev; /* [V+1] */
  const int32_t* edges_dev;
} VbdRefAdjacency;

#define VBD_NOALLOC_MAX_PARTICLES 32768
#define VBD_NOALLOC_MAX_CONTACT_SLOTS 4

/* A cloth step for callers that may not allocate device memory: a host application that owns all
   device memory through its own pool and forbids plug-ins to call cudaMalloc, or code that steps the
   cloth while capturing a larger CUDA graph, where an allocation would break the capture. No
   counterpart in the reference (there, SolverVBD.__init__ always allocates its scratch).
   Takes the model arrays in the reference layout (only the particle, triangle, hinge, color, gravity
   and shape-material fields of VbdModelDesc are read) and the adjacency above, and runs the same
   per-color FP32 step as vbd_step with the same side effects on the state arrays. It calls no
   cudaMalloc/cudaFree: its per-particle scratch and an error word are one fixed __device__ array of
   2,097,408 bytes (VBD_NOALLOC_MAX_PARTICLES particles) that every GPU loading the library keeps until
   exit. The first call with a device current looks up that array's address (cudaGetSymbolAddress); make
   it before any stream capture. All calls share the array: calls that overlap on the GPU race and must be
   serialised.
   Contacts: each particle keeps the VBD_NOALLOC_MAX_CONTACT_SLOTS contacts of lowest index in the contact
   list, whatever the thread timing; a particle with more drops the rest and sets
   VBD_DEVERR_CONTACT_OVERFLOW (read it with vbd_step_noalloc_error).
   Limits: at most VBD_NOALLOC_MAX_PARTICLES particles (else VBD_ERR_TOO_LARGE, nothing launched),
   static shapes with a fixed penalty (avbd beta = 0, the reference default), no springs or tetrahedra
   (else VBD_ERR_UNSUPPORTED). Inputs are trusted like the reference kernels trust theirs. */
int vbd_step_noalloc(const VbdModelDesc* model, const VbdRefAdjacency* adjacency, int32_t iterations,
                     float friction_epsilon, float* q_in_dev, float* q_out_dev, const float* qd_in_dev,
                     float* qd_out_dev, const float* particle_f_dev, const VbdContactsDesc* contacts, float dt,
                     void* stream);

/* The VBD_DEVERR_* bits of the last vbd_step_noalloc call on the current device (cleared when a call
   starts): contact overflow, contacts out of range, non-finite or singular (skipped) block solves. Waits for
   `stream`, then copies one int from the fixed array; allocates nothing. */
int vbd_step_noalloc_error(int32_t* bits, void* stream);

/* ---------------------------------------------------------------- particle self-contact */

/* Self-contact settings, with the meaning of the SolverVBD keywords (solver_vbd.py:204-216). */
typedef struct VbdSelfContactDesc {
  double radius;                /* particle_self_contact_radius: contact distance of the barrier */
  double margin;                /* particle_self_contact_margin: detection distance (>= radius) */
  double relaxation;            /* particle_conservative_bound_relaxation (gamma of the truncation) */
  double edge_parallel_epsilon; /* particle_edge_parallel_epsilon */
  double rest_exclusion_radius; /* particle_rest_shape_contact_exclusion_radius (0 = off) */
  int32_t vertex_buffer_size;   /* particle_vertex_contact_buffer_size: triangles kept per vertex */
  int32_t edge_buffer_size;     /* particle_edge_contact_buffer_size: edges kept per edge */
  int32_t detection_interval;   /* particle_collision_detection_interval */
  const float* rest_q_dev;      /* [V,3] Model.particle_q (rest shape); read when rest_exclusion_radius > 0 */
  /* collision filters (vbd_build_contact_filters plus the external filtering maps), CSR, or NULL */
  const int32_t* vt_filter_offsets_host; /* [V+1] */
  const int32_t* vt_filter_host;         /* triangles skipped per vertex */
  const int32_t* ee_filter_offsets_host; /* [E+1] */
  const int32_t* ee_filter_host;         /* edges skipped per edge */
} VbdSelfContactDesc;

/* Turns on particle self-contact for h (SolverVBD(particle_enable_self_contact=True),
   solver_vbd.py:489-526): vertex-triangle and edge-edge barrier contact with damping and friction
   (particle_vbd_kernels.py:1193-1779, accumulated per color as :1930-2071), with stiffness, damping and
   friction taken from the model's soft_contact_ke/kd/mu as the reference does; collision detection
   (tri_mesh_collision.py:333-413, geometry/kernels.py:1252-1497) at the start of each step and at the
   iterations i with i % interval == 0 (interval 0: i == 0 only; negative: never), and the
   penetration-free truncation after the forward step and after every color (particle_vbd_kernels.py:
   2475-2897, solver_vbd.py:1669-1766, 2151-2337). Needs the per-color schedule with the CSR layout
   (else VBD_ERR_UNSUPPORTED). Allocates its buffers here (synchronizes the device); VBD_ERR_TOO_LARGE
   when V x vertex_buffer_size or E x edge_buffer_size reaches 2^29. A second call replaces the settings. */
int vbd_set_self_contact(VbdHandle h, const VbdSelfContactDesc* desc);

/* Pairs recorded by the last detection of h's step and its overflow flags (bit 0: a vertex had more
   triangles than vertex_buffer_size, bit 2: an edge had more edges than edge_buffer_size; the
   lowest ids are kept). Synchronizes the stream. */
int vbd_get_self_contact_counts(VbdHandle h, int32_t* vt_pairs, int32_t* ee_pairs, int32_t* flags, void* stream);

/* Topological collision filters of SolverVBD._compute_particle_contact_filtering_list for a threshold
   ring >= 2 (build_vertex_n_ring_tris_collision_filter / build_edge_n_ring_edge_collision_filter,
   particle_vbd_kernels.py:2107-2255): per vertex v the triangles incident to a vertex within ring - 1
   edge steps of v other than v, less v's own triangles; per edge (a, b) the edges with an endpoint within
   ring - 1 steps of a or b other than a and b, less the edges in which a or b takes any of the four
   roles. Rows sorted. Call once with vt_list/ee_list NULL to get the offsets ([V+1], [E+1]), then with
   lists of vt_offsets[V] and ee_offsets[E] ints. */
int vbd_build_contact_filters(int32_t particle_count, int32_t tri_count, const int32_t* tri_indices_host,
                              int32_t edge_count, const int32_t* edge_indices_host, int32_t ring,
                              int32_t* vt_offsets_out, int32_t* vt_list_out, int32_t* ee_offsets_out,
                              int32_t* ee_list_out);

/* Stand-alone detector with the buffers of TriMeshCollisionDetector (tri_mesh_collision.py:91-413):
   vertex_colliding_triangles (2 ints per slot: vertex, triangle; -1 when empty), its counts and
   minimum distances, edge_colliding_edges likewise, and resize_flags (index 0 vertex, 2 edge overflow;
   set, never cleared, as the reference does). Pairs closer than max_query_radius, not adjacent, not
   filtered and, when min_query_radius > 0, not closer than that in ref_pos (the reference's
   min_distance_filtering_ref_pos). Slots hold the lowest primitive ids in increasing order. */
typedef struct VbdCollider* VbdColliderHandle;
int vbd_collider_create(int32_t particle_count, int32_t tri_count, const int32_t* tri_indices_dev, int32_t edge_count,
                        const int32_t* edge_indices_dev, int32_t vertex_buffer_size, int32_t edge_buffer_size,
                        float edge_parallel_epsilon, const int32_t* vt_filter_offsets_host,
                        const int32_t* vt_filter_host, const int32_t* ee_filter_offsets_host,
                        const int32_t* ee_filter_host, VbdColliderHandle* out);
/* what: bit 0 vertex-triangle (vertex_triangle_collision_detection), bit 1 edge-edge
   (edge_edge_collision_detection). Outputs of a pass not asked for are not touched. */
int vbd_collider_detect(VbdColliderHandle h, int32_t what, const float* pos_dev, float max_query_radius,
                        float min_query_radius, const float* ref_pos_dev, int32_t* vertex_colliding_triangles_dev,
                        int32_t* vertex_colliding_triangles_count_dev, float* vertex_colliding_triangles_min_dist_dev,
                        int32_t* edge_colliding_edges_dev, int32_t* edge_colliding_edges_count_dev,
                        float* edge_colliding_edges_min_dist_dev, int32_t* resize_flags_dev, void* stream);
/* record_triangle_contacting_vertices (tri_mesh_collision.py:170-200, geometry/kernels.py:1373-1384): every
   later vertex-triangle detection also fills the caller's triangle -> colliding vertices buffers, triangle t's
   at vertices_dev[t * buffer_size ...]: the vertex ids of its pairs (the buffer_size smallest, increasing; -1
   past them), count_dev[t] = all pairs found (may exceed the buffer; resize flag 1 is then set) and
   min_dist_dev[t] = the smallest pair distance (max_query_radius when none). buffer_size 0 turns it off. The
   buffers must outlive the detections. */
int vbd_collider_set_triangle_buffers(VbdColliderHandle h, int32_t buffer_size, int32_t* vertices_dev,
                                      int32_t* count_dev, float* min_dist_dev);
int vbd_collider_destroy(VbdColliderHandle h);

/* ---------------------------------------------------------------- host-side model preparation */

/* Particle coloring of the graph of ModelBuilder.color (builder.py:9304-9396,
   graph_coloring.py:99-236): triangle edges plus, when include_bending, all pairs of each active
   hinge's four vertices. Degree-ordered greedy assignment followed by a balancing pass that moves
   vertices from the largest to the smallest admissible colors until max/min <= target_ratio.
   Replaces wp.utils.graph_coloring_assign/balance (Warp native, not in the reference tree).
   colors_out: [V]. Returns the number of colors (>= 0) or a negative error. */
int vbd_color_particles(int32_t particle_count, int32_t tri_count, const int32_t* tri_indices_host,
                        const float* tri_materials_host, int32_t edge_count, const int32_t* edge_indices_host,
                        const float* edge_bending_properties_host, int32_t include_bending, float target_ratio,
                        int32_t* colors_out);

/* Coloring of any particle graph, given as pair_count (a, b) index pairs (duplicates and a == b ignored), e.g.
   the graph of ModelBuilder.color (construct_particle_graph, graph_coloring.py:200-240: triangle edges, hinge
   vertex pairs, the six vertex pairs of every active tet). algorithm: 0 = MCS (the maximum cardinality search
   order, the reference's default ColoringAlgorithm.MCS), 1 = degree-ordered greedy (ColoringAlgorithm.GREEDY);
   then the balancing pass of vbd_color_particles when target_ratio > 1. Returns the number of colors or an
   error. */
int vbd_color_graph(int32_t particle_count, int32_t pair_count, const int32_t* pairs_host, int32_t algorithm,
                    float target_ratio, int32_t* colors_out);

/* Vertex -> (element, order) adjacency in the reference layout (ParticleForceElementAdjacencyInfo,
   particle_vbd_kernels.py:66-151, fill order :639-738): offsets count two ints per entry. */
int vbd_build_adjacency(int32_t particle_count, int32_t tri_count, const int32_t* tri_indices_host,
                        int32_t edge_count, const int32_t* edge_indices_host, int32_t* face_offsets_out,
                        int32_t* faces_out, int32_t* edge_offsets_out, int32_t* edges_out);

/* ---------------------------------------------------------------- particle-shape contacts */

/* Soft contacts of active particles against static shapes, as CollisionPipeline.collide writes
   them (collide.py:1212-1246, geometry/kernels.py:1001-1140) for shape types 0 = infinite plane
   through shape_pos with unit normal shape_normal (GeoType.PLANE with zero extents; NULL normals
   mean +Z) and 1 = sphere of radius shape_radius at shape_pos; at most 16 shapes. One contact per
   (particle, shape) within margin + radius. As in the reference, slots come from an atomic
   counter, so the order of contacts is not fixed; count_dev receives the number found (it may
   exceed soft_contact_max, entries beyond it are dropped). */
int vbd_soft_contacts(int32_t particle_count, const float* q_dev, const float* radius_dev, const int32_t* flags_dev,
                      int32_t shape_count, const int32_t* shape_type_host, const float* shape_pos_host,
                      const float* shape_radius_host, const float* shape_normal_host, float margin,
                      int32_t soft_contact_max, int32_t* count_dev,
                      int32_t* particle_dev, int32_t* shape_dev, float* body_pos_dev, float* body_vel_dev,
                      float* normal_dev, void* stream);

/* Soft contacts against static analytic shapes, as CollisionPipeline.collide writes them for shapes without a
   body (create_soft_contacts, geometry/kernels.py:1001-1140, with the SDFs and gradients of
   geometry/kernels.py:132-600). shape_type holds the reference's GeoType values: 1 plane (local +Z normal;
   scale (width, length), 0 = infinite, else the reference's Chebyshev distance to the quad), 3 sphere (r),
   4 capsule (r, half height; along local Z), 5 ellipsoid (rx, ry, rz), 6 cylinder (r, half height; along local
   Z), 7 box (half extents), 9 cone (base radius, half height; base at local z = -half height, apex at
   +half height); heightfields (2) and meshes (8, 10) need vbd_soft_contacts_table; other types return
   VBD_ERR_UNSUPPORTED. shape_transform_host [S,7]: position and
   rotation quaternion (x, y, z, w) of each shape; shape_scale_host [S,3]; at most 16 shapes. Contacts are
   written as vbd_soft_contacts writes them: the contact point on the surface in world (the body frame of a
   static shape), zero body velocity, the world normal; slots from an atomic counter. */
int vbd_soft_contacts_shapes(int32_t particle_count, const float* q_dev, const float* radius_dev,
                             const int32_t* flags_dev, int32_t shape_count, const int32_t* shape_type_host,
                             const float* shape_transform_host, const float* shape_scale_host, float margin,
                             int32_t soft_contact_max, int32_t* count_dev, int32_t* particle_dev, int32_t* shape_dev,
                             float* body_pos_dev, float* body_vel_dev, float* normal_dev, void* stream);

/* One heightfield grid (HeightfieldData, utils/heightfield.py:65-77, as the reference builder fills it,
   sim/builder.py:10698-10718): nrow x ncol elevations normalized to [0, 1] starting at data_offset in the
   concatenated elevation array; height z = min_z + e (max_z - min_z); the grid spans [-hx, hx] x [-hy, hy] of the
   shape frame. The shape's scale is already applied (hx = |hx sx|, hy = |hy sy|, min_z sz, max_z sz). */
typedef struct VbdHeightfield {
  int32_t data_offset;
  int32_t nrow;
  int32_t ncol;
  float hx;
  float hy;
  float min_z;
  float max_z;
} VbdHeightfield;

/* A static triangle mesh for particle contacts (GeoType 8 MESH and 10 CONVEX_MESH; the wp.Mesh the reference
   builds from Mesh.vertices and Mesh.indices, geometry/types.py:1436-1453, with zero velocities). points_host
   [point_count,3] in the mesh frame, indices_host [tri_count,3]. Builds a bounding-volume hierarchy and the
   angle-weighted pseudo-normals that decide inside and outside on the host and uploads them (synchronous). */
typedef struct VbdMeshImpl* VbdMeshHandle;
int vbd_mesh_create(const float* points_host, int32_t point_count, const int32_t* indices_host, int32_t tri_count,
                    VbdMeshHandle* out);
int vbd_mesh_destroy(VbdMeshHandle mesh);

/* The shapes a contact generation runs against, in the reference Model's layout (at most 16 shapes).
   shape_type_host [S]: GeoType values; shape_transform_host [S,7]: position and rotation (x, y, z, w);
   shape_scale_host [S,3]. Heightfield shape s (type 2) takes grid shape_heightfield_index_host[s] of
   heightfields_host[heightfield_count] over elevations_dev (elevation_count floats). Mesh shape s (types 8 and
   10) takes shape_mesh_host[s]; its scale must have no zero component. The arrays for a kind of shape may be
   NULL when no shape of that kind is present. shape_flags_host [S] (ShapeFlags bits; NULL = all collide): shapes
   without COLLIDE_PARTICLES (1 << 2) are skipped. shape_world_host [S] and particle_world_dev [particle_count]
   (NULL = all global): a particle and a shape of different worlds do not collide unless either is global (-1),
   as create_soft_contacts filters them (geometry/kernels.py:1031-1043). */
typedef struct VbdShapeTable {
  int32_t shape_count;
  const int32_t* shape_type_host;
  const float* shape_transform_host;
  const float* shape_scale_host;
  const int32_t* shape_heightfield_index_host;
  int32_t heightfield_count;
  const VbdHeightfield* heightfields_host;
  const float* elevations_dev;
  int64_t elevation_count;
  const VbdMeshHandle* shape_mesh_host;
  const int32_t* shape_flags_host;
  const int32_t* shape_world_host;
  const int32_t* particle_world_dev;
  /* shapes on bodies (geometry/kernels.py:1045-1056): shape s is carried by body shape_body_host[s] (-1 = static,
     NULL = all static) of body_count bodies; body_q_dev [body_count, 7] holds the body transforms (p, q xyzw) for
     vbd_soft_contacts_table (the shape sets take them per call instead) */
  const int32_t* shape_body_host;
  int32_t body_count;
  const float* body_q_dev;
} VbdShapeTable;

/* vbd_soft_contacts_shapes over a full shape table: the analytic types, heightfields (sample_sdf_grad_heightfield,
   utils/heightfield.py:94-205; grids with nrow or ncol below 2 give no contacts, as in the reference) and
   triangle meshes (geometry/kernels.py:1091-1113: the particle in the mesh's unscaled frame, the closest point
   within margin + radius / min|scale| and its pseudo-normal sign; distance and normal from the scaled closest
   point). Returns VBD_ERR_INVALID_ARGUMENT for a heightfield index out of range, a grid that overruns
   elevation_count, a non-positive or non-finite hx or hy (for which the reference's cell index is undefined),
   a missing mesh handle or a mesh scale with a zero or non-finite component; VBD_ERR_UNSUPPORTED for Gaussians
   and unknown types. */
int vbd_soft_contacts_table(int32_t particle_count, const float* q_dev, const float* radius_dev,
                            const int32_t* flags_dev, const VbdShapeTable* shapes, float margin,
                            int32_t soft_contact_max, int32_t* count_dev, int32_t* particle_dev, int32_t* shape_dev,
                            float* body_pos_dev, float* body_vel_dev, float* normal_dev, void* stream);

/* A model's shapes uploaded once for contact generation, any number of shapes and worlds: the shapes with
   COLLIDE_PARTICLES, their records and, per world, the list of its shapes (create_soft_contacts' world filter,
   geometry/kernels.py:1036-1043). Takes the VbdShapeTable fields except particle_world_dev and body_q_dev; world
   indices must be -1 (global) or non-negative, body indices -1 (static) or below body_count. The mesh handles and
   the elevation array the table names must outlive the set. */
typedef struct VbdShapeSetImpl* VbdShapeSetHandle;
int vbd_shape_set_create(const VbdShapeTable* shapes, VbdShapeSetHandle* out);
int vbd_shape_set_destroy(VbdShapeSetHandle set);
/* Sets of up to 16 shapes launch with their records as a kernel parameter, read through the constant bank (the
   default, enable = 1); enable = 0 sends every size through the global-memory kernel and its world lists. Both
   give the same contacts. */
int vbd_shape_set_use_parameter_table(VbdShapeSetHandle set, int32_t enable);

/* Soft contacts of every active particle against a shape set, written as vbd_soft_contacts_shapes writes them. A
   particle of world w (particle_world_dev; NULL = all global) tests the global shapes and world w's shapes; a
   global particle tests every shape. body_q_dev: the body transforms [bodies, 7] (p, q xyzw) of this call
   (state.body_q), required when a shape of the set is on a body, else ignored; such a shape's contact point is
   written in its body's frame and its normal in world (create_soft_contacts, geometry/kernels.py:1045-1056,
   1128-1140). */
int vbd_soft_contacts_set(VbdShapeSetHandle set, int32_t particle_count, const float* q_dev, const float* radius_dev,
                          const int32_t* flags_dev, const int32_t* particle_world_dev, const float* body_q_dev,
                          float margin, int32_t soft_contact_max, int32_t* count_dev, int32_t* particle_dev,
                          int32_t* shape_dev, float* body_pos_dev, float* body_vel_dev, float* normal_dev,
                          void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VBD_B200_H */
