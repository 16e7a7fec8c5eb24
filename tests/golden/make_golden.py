"""Generate golden vectors for the cloth VBD path by executing the reference's own code.

Run where a checkout of the reference project is readable, naming its root (or set ``VBD_REFERENCE_ROOT``)::

    python tests/golden/make_golden.py --ref PATH/TO/newton-ChysX [--out tests/golden]

Warp is not installed, so ``warp_shim.py`` stands in for the Warp builtins and the
reference's kernel bodies run as plain float64 Python. The functions are lifted out of
the reference sources with ``ast`` (decorators and annotations dropped) and executed
unchanged:

* ``newton/_src/solvers/vbd/particle_vbd_kernels.py``: adjacency builders ``:639-738``,
  ``evaluate_neo_hookean_membrane_force_hessian :865-1025``, bending ``:1028-1190``,
  ``forward_step :1782-1807``, ``update_velocity :1900-1903``, ``apply_truncation_ts :2877-2897``,
  ``accumulate_particle_body_contact_force_and_hessian :2900-2967``, ``solve_elasticity :3135-3273``;
* ``newton/_src/solvers/vbd/rigid_vbd_kernels.py``: ``_average_contact_material :314-330``,
  ``_compute_body_particle_contact_force :727-759``, ``_eval_body_particle_contact :762-834``,
  ``compute_projected_isotropic_friction :891-934``, ``init_body_particle_contacts :2318-2361``,
  ``update_duals_body_particle_contacts :3755-3799``;
* self-contact: ``particle_vbd_kernels.py`` ``evaluate_self_contact_force_norm :1193-1222``,
  ``damp_collision :1225-1238``, ``evaluate_edge_edge_contact_2_vertices :1371-1506``,
  ``evaluate_vertex_triangle_collision_force_hessian_4_vertices :1599-1745``, ``compute_friction :1748-1779``,
  ``accumulate_self_contact_force_and_hessian :1930-2071``, the n-ring filters ``:2074-2255``, the
  division planes and ``planar_truncation_t :2475-2742``, ``apply_planar_truncation_parallel_by_collision
  :2744-2874``; ``geometry/kernels.py`` ``triangle_closest_point :64-128``, the detection kernels
  ``:1229-1497``; ``math/__init__.py`` ``orthonormal_basis``; ``geometry/broad_phase_common.py``
  ``binary_search``. ``SelfContactRef`` mirrors ``TriMeshCollisionDetector`` (``tri_mesh_collision.py:91-413``)
  with the shim's brute-force box query standing in for ``wp.Bvh``;
* ``newton/_src/sim/builder.py``: ``add_triangles :7716-7826``, ``add_edges :7966-8061``,
  ``add_cloth_grid :8063-8186``, ``add_cloth_mesh :8188-8341``; ``newton/_src/utils/mesh.py``:
  ``MeshAdjacency :183-262``.

The launch sequence of ``SolverVBD.step`` (``solver_vbd.py:1575-1622, 1669-1766, 2151-2337,
2339-2376, 2763-2774``) is mirrored by ``ref_step`` below; every kernel body it calls is the
reference's. Contacts for a ground plane / static sphere follow ``create_soft_contacts``
(``geometry/kernels.py:1001-1140``) for those two shape types. Colorings come from a
plain greedy pass here (the reference's coloring lives in Warp's native library) and are
stored with the fixtures, so every consumer sweeps the same color order.
"""

from __future__ import annotations

import argparse
import ast
import dataclasses
import math
import os
import sys
import types
import warnings
from collections.abc import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import warp_shim as wp  # noqa: E402


class ParticleFlags:
    ACTIVE = 1 << 0


class _BvhLoopRewrite(ast.NodeTransformer):
    """``while wp.bvh_query_next(query, i): ...`` -> ``for i in query: ...``.

    Warp's ``bvh_query_next`` writes the next primitive index through its second argument, which
    plain Python cannot do; the shim's ``bvh_query_aabb`` returns the list of hits instead. The loop
    body (including its ``continue`` statements) is unchanged."""

    def visit_While(self, node):
        self.generic_visit(node)
        t = node.test
        if isinstance(t, ast.Call) and isinstance(t.func, ast.Attribute) and t.func.attr == "bvh_query_next":
            query, index = t.args
            loop = ast.For(target=ast.Name(id=index.id, ctx=ast.Store()), iter=query, body=node.body, orelse=[],
                           type_comment=None)  # fmt: skip
            return ast.copy_location(loop, node)
        return node


def _lift(path: str, names: set[str], ns: dict, classes: dict[str, set[str]] | None = None):
    """Execute the named top-level functions (and selected class methods) of ``path`` in ``ns``."""
    with open(path) as f:
        tree = ast.parse(f.read(), filename=path)

    def strip(fn):
        fn.decorator_list = []
        fn.returns = None
        for a in fn.args.args + fn.args.kwonlyargs + fn.args.posonlyargs:
            a.annotation = None
        if fn.args.vararg:
            fn.args.vararg.annotation = None
        if fn.args.kwarg:
            fn.args.kwarg.annotation = None
        return fn

    found = set()
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in names:
            fn = ast.fix_missing_locations(_BvhLoopRewrite().visit(strip(node)))
            mod = ast.Module(body=[fn], type_ignores=[])
            exec(compile(mod, path, "exec"), ns)
            found.add(node.name)
        if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            if node.targets[0].id in names:  # module constants such as ``X = wp.constant(0)``
                exec(compile(ast.Module(body=[node], type_ignores=[]), path, "exec"), ns)
                found.add(node.targets[0].id)
        if classes and isinstance(node, ast.ClassDef) and node.name in classes:
            wanted = classes[node.name]
            if wanted == {"*"}:
                for sub in ast.walk(node):
                    if isinstance(sub, ast.FunctionDef):
                        strip(sub)
                    if isinstance(sub, ast.AnnAssign):
                        pass
                mod = ast.Module(body=[node], type_ignores=[])
                exec(compile(mod, path, "exec"), ns)
                found.add(node.name)
            else:
                for sub in node.body:
                    if isinstance(sub, ast.FunctionDef) and sub.name in wanted:
                        mod = ast.Module(body=[strip(sub)], type_ignores=[])
                        exec(compile(mod, path, "exec"), ns)
                        found.add(sub.name)
    expected = set(names)
    for cname, wanted in (classes or {}).items():
        expected |= {cname} if wanted == {"*"} else set(wanted)
    missing = expected - found
    if missing:
        raise RuntimeError(f"not found in {path}: {sorted(missing)}")


def load_reference(ref: str) -> dict:
    module = types.ModuleType("vbd_reference_lifted")
    sys.modules[module.__name__] = module
    ns: dict = module.__dict__
    ns.update({
        "wp": wp,
        "np": np,
        "math": math,
        "ParticleFlags": ParticleFlags,
        "VBD_DEBUG_PRINTING_OPTIONS": set(),
        "dataclass": dataclasses.dataclass,
        "warnings": warnings,
        "Sequence": Sequence,
        "Any": object,
    })
    vbd = os.path.join(ref, "newton/_src/solvers/vbd")
    _lift(
        os.path.join(vbd, "rigid_vbd_kernels.py"),
        {
            "_average_contact_material",
            "_compute_body_particle_contact_force",
            "_eval_body_particle_contact",
            "compute_projected_isotropic_friction",
            "init_body_particle_contacts",
            "update_duals_body_particle_contacts",
        },
        ns,
    )
    _lift(
        os.path.join(vbd, "particle_vbd_kernels.py"),
        {
            "get_vertex_num_adjacent_edges",
            "get_vertex_adjacent_edge_id_order",
            "get_vertex_num_adjacent_faces",
            "get_vertex_adjacent_face_id_order",
            "_count_num_adjacent_edges",
            "_fill_adjacent_edges",
            "_count_num_adjacent_faces",
            "_fill_adjacent_faces",
            "evaluate_neo_hookean_membrane_force_hessian",
            "compute_normalized_vector_derivative",
            "compute_angle_derivative",
            "evaluate_dihedral_angle_based_bending_force_hessian",
            "forward_step",
            "update_velocity",
            "apply_truncation_ts",
            "accumulate_particle_body_contact_force_and_hessian",
            "solve_elasticity",
        },
        ns,
    )
    # volumetric (tetrahedra) and spring elements (particle_vbd_kernels.py:150-242, 335-546, 774-825, 2258-2397)
    ns["vec9"], ns["mat99"], ns["mat93"], ns["mat43"] = wp._vec_ctor(9), wp._mat_ctor(9, 9), wp._mat_ctor(9, 3), wp._mat_ctor(4, 3)
    _lift(
        os.path.join(vbd, "particle_vbd_kernels.py"),
        {
            "get_vertex_num_adjacent_tets",
            "get_vertex_adjacent_tet_id_order",
            "_count_num_adjacent_tets",
            "_fill_adjacent_tets",
            "assemble_tet_vertex_force_and_hessian",
            "evaluate_volumetric_neo_hookean_force_and_hessian",
            "compute_cofactor",
            "evaluate_spring_force_and_hessian_both_vertices",
            "accumulate_spring_force_and_hessian",
        },
        ns,
    )
    # self-contact (particle_vbd_kernels.py:1193-2255, 2475-2874) and its geometry helpers
    ns["mat32"] = wp.mat32
    _lift(os.path.join(ref, "newton/_src/math/__init__.py"), {"orthonormal_basis"}, ns)
    _lift(os.path.join(ref, "newton/_src/geometry/broad_phase_common.py"), {"binary_search"}, ns)
    _lift(
        os.path.join(ref, "newton/_src/geometry/kernels.py"),
        {
            "triangle_closest_point",
            "vertex_adjacent_to_triangle",
            "vertex_triangle_collision_detection_kernel",
            "edge_colliding_edges_detection_kernel",
            "TRI_CONTACT_FEATURE_VERTEX_A",
            "TRI_CONTACT_FEATURE_VERTEX_B",
            "TRI_CONTACT_FEATURE_VERTEX_C",
            "TRI_CONTACT_FEATURE_EDGE_AB",
            "TRI_CONTACT_FEATURE_EDGE_AC",
            "TRI_CONTACT_FEATURE_EDGE_BC",
            "TRI_CONTACT_FEATURE_FACE_INTERIOR",
            "VERTEX_COLLISION_BUFFER_OVERFLOW_INDEX",
            "TRI_COLLISION_BUFFER_OVERFLOW_INDEX",
            "EDGE_COLLISION_BUFFER_OVERFLOW_INDEX",
        },
        ns,
    )
    _lift(
        os.path.join(vbd, "particle_vbd_kernels.py"),
        {
            "NUM_THREADS_PER_COLLISION_PRIMITIVE",
            "evaluate_self_contact_force_norm",
            "damp_collision",
            "evaluate_edge_edge_contact_2_vertices",
            "evaluate_vertex_triangle_collision_force_hessian_4_vertices",
            "compute_friction",
            "accumulate_self_contact_force_and_hessian",
            "_csr_row",
            "set_to_csr",
            "one_ring_vertices",
            "leq_n_ring_vertices",
            "build_vertex_n_ring_tris_collision_filter",
            "build_edge_n_ring_edge_collision_filter",
            "segment_plane_intersects",
            "create_vertex_triangle_division_plane_closest_pt",
            "robust_edge_pair_normal",
            "create_edge_edge_division_plane_closest_pt",
            "planar_truncation_t",
            "apply_planar_truncation_parallel_by_collision",
        },
        ns,
    )
    # particle-shape contact generation: the analytic SDFs of create_soft_contacts (geometry/kernels.py:132-600)
    ns["Axis"] = types.SimpleNamespace(X=0, Y=1, Z=2)
    _lift(
        os.path.join(ref, "newton/_src/geometry/kernels.py"),
        {"_sdf_point_to_z_up", "_sdf_vector_from_z_up", "sdf_sphere", "sdf_sphere_grad", "sdf_box", "sdf_box_grad",
         "sdf_capsule", "sdf_capsule_grad", "sdf_cylinder", "sdf_cylinder_grad", "sdf_ellipsoid", "sdf_ellipsoid_grad",
         "sdf_plane", "_sdf_capped_cone_z", "sdf_cone", "sdf_cone_grad"},
        ns,
    )  # fmt: skip
    _lift(os.path.join(ref, "newton/_src/utils/heightfield.py"),
          {"_heightfield_surface_query", "sample_sdf_grad_heightfield"}, ns)  # fmt: skip
    # the contact generation kernel itself, for analytic shapes and heightfields (no mesh shapes are launched)
    ns["GeoType"] = types.SimpleNamespace(PLANE=1, HFIELD=2, SPHERE=3, CAPSULE=4, ELLIPSOID=5, CYLINDER=6, BOX=7, MESH=8,
                                          CONE=9, CONVEX_MESH=10)  # fmt: skip
    ns["ShapeFlags"] = types.SimpleNamespace(COLLIDE_PARTICLES=1 << 2)
    _lift(os.path.join(ref, "newton/_src/geometry/kernels.py"), {"counter_increment", "create_soft_contacts"}, ns)
    _lift(os.path.join(ref, "newton/_src/utils/mesh.py"), set(), ns, classes={"MeshAdjacency": {"*"}})
    _lift(
        os.path.join(ref, "newton/_src/sim/builder.py"),
        set(),
        ns,
        classes={"ModelBuilder": {"add_triangles", "add_edges", "add_cloth_grid", "add_cloth_mesh", "add_particle",
                                  "add_spring", "add_triangle", "add_tetrahedron", "add_edge", "add_soft_grid"}},
    )
    return ns


# ----------------------------------------------------------------------------- builder
class FakeBuilder:
    """Holds the list-valued fields the reference builder methods append to."""

    def __init__(self, ns):
        self.ns = ns
        self.particle_q, self.particle_qd, self.particle_mass = [], [], []
        self.particle_radius, self.particle_flags = [], []
        self.tri_indices, self.tri_poses, self.tri_activations = [], [], []
        self.tri_materials, self.tri_areas = [], []
        self.edge_indices, self.edge_rest_angle, self.edge_rest_length = [], [], []
        self.edge_bending_properties = []
        self.default_tri_ke, self.default_tri_ka, self.default_tri_kd = 100.0, 100.0, 10.0
        self.default_tri_drag, self.default_tri_lift = 0.0, 0.0
        self.default_edge_ke, self.default_edge_kd = 100.0, 0.0
        self.default_spring_ke, self.default_spring_kd = 100.0, 0.0
        self.default_particle_radius = 0.1
        for name in ("add_triangles", "add_edges", "add_cloth_grid", "add_cloth_mesh"):
            setattr(self, name, types.MethodType(ns[name], self))

    def add_particles(self, pos, vel, mass, radius=None, flags=None, custom_attributes=None):
        for i in range(len(pos)):
            self.particle_q.append(tuple(float(x) for x in pos[i]))
            self.particle_qd.append(tuple(float(x) for x in np.asarray(vel[i], dtype=float)))
            self.particle_mass.append(float(mass[i]))
            self.particle_radius.append(float(radius[i]) if radius is not None else self.default_particle_radius)
            self.particle_flags.append(ParticleFlags.ACTIVE)

    def arrays(self) -> dict:
        mass = np.array(self.particle_mass, dtype=np.float64)
        return {
            "particle_q": np.array(self.particle_q, dtype=np.float64).reshape(-1, 3),
            "particle_qd": np.array(self.particle_qd, dtype=np.float64).reshape(-1, 3),
            "particle_mass": mass,
            "particle_inv_mass": np.where(mass > 0.0, 1.0 / np.where(mass > 0.0, mass, 1.0), 0.0),
            "particle_radius": np.array(self.particle_radius, dtype=np.float64),
            "particle_flags": np.array(self.particle_flags, dtype=np.int32),
            "tri_indices": np.array(self.tri_indices, dtype=np.int32).reshape(-1, 3),
            "tri_poses": np.array(self.tri_poses, dtype=np.float64).reshape(-1, 2, 2),
            "tri_materials": np.array(self.tri_materials, dtype=np.float64).reshape(-1, 5),
            "tri_areas": np.array(self.tri_areas, dtype=np.float64),
            "edge_indices": np.array(self.edge_indices, dtype=np.int32).reshape(-1, 4),
            "edge_rest_angle": np.array(self.edge_rest_angle, dtype=np.float64),
            "edge_rest_length": np.array(self.edge_rest_length, dtype=np.float64),
            "edge_bending_properties": np.array(self.edge_bending_properties, dtype=np.float64).reshape(-1, 2),
        }


class SoftBuilder(FakeBuilder):
    """FakeBuilder plus the particle, spring and tetrahedron fields that ``add_soft_grid`` and friends
    append to; particle positions are kept as shim vectors, as the reference's builder math expects."""

    def __init__(self, ns):
        super().__init__(ns)
        self.particle_world, self.current_world = [], -1
        self.spring_indices, self.spring_rest_length, self.spring_stiffness = [], [], []
        self.spring_damping, self.spring_control = [], []
        self.tet_indices, self.tet_poses, self.tet_activations, self.tet_materials = [], [], [], []
        for name in ("add_particle", "add_spring", "add_triangle", "add_tetrahedron", "add_edge", "add_soft_grid"):
            setattr(self, name, types.MethodType(ns[name], self))

    @property
    def particle_count(self):
        return len(self.particle_q)

    def arrays(self) -> dict:
        q = [np.asarray(x, dtype=np.float64) for x in self.particle_q]
        qd = [np.asarray(x, dtype=np.float64) for x in self.particle_qd]
        saved = self.particle_q, self.particle_qd
        self.particle_q, self.particle_qd = q, qd
        try:
            out = super().arrays()
        finally:
            self.particle_q, self.particle_qd = saved
        out.update(
            spring_indices=np.array(self.spring_indices, dtype=np.int32).reshape(-1, 2),
            spring_rest_length=np.array(self.spring_rest_length, dtype=np.float64),
            spring_stiffness=np.array(self.spring_stiffness, dtype=np.float64),
            spring_damping=np.array(self.spring_damping, dtype=np.float64),
            tet_indices=np.array(self.tet_indices, dtype=np.int32).reshape(-1, 4),
            tet_poses=np.array(self.tet_poses, dtype=np.float64).reshape(-1, 3, 3),
            tet_materials=np.array(self.tet_materials, dtype=np.float64).reshape(-1, 3),
        )  # fmt: skip
        return out


def greedy_coloring(n, tri_indices, edge_indices, edge_props, tet_indices=(), spring_indices=()):
    """Greedy coloring of the particle graph of ``construct_particle_graph`` (graph_coloring.py:199-236):
    triangle edges, active hinges' vertex pairs, tetrahedra's vertex pairs, plus the springs' endpoints
    (the solve needs them in different colors)."""
    adj = [set() for _ in range(n)]

    def link(a, b):
        if a >= 0 and b >= 0 and a != b:
            adj[a].add(b)
            adj[b].add(a)

    for t in tri_indices:
        link(t[0], t[1])
        link(t[0], t[2])
        link(t[1], t[2])
    for e, p in zip(edge_indices, edge_props, strict=True):
        if p[0] != 0.0 or p[1] != 0.0:
            for i in range(4):
                for j in range(i + 1, 4):
                    link(e[i], e[j])
    for t in tet_indices:
        for i in range(4):
            for j in range(i + 1, 4):
                link(t[i], t[j])
    for sp in spring_indices:
        link(sp[0], sp[1])
    colors = -np.ones(n, dtype=np.int32)
    for v in sorted(range(n), key=lambda v: -len(adj[v])):
        used = {colors[u] for u in adj[v]}
        c = 0
        while c in used:
            c += 1
        colors[v] = c
    groups = [np.nonzero(colors == c)[0].astype(np.int32) for c in range(colors.max() + 1)]
    return colors, groups


# ----------------------------------------------------------------------------- contacts
def plane_contacts(q, radius, flags, margin, shape_index=0):
    """Soft contacts of particles against the ground plane z=0 (infinite ``sdf_plane``)."""
    out = []
    for i, x in enumerate(q):
        if not (flags[i] & ParticleFlags.ACTIVE):
            continue
        d = x[2]
        if d < margin + radius[i]:
            n = np.array([0.0, 0.0, 1.0])
            out.append((i, shape_index, x - n * d, np.zeros(3), n))
    return out


def sphere_contacts(q, radius, flags, margin, center, r_sphere, shape_index=0):
    """Soft contacts against a static sphere (``sdf_sphere``/``sdf_sphere_grad``, geometry/kernels.py:163-190)."""
    out = []
    for i, x in enumerate(q):
        if not (flags[i] & ParticleFlags.ACTIVE):
            continue
        xl = x - center
        L = np.linalg.norm(xl)
        d = L - r_sphere
        n = xl / L if L > 1e-8 else np.array([0.0, 0.0, 1.0])
        if d < margin + radius[i]:
            out.append((i, shape_index, xl - n * d, np.zeros(3), n))
    return out


# ----------------------------------------------------------------------------- step driver
def build_adjacency(ns, tri_indices, edge_indices, n):
    tri = wp.array2d(tri_indices, int)
    edges = wp.array2d(edge_indices, int)
    cnt = wp.scalar_array(np.zeros(n, dtype=np.int64), int)
    ns["_count_num_adjacent_faces"](tri, cnt)
    f_off = np.concatenate([[0], np.cumsum(np.array(cnt.items) * 2)]).astype(np.int64)
    f_adj = wp.scalar_array(np.zeros(int(f_off[-1]), dtype=np.int64), int)
    ns["_fill_adjacent_faces"](tri, wp.scalar_array(f_off, int), wp.scalar_array(np.zeros(n), int), f_adj)
    cnt = wp.scalar_array(np.zeros(n, dtype=np.int64), int)
    ns["_count_num_adjacent_edges"](edges, cnt)
    e_off = np.concatenate([[0], np.cumsum(np.array(cnt.items) * 2)]).astype(np.int64)
    e_adj = wp.scalar_array(np.zeros(int(e_off[-1]), dtype=np.int64), int)
    ns["_fill_adjacent_edges"](edges, wp.scalar_array(e_off, int), wp.scalar_array(np.zeros(n), int), e_adj)
    return f_off, np.array(f_adj.items), e_off, np.array(e_adj.items)


def build_tet_adjacency(ns, tet_indices, n):
    tets = wp.array2d(np.asarray(tet_indices).reshape(-1, 4), int)
    cnt = wp.scalar_array(np.zeros(n, dtype=np.int64), int)
    ns["_count_num_adjacent_tets"](tets, cnt)
    off = np.concatenate([[0], np.cumsum(np.array(cnt.items) * 2)]).astype(np.int64)
    adj = wp.scalar_array(np.zeros(int(off[-1]), dtype=np.int64), int)
    ns["_fill_adjacent_tets"](tets, wp.scalar_array(off, int), wp.scalar_array(np.zeros(n), int), adj)
    return off, np.array(adj.items)


class RefScene:
    """Model arrays as shim arrays, plus the solver scratch of ``SolverVBD._init_particle_system``."""

    def __init__(self, ns, m: dict, groups, colors, gravity, soft, shapes):
        self.ns = ns
        self.m = m
        n = len(m["particle_q"])
        self.n = n
        self.groups = groups
        self.colors = colors
        self.gravity = wp.vec_array(np.asarray(gravity).reshape(1, 3))
        f_off, f_adj, e_off, e_adj = build_adjacency(ns, m["tri_indices"], m["edge_indices"], n)
        t_off, t_adj = build_tet_adjacency(ns, m.get("tet_indices", np.zeros((0, 4), np.int32)), n)
        self.adj = types.SimpleNamespace(
            v_adj_faces=wp.scalar_array(f_adj, int),
            v_adj_faces_offsets=wp.scalar_array(f_off, int),
            v_adj_edges=wp.scalar_array(e_adj, int),
            v_adj_edges_offsets=wp.scalar_array(e_off, int),
            v_adj_tets=wp.scalar_array(t_adj, int),
            v_adj_tets_offsets=wp.scalar_array(t_off, int),
        )
        self.tet_adjacency_np = (t_off, t_adj)
        nt = len(m.get("tet_indices", ()))
        self.tet_indices = wp.array2d(m["tet_indices"], int) if nt else wp.Array([])
        self.tet_poses = wp.mat33_array(m["tet_poses"]) if nt else wp.Array([])
        self.tet_materials = wp.array2d(m["tet_materials"]) if nt else wp.Array([])
        ns_ = len(m.get("spring_rest_length", ()))
        self.spring_count = ns_
        if ns_:
            self.spring_indices = wp.scalar_array(np.asarray(m["spring_indices"]).reshape(-1), int)
            self.spring_rest_length = wp.scalar_array(m["spring_rest_length"])
            self.spring_stiffness = wp.scalar_array(m["spring_stiffness"])
            self.spring_damping = wp.scalar_array(m["spring_damping"])
        self.adjacency_np = (f_off, f_adj, e_off, e_adj)
        self.mass = wp.scalar_array(m["particle_mass"])
        self.inv_mass = wp.scalar_array(m["particle_inv_mass"])
        self.flags = wp.scalar_array(m["particle_flags"], int)
        self.radius = wp.scalar_array(m["particle_radius"])
        self.tri_indices = wp.array2d(m["tri_indices"], int)
        self.tri_poses = wp.mat22_array(m["tri_poses"])
        self.tri_materials = wp.array2d(m["tri_materials"])
        self.tri_areas = wp.scalar_array(m["tri_areas"])
        self.edge_indices = wp.array2d(m["edge_indices"], int)
        self.edge_rest_angle = wp.scalar_array(m["edge_rest_angle"])
        self.edge_rest_length = wp.scalar_array(m["edge_rest_length"])
        self.edge_bending_properties = wp.array2d(m["edge_bending_properties"])
        self.empty = wp.Array([])
        self.soft_ke, self.soft_kd, self.soft_mu = soft
        self.shape_ke = wp.scalar_array([s[0] for s in shapes])
        self.shape_kd = wp.scalar_array([s[1] for s in shapes])
        self.shape_mu = wp.scalar_array([s[2] for s in shapes])
        self.shape_body = wp.scalar_array([-1 for _ in shapes], int)
        self.particle_colors = wp.scalar_array(colors, int)


class SelfContactRef:
    """Self-contact state of ``SolverVBD`` (``solver_vbd.py:489-526, 1339-1404``) and its
    ``TriMeshCollisionDetector`` (``tri_mesh_collision.py:91-413``) for a shim run."""

    def __init__(self, ns, sc: RefScene, *, radius, margin, relaxation=0.85, vertex_buffer=32, edge_buffer=64,
                 interval=0, ee_eps=1e-5, ring=2, rest_exclusion=0.0):  # fmt: skip
        self.ns, self.sc = ns, sc
        m = sc.m
        self.V, self.T, self.E = sc.n, len(m["tri_indices"]), len(m["edge_indices"])
        self.radius, self.margin, self.relaxation = radius, margin, relaxation
        self.vb, self.eb, self.interval, self.ee_eps = vertex_buffer, edge_buffer, interval, ee_eps
        self.ring, self.rest_exclusion = ring, rest_exclusion
        f_off, f_adj, e_off, e_adj = sc.adjacency_np
        self.vt_filter = self.ee_filter = (None, None)
        if ring >= 2:  # _compute_particle_contact_filtering_list (solver_vbd.py:1339-1404)
            vt_sets = ns["build_vertex_n_ring_tris_collision_filter"](ring, self.V, m["edge_indices"], e_adj, e_off, f_adj,
                                                                      f_off)  # fmt: skip
            ee_sets = ns["build_edge_n_ring_edge_collision_filter"](ring, m["edge_indices"], e_adj, e_off)
            self.vt_filter = ns["set_to_csr"](vt_sets)
            self.ee_filter = ns["set_to_csr"](ee_sets)
        self.rest_q = wp.vec_array(m["particle_q"])  # particle_q_rest = model.particle_q
        self.vt_offsets = wp.scalar_array(np.arange(self.V + 1) * vertex_buffer, int)
        self.vt_sizes = wp.scalar_array(np.full(self.V, vertex_buffer), int)
        self.ee_offsets = wp.scalar_array(np.arange(self.E + 1) * edge_buffer, int)
        self.ee_sizes = wp.scalar_array(np.full(self.E, edge_buffer), int)
        self.launch_size = max(self.V, self.E) * ns["NUM_THREADS_PER_COLLISION_PRIMITIVE"]

    def detect(self, pos):
        """``_collision_detection_penetration_free`` after its position copy (solver_vbd.py:2834-2850)."""
        ns, m = self.ns, self.sc.m
        P = wp.to_numpy(pos)
        tri, edg = m["tri_indices"], m["edge_indices"]
        bvh_tris = wp.Bvh(np.minimum(np.minimum(P[tri[:, 0]], P[tri[:, 1]]), P[tri[:, 2]]),
                          np.maximum(np.maximum(P[tri[:, 0]], P[tri[:, 1]]), P[tri[:, 2]]))  # fmt: skip
        bvh_edges = wp.Bvh(np.minimum(P[edg[:, 2]], P[edg[:, 3]]), np.maximum(P[edg[:, 2]], P[edg[:, 3]]))
        self.resize_flags = wp.scalar_array(np.zeros(4), int)
        self.vt = wp.scalar_array(-np.ones(2 * self.V * self.vb), int)
        self.vt_count = wp.scalar_array(np.zeros(self.V), int)
        self.vt_min = wp.scalar_array(np.zeros(self.V))
        tri_min = wp.scalar_array(np.full(self.T, self.margin))
        vf, vfo = self.vt_filter
        wp.launch(
            ns["vertex_triangle_collision_detection_kernel"], self.V, self.margin, self.rest_exclusion, bvh_tris, pos,
            self.sc.tri_indices, self.vt_offsets, self.vt_sizes, None, None,
            None if vf is None else wp.scalar_array(vf, int), None if vfo is None else wp.scalar_array(vfo, int),
            self.rest_q, self.vt, self.vt_count, self.vt_min, None, None, tri_min, self.resize_flags,
        )  # fmt: skip
        self.ee = wp.scalar_array(-np.ones(2 * self.E * self.eb), int)
        self.ee_count = wp.scalar_array(np.zeros(self.E), int)
        self.ee_min = wp.scalar_array(np.zeros(self.E))
        ef, efo = self.ee_filter
        wp.launch(
            ns["edge_colliding_edges_detection_kernel"], self.E, self.margin, self.rest_exclusion, bvh_edges, pos,
            self.sc.edge_indices, self.ee_offsets, self.ee_sizes, self.ee_eps,
            None if ef is None else wp.scalar_array(ef, int), None if efo is None else wp.scalar_array(efo, int),
            self.rest_q, self.ee, self.ee_count, self.ee_min, self.resize_flags,
        )  # fmt: skip
        self.info = [types.SimpleNamespace(
            vertex_colliding_triangles=self.vt, vertex_colliding_triangles_offsets=self.vt_offsets,
            vertex_colliding_triangles_buffer_sizes=self.vt_sizes, edge_colliding_edges=self.ee,
            edge_colliding_edges_offsets=self.ee_offsets, edge_colliding_edges_buffer_sizes=self.ee_sizes,
        )]  # fmt: skip

    def record(self):
        return {
            "vt": np.array(self.vt.items, dtype=np.int32), "vt_count": np.array(self.vt_count.items, dtype=np.int32),
            "vt_min": np.array(self.vt_min.items), "ee": np.array(self.ee.items, dtype=np.int32),
            "ee_count": np.array(self.ee_count.items, dtype=np.int32), "ee_min": np.array(self.ee_min.items),
            "resize_flags": np.array(self.resize_flags.items, dtype=np.int32),
        }  # fmt: skip


def ref_step(sc: RefScene, q_in, qd_in, f_ext, contacts, dt, iterations, friction_epsilon=1e-2, beta=0.0, selfc=None,
             trace=None, bodies=None):  # fmt: skip
    """One ``SolverVBD.step``; ``selfc`` turns self-contact on. ``trace`` (a list) receives the collision buffers of
    every detection. ``bodies``: shapes on bodies moved by an external rigid solver
    (``integrate_with_external_rigid_solver=True``), a dict of ``shape_body`` [S], ``body_q_in`` / ``body_q_out``
    (lists of (p, q xyzw)), ``body_qd_out`` [B, 6] and ``body_com`` [B, 3]: the contact kernels then read
    ``state_out.body_q``, ``state_in.body_q`` as the previous pose and ``state_out.body_qd``
    (solver_vbd.py:2157-2168, 2349-2374); without it every shape is static."""
    ns = sc.ns
    n = sc.n
    state_in_q = wp.vec_array(q_in)
    state_in_qd = wp.vec_array(qd_in)
    particle_f = wp.vec_array(f_ext)
    state_out_q = wp.vec_array(np.zeros((n, 3)))
    state_out_qd = wp.vec_array(np.zeros((n, 3)))
    q_prev = wp.vec_array(np.zeros((n, 3)))
    inertia = wp.vec_array(np.zeros((n, 3)))

    cmax = max(len(contacts), 1)
    cnt = wp.scalar_array([len(contacts)], int)
    c_particle = wp.scalar_array([c[0] for c in contacts] + [-1] * (cmax - len(contacts)), int)
    c_shape = wp.scalar_array([c[1] for c in contacts] + [-1] * (cmax - len(contacts)), int)
    pad = [np.zeros(3)] * (cmax - len(contacts))
    c_body_pos = wp.vec_array(np.array([c[2] for c in contacts] + pad))
    c_body_vel = wp.vec_array(np.array([c[3] for c in contacts] + pad))
    c_normal = wp.vec_array(np.array([c[4] for c in contacts] + pad))
    pen_k = wp.scalar_array(np.zeros(cmax))
    mat_kd = wp.scalar_array(np.zeros(cmax))
    mat_mu = wp.scalar_array(np.zeros(cmax))
    mat_ke = wp.scalar_array(np.zeros(cmax))
    k_start = -1.0 if beta == 0.0 else 1.0e2

    shape_body, body_q, body_q_prev, body_qd, body_com = sc.shape_body, sc.empty, None, sc.empty, sc.empty
    if bodies is not None:
        shape_body = wp.scalar_array(list(bodies["shape_body"]), int)
        body_q = [(np.asarray(p, dtype=float), np.asarray(q, dtype=float)) for p, q in bodies["body_q_out"]]
        body_q_prev = [(np.asarray(p, dtype=float), np.asarray(q, dtype=float)) for p, q in bodies["body_q_in"]]
        body_qd = [wp.spatial_vector(*v) for v in np.asarray(bodies["body_qd_out"], dtype=float)]
        body_com = wp.vec_array(np.asarray(bodies["body_com"], dtype=float).reshape(-1, 3))
    # _initialize_rigid_bodies -> init_body_particle_contacts (solver_vbd.py:2119-2149)
    wp.launch(
        ns["init_body_particle_contacts"], cmax, cnt, c_shape, sc.soft_ke, sc.soft_kd, sc.soft_mu,
        sc.shape_ke, sc.shape_kd, sc.shape_mu, k_start, pen_k, mat_kd, mat_mu, mat_ke,
    )  # fmt: skip

    # _initialize_particles (solver_vbd.py:1731-1766)
    pos_prev_cd = wp.vec_array(wp.to_numpy(state_in_q))
    disp = wp.vec_array(np.zeros((n, 3)))

    def detect():
        pos_prev_cd.items = [wp.Vec(x.a) for x in state_in_q.items]
        disp.items = [wp.vec3() for _ in range(n)]
        selfc.detect(state_in_q)
        if trace is not None:
            trace.append(selfc.record())

    if selfc is not None:
        detect()
    wp.launch(
        ns["forward_step"], n, dt, sc.gravity, q_prev, state_in_q, state_in_qd, sc.inv_mass, particle_f,
        sc.flags, inertia, disp,
    )  # fmt: skip
    ts = wp.scalar_array(np.ones(n))

    def truncate():  # _penetration_free_truncation (solver_vbd.py:1669-1729)
        ts.items = [1.0] * n
        if selfc is None:
            wp.launch(ns["apply_truncation_ts"], n, pos_prev_cd, disp, ts, wp.inf, disp, state_in_q)
            return
        wp.launch(
            ns["apply_planar_truncation_parallel_by_collision"], selfc.launch_size, pos_prev_cd, disp, sc.tri_indices,
            sc.edge_indices, selfc.info, selfc.ee_eps, selfc.relaxation, ts,
        )  # fmt: skip
        wp.launch(ns["apply_truncation_ts"], n, pos_prev_cd, disp, ts, selfc.margin * selfc.relaxation * 0.5, disp,
                  state_in_q)  # fmt: skip

    truncate()
    for _it in range(iterations):
        # _solve_rigid_body_iteration with no bodies: dual update only (solver_vbd.py:2339-2376)
        wp.launch(
            ns["update_duals_body_particle_contacts"], cmax, cnt, c_particle, c_shape, c_body_pos, c_normal,
            state_in_q, sc.radius, shape_body, body_q, mat_ke, beta, pen_k,
        )  # fmt: skip
        # _solve_particle_iteration (solver_vbd.py:2151-2337)
        if selfc is not None and ((selfc.interval == 0 and _it == 0) or (selfc.interval >= 1 and _it % selfc.interval == 0)):
            detect()
        forces = wp.vec_array(np.zeros((n, 3)))
        hessians = wp.mat33_array(np.zeros((n, 3, 3)))
        for color in range(len(sc.groups)):
            wp.launch(
                ns["accumulate_particle_body_contact_force_and_hessian"], cmax, dt, color, q_prev, state_in_q,
                sc.particle_colors, friction_epsilon, sc.radius, c_particle, cnt, cmax, pen_k, mat_kd, mat_mu,
                sc.shape_mu, shape_body, body_q, body_q_prev, body_qd, body_com, c_shape, c_body_pos, c_body_vel,
                c_normal, forces, hessians,
            )  # fmt: skip
            if sc.spring_count:  # solver_vbd.py:2224-2243
                wp.launch(
                    ns["accumulate_spring_force_and_hessian"], sc.spring_count, dt, color, q_prev, state_in_q,
                    sc.particle_colors, sc.spring_count, sc.spring_indices, sc.spring_rest_length, sc.spring_stiffness,
                    sc.spring_damping, forces, hessians,
                )  # fmt: skip
            if selfc is not None:
                wp.launch(
                    ns["accumulate_self_contact_force_and_hessian"], selfc.launch_size, dt, color, q_prev, state_in_q,
                    sc.particle_colors, sc.tri_indices, sc.edge_indices, selfc.info, selfc.radius, sc.soft_ke,
                    sc.soft_kd, sc.soft_mu, friction_epsilon, selfc.ee_eps, forces, hessians,
                )  # fmt: skip
            group = wp.scalar_array(sc.groups[color], int)
            wp.launch(
                ns["solve_elasticity"], len(sc.groups[color]), dt, group, q_prev, state_in_q, sc.mass, inertia,
                sc.flags, sc.tri_indices, sc.tri_poses, sc.tri_materials, sc.tri_areas, sc.edge_indices,
                sc.edge_rest_angle, sc.edge_rest_length, sc.edge_bending_properties, sc.tet_indices, sc.tet_poses,
                sc.tet_materials, sc.adj, forces, hessians, disp,
            )  # fmt: skip
            truncate()
        state_out_q = wp.vec_array(wp.to_numpy(state_in_q))
    wp.launch(ns["update_velocity"], n, dt, q_prev, state_out_q, state_out_qd)
    return wp.to_numpy(state_in_q), wp.to_numpy(state_out_q), wp.to_numpy(state_out_qd)


def contacts_to_arrays(contacts, cmax):
    k = len(contacts)
    particle = -np.ones(cmax, dtype=np.int32)
    shape = -np.ones(cmax, dtype=np.int32)
    body_pos = np.zeros((cmax, 3))
    body_vel = np.zeros((cmax, 3))
    normal = np.zeros((cmax, 3))
    for i, c in enumerate(contacts):
        particle[i], shape[i] = c[0], c[1]
        body_pos[i], body_vel[i], normal[i] = c[2], c[3], c[4]
    return np.int32(k), particle, shape, body_pos, body_vel, normal


# ----------------------------------------------------------------------------- scenes
def lame(E, nu, h):
    return E * h / (2.0 * (1.0 + nu)), E * h * nu / (1.0 - nu * nu)


def scene_grid(ns, *, dim, cell, pos, rot, vel, mass, mu, lam, tri_kd, edge_ke, edge_kd, radius, pinned):
    b = FakeBuilder(ns)
    b.add_cloth_grid(
        pos=wp.vec3(*pos), rot=rot, vel=wp.vec3(*vel), dim_x=dim, dim_y=dim, cell_x=cell, cell_y=cell, mass=mass,
        tri_ke=mu, tri_ka=lam, tri_kd=tri_kd, edge_ke=edge_ke, edge_kd=edge_kd, particle_radius=radius,
    )  # fmt: skip
    for p in pinned:
        b.particle_flags[p] = b.particle_flags[p] & ~ParticleFlags.ACTIVE
    return b


def run_scene(ns, name, b: FakeBuilder, *, gravity, soft, shapes, contact_fn, dt, iterations, substeps, seed, beta=0.0,
              friction_epsilon=1e-2, f_ext_scale=0.0, self_contact=None, q_start=None, qd_start=None,
              bodies=None):  # fmt: skip
    """``bodies``: dict of ``shape_body``, ``body_com`` and ``motion(s) -> (body_q_in, body_q_out, body_qd_out)``
    of substep s; ``contact_fn`` then also takes ``body_q_in`` (contacts are generated before the step)."""
    m = b.arrays()
    colors, groups = greedy_coloring(len(m["particle_q"]), m["tri_indices"], m["edge_indices"], m["edge_bending_properties"],
                                     m.get("tet_indices", ()), m.get("spring_indices", ()))  # fmt: skip
    sc = RefScene(ns, m, groups, colors, gravity, soft, shapes)
    selfc = None if self_contact is None else SelfContactRef(ns, sc, **self_contact)
    n = sc.n
    rng = np.random.default_rng(seed)
    q = m["particle_q"].copy() if q_start is None else np.asarray(q_start, dtype=np.float64).copy()
    qd = m["particle_qd"].copy() if qd_start is None else np.asarray(qd_start, dtype=np.float64).copy()
    out = {f"model_{k}": v for k, v in m.items()}
    if len(m.get("tet_indices", ())):
        out["adj_tet_offsets"], out["adj_tets"] = (a.astype(np.int32) for a in sc.tet_adjacency_np)
    if selfc is not None:
        out.update({f"sc_{k}": np.float64(v) for k, v in self_contact.items()})
        for key, (flat, offs) in (("vt_filter", selfc.vt_filter), ("ee_filter", selfc.ee_filter)):
            if flat is not None:
                out[f"sc_{key}"], out[f"sc_{key}_offsets"] = flat.astype(np.int32), offs.astype(np.int32)
    f_off, f_adj, e_off, e_adj = sc.adjacency_np
    out.update(
        adj_face_offsets=f_off.astype(np.int32), adj_faces=f_adj.astype(np.int32),
        adj_edge_offsets=e_off.astype(np.int32), adj_edges=e_adj.astype(np.int32),
        particle_colors=colors, color_offsets=np.concatenate([[0], np.cumsum([len(g) for g in groups])]).astype(np.int32),
        color_particles=np.concatenate(groups).astype(np.int32), gravity=np.asarray(gravity, dtype=np.float64),
        soft=np.asarray(soft, dtype=np.float64), shapes=np.asarray(shapes, dtype=np.float64).reshape(-1, 3),
        dt=np.float64(dt), iterations=np.int32(iterations), substeps=np.int32(substeps), beta=np.float64(beta),
        friction_epsilon=np.float64(friction_epsilon),
    )  # fmt: skip
    cmax = n * max(len(shapes), 1)
    if bodies is not None:
        out["shape_body"] = np.asarray(bodies["shape_body"], dtype=np.int32)
        out["body_com"] = np.asarray(bodies["body_com"], dtype=np.float64).reshape(-1, 3)
    for s in range(substeps):
        f_ext = rng.normal(0.0, 1.0, size=(n, 3)) * f_ext_scale
        step_bodies = None
        if bodies is not None:
            bq_in, bq_out, bqd_out = bodies["motion"](s)
            step_bodies = dict(shape_body=bodies["shape_body"], body_q_in=bq_in, body_q_out=bq_out,
                               body_qd_out=bqd_out, body_com=bodies["body_com"])  # fmt: skip
            out[f"s{s}_body_q_in"] = np.array([list(p) + list(q) for p, q in bq_in], dtype=np.float64)
            out[f"s{s}_body_q_out"] = np.array([list(p) + list(q) for p, q in bq_out], dtype=np.float64)
            out[f"s{s}_body_qd_out"] = np.asarray(bqd_out, dtype=np.float64).reshape(-1, 6)
            contacts = contact_fn(q, m["particle_radius"], m["particle_flags"], bq_in)
        else:
            contacts = contact_fn(q, m["particle_radius"], m["particle_flags"]) if contact_fn else []
        cnt, cp, cs, cbp, cbv, cn = contacts_to_arrays(contacts, cmax)
        out[f"s{s}_q_in"], out[f"s{s}_qd_in"], out[f"s{s}_f_ext"] = q.copy(), qd.copy(), f_ext
        out[f"s{s}_contact_count"], out[f"s{s}_contact_particle"], out[f"s{s}_contact_shape"] = cnt, cp, cs
        out[f"s{s}_contact_body_pos"], out[f"s{s}_contact_body_vel"], out[f"s{s}_contact_normal"] = cbp, cbv, cn
        trace = []
        q_in_after, q_out, qd_out = ref_step(sc, q, qd, f_ext, contacts, dt, iterations, friction_epsilon, beta, selfc,
                                             trace, step_bodies)  # fmt: skip
        out[f"s{s}_q_in_after"], out[f"s{s}_q_out"], out[f"s{s}_qd_out"] = q_in_after, q_out, qd_out
        for k, rec in enumerate(trace):  # collision buffers of each detection of this substep
            for key, val in rec.items():
                out[f"s{s}_cd{k}_{key}"] = val
        if trace:
            nvt = sum(int(min(c, selfc.vb)) for c in trace[0]["vt_count"])
            nee = sum(int(min(c, selfc.eb)) for c in trace[0]["ee_count"])
            print(f"  {name}: substep {s} detections={len(trace)} vt pairs={nvt} ee pairs={nee}")
        q, qd = q_out, qd_out
        print(f"  {name}: substep {s} contacts={len(contacts)} |dq|max={np.abs(q_out - out[f's{s}_q_in']).max():.3e}")
    return out


def element_cases(ns, seed=7):
    """Per-element force/Hessian goldens on random inputs, both with and without damping."""
    rng = np.random.default_rng(seed)
    mem = []
    for i in range(64):
        X = rng.normal(size=(3, 3))
        rest = np.array([[0.0, 0.0], [rng.uniform(0.5, 1.5), rng.uniform(-0.2, 0.2)], [rng.uniform(-0.3, 0.3), rng.uniform(0.5, 1.5)]])
        Dm = np.stack([rest[1] - rest[0], rest[2] - rest[0]], axis=1)
        pose = np.linalg.inv(Dm)
        area = 0.5 * np.linalg.det(Dm)
        mu, lam = rng.uniform(0.1, 10.0), rng.uniform(0.0, 10.0)
        damping = 0.0 if i % 2 == 0 else rng.uniform(1e-3, 1e-1)
        dt = 1.0 / 600.0
        Xprev = X + rng.normal(scale=1e-2, size=(3, 3))
        order = i % 3
        f, H = ns["evaluate_neo_hookean_membrane_force_hessian"](
            0, order, wp.vec_array(X), wp.vec_array(Xprev), wp.array2d([[0, 1, 2]], int), wp.mat22(pose), area, mu,
            lam, damping, dt,
        )  # fmt: skip
        mem.append(np.concatenate([X.ravel(), Xprev.ravel(), pose.ravel(), [area, mu, lam, damping, dt, order], f.a, H.a.ravel()]))
    bend = []
    for i in range(64):
        X = rng.normal(size=(4, 3))
        Xprev = X + rng.normal(scale=1e-2, size=(4, 3))
        rest_angle = rng.uniform(-1.0, 1.0)
        rest_len = rng.uniform(0.5, 2.0)
        ke = rng.uniform(1e-3, 10.0)
        kd = 0.0 if i % 2 == 0 else rng.uniform(1e-3, 1e-1)
        dt = 1.0 / 600.0
        order = i % 4
        boundary = 1 if i % 16 == 15 else 0
        eidx = [[-1 if boundary else 0, 1, 2, 3]]
        f, H = ns["evaluate_dihedral_angle_based_bending_force_hessian"](
            0, order, wp.vec_array(X), wp.vec_array(Xprev), wp.array2d(eidx, int), wp.scalar_array([rest_angle]),
            wp.scalar_array([rest_len]), ke, kd, dt,
        )  # fmt: skip
        bend.append(np.concatenate([X.ravel(), Xprev.ravel(), [rest_angle, rest_len, ke, kd, dt, order, boundary], f.a, H.a.ravel()]))
    con = []
    for i in range(64):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        pen = rng.uniform(1e-4, 1e-2)
        rel = rng.normal(scale=[1e-2, 1e-4, 1e-6][i % 3], size=3)
        ke, kd, mu = rng.uniform(1e2, 1e4), rng.uniform(0.0, 10.0), rng.uniform(0.0, 1.0)
        eps, dt = 1e-2, 1.0 / 600.0
        f, H = ns["_compute_body_particle_contact_force"](pen, wp.vec3(n), wp.vec3(rel), ke, kd, mu, eps, dt)
        con.append(np.concatenate([[pen], n, rel, [ke, kd, mu, eps, dt], f.a, H.a.ravel()]))
    return {"membrane": np.array(mem), "bending": np.array(bend), "contact": np.array(con)}


def selfcontact_cases(ns, seed=11):
    """Per-pair goldens of the self-contact terms and of the division-plane truncation."""
    rng = np.random.default_rng(seed)
    radius, ke, kd, mu, eps, dt = 0.02, 1.0e4, 1.0e-3, 0.4, 1.0e-2, 1.0 / 600.0
    vt, ee, vtp, eep, cp = [], [], [], [], []
    for i in range(96):
        a, b, c = rng.normal(scale=0.05, size=(3, 3))
        n = np.cross(b - a, c - a)
        n /= np.linalg.norm(n)
        w = rng.dirichlet([1.0, 1.0, 1.0]) if i % 3 else rng.uniform(-0.5, 1.2, size=3)
        w = w / w.sum()
        # distances covering the quadratic (< d_min), log-barrier (< r/2), linear (< r) and no-contact regions
        d = [5e-6, 0.004, 0.013, 0.025][i % 4] * (1.0 if i % 8 < 4 else -1.0)
        p = w[0] * a + w[1] * b + w[2] * c + n * d
        X = np.stack([a, b, c, p])
        Xa = X + rng.normal(scale=[1e-3, 1e-5, 1e-7][i % 3], size=(4, 3))
        res = ns["evaluate_vertex_triangle_collision_force_hessian_4_vertices"](
            3, 0, wp.vec_array(X), wp.vec_array(Xa), wp.array2d([[0, 1, 2]], int), radius, ke, kd, mu, eps, dt)
        fs = np.concatenate([np.asarray(res[1 + k].a) for k in range(4)])
        hs = np.concatenate([np.asarray(res[5 + k].a).ravel() for k in range(4)])
        vt.append(np.concatenate([X.ravel(), Xa.ravel(), [float(res[0])], fs, hs]))
        cpt, bary, feat = ns["triangle_closest_point"](wp.vec3(a), wp.vec3(b), wp.vec3(c), wp.vec3(p))
        cp.append(np.concatenate([X.ravel(), cpt.a, bary.a, [feat]]))
        disp = rng.normal(scale=0.01, size=(4, 3))
        dummy, nrm, dpt = ns["create_vertex_triangle_division_plane_closest_pt"](
            wp.vec3(p), wp.vec3(disp[3]), wp.vec3(a), wp.vec3(disp[0]), wp.vec3(b), wp.vec3(disp[1]), wp.vec3(c),
            wp.vec3(disp[2]))  # fmt: skip
        ts = [ns["planar_truncation_t"](wp.vec3(x), wp.vec3(dx), nrm, dpt, 1e-5, 0.85)
              for x, dx in ((p, disp[3]), (a, disp[0]), (b, disp[1]), (c, disp[2]))]  # fmt: skip
        vtp.append(np.concatenate([X.ravel(), disp.ravel(), [float(x) for x in dummy], nrm.a, dpt.a, ts]))
    for i in range(96):
        p1, q1 = rng.normal(scale=0.05, size=(2, 3))
        u = rng.normal(size=3)
        u -= u.dot(q1 - p1) * (q1 - p1) / np.dot(q1 - p1, q1 - p1)
        u /= np.linalg.norm(u)
        s0, t0 = rng.uniform(-0.3, 1.3, size=2)
        d = [5e-6, 0.004, 0.013, 0.025][i % 4]
        dir2 = rng.normal(size=3)
        p2c = p1 + (q1 - p1) * s0 + u * d
        p2 = p2c - dir2 * 0.05 * t0
        q2 = p2 + dir2 * 0.05
        X = np.stack([p1, q1, p2, q2])
        Xa = X + rng.normal(scale=[1e-3, 1e-5, 1e-7][i % 3], size=(4, 3))
        edges = wp.array2d([[-1, -1, 0, 1], [-1, -1, 2, 3]], int)
        res = ns["evaluate_edge_edge_contact_2_vertices"](0, 1, wp.vec_array(X), wp.vec_array(Xa), edges, radius, ke, kd,
                                                          mu, eps, dt, 1e-5)  # fmt: skip
        st = wp.closest_point_edge_edge(wp.vec3(p1), wp.vec3(q1), wp.vec3(p2), wp.vec3(q2), 1e-5)
        ee.append(np.concatenate([X.ravel(), Xa.ravel(), [float(res[0])], res[1].a, res[2].a, res[3].a.ravel(),
                                  res[4].a.ravel(), st.a]))  # fmt: skip
        disp = rng.normal(scale=0.01, size=(4, 3))
        dummy, nrm, dpt = ns["create_edge_edge_division_plane_closest_pt"](
            wp.vec3(p1), wp.vec3(disp[0]), wp.vec3(q1), wp.vec3(disp[1]), wp.vec3(p2), wp.vec3(disp[2]), wp.vec3(q2),
            wp.vec3(disp[3]))  # fmt: skip
        ts = [ns["planar_truncation_t"](wp.vec3(X[k]), wp.vec3(disp[k]), nrm, dpt, 1e-5, 0.85) for k in range(4)]
        eep.append(np.concatenate([X.ravel(), disp.ravel(), [float(x) for x in dummy], nrm.a, dpt.a, ts]))
    norm = []
    for dis in np.concatenate([np.geomspace(1e-7, 0.03, 40), [1e-5, 0.01, 0.02]]):
        dEdD, d2E = ns["evaluate_self_contact_force_norm"](float(dis), radius, ke)
        norm.append([dis, dEdD, d2E])
    return {"vt": np.array(vt), "ee": np.array(ee), "vt_plane": np.array(vtp), "ee_plane": np.array(eep),
            "closest": np.array(cp), "norm": np.array(norm)}  # fmt: skip


GEO_PLANE, GEO_SPHERE, GEO_CAPSULE, GEO_ELLIPSOID, GEO_CYLINDER, GEO_BOX = 1, 3, 4, 5, 6, 7


def shape_contact_cases(ns, seed=17):
    """Particle-shape soft contacts against static analytic shapes, computed as create_soft_contacts
    (geometry/kernels.py:1001-1140) does for shapes without a body: the particle in the shape frame, the
    shape's lifted SDF and gradient, and for d < margin + radius the contact point x_local - n d and the normal
    mapped back to world. Contacts are listed in thread-id order (particle-major), the order of a serial
    launch."""
    rng = np.random.default_rng(seed)

    def quat(axis, ang):
        return wp.quat_from_axis_angle(np.asarray(axis, dtype=float), ang)

    shapes = [  # type, position, rotation (x, y, z, w), scale
        (GEO_PLANE, (0.0, 0.0, 0.0), wp.quat_identity(), (0.0, 0.0, 0.0)),
        (GEO_PLANE, (-0.6, 0.5, 0.25), quat((1.0, 0.2, 0.0), 0.4), (0.6, 0.4, 0.0)),
        (GEO_SPHERE, (0.5, 0.0, 0.3), wp.quat_identity(), (0.25, 0.0, 0.0)),
        (GEO_BOX, (-0.4, -0.4, 0.3), quat((0.3, 1.0, 0.2), 0.7), (0.3, 0.2, 0.1)),
        (GEO_CAPSULE, (0.2, 0.6, 0.35), quat((1.0, 0.0, 0.3), 1.1), (0.1, 0.2, 0.0)),
        (GEO_CYLINDER, (0.6, -0.6, 0.2), quat((0.0, 1.0, 1.0), 0.5), (0.15, 0.1, 0.0)),
        (GEO_ELLIPSOID, (-0.1, 0.0, 0.5), quat((1.0, 1.0, 0.0), 0.9), (0.3, 0.2, 0.15)),
    ]
    n = 6000
    q = np.stack([rng.uniform(-1.0, 1.0, n), rng.uniform(-1.0, 1.0, n), rng.uniform(-0.1, 0.8, n)], axis=1)
    radius = rng.uniform(0.005, 0.02, n)
    flags = np.where(rng.uniform(size=n) < 0.9, 1, 0).astype(np.int32)
    margin = 0.02
    out = {k: [] for k in ("particle", "shape", "body_pos", "body_vel", "normal", "distance")}
    for i in range(n):
        if not (flags[i] & 1):
            continue
        for s, (typ, pos, rot, sc) in enumerate(shapes):
            X_ws = (np.asarray(pos, dtype=float), np.asarray(rot, dtype=float))
            X_sw = wp.transform_inverse(X_ws)
            x_local = wp.transform_point(X_sw, wp.vec3(*q[i]))
            scale = wp.vec3(*sc)
            d, nn, v = 1.0e6, wp.vec3(), wp.vec3()
            if typ == GEO_SPHERE:
                d, nn = ns["sdf_sphere"](x_local, scale[0]), ns["sdf_sphere_grad"](x_local, scale[0])
            if typ == GEO_BOX:
                d = ns["sdf_box"](x_local, scale[0], scale[1], scale[2])
                nn = ns["sdf_box_grad"](x_local, scale[0], scale[1], scale[2])
            if typ == GEO_CAPSULE:
                d = ns["sdf_capsule"](x_local, scale[0], scale[1], 2)
                nn = ns["sdf_capsule_grad"](x_local, scale[0], scale[1], 2)
            if typ == GEO_CYLINDER:
                d = ns["sdf_cylinder"](x_local, scale[0], scale[1], 2)
                nn = ns["sdf_cylinder_grad"](x_local, scale[0], scale[1], 2)
            if typ == GEO_ELLIPSOID:
                d, nn = ns["sdf_ellipsoid"](x_local, scale), ns["sdf_ellipsoid_grad"](x_local, scale)
            if typ == GEO_PLANE:
                d, nn = ns["sdf_plane"](x_local, scale[0] * 0.5, scale[1] * 0.5), wp.vec3(0.0, 0.0, 1.0)
            if d < margin + radius[i]:
                out["particle"].append(i)
                out["shape"].append(s)
                out["body_pos"].append(np.asarray(wp.transform_point(X_ws, x_local - nn * d)))
                out["body_vel"].append(np.asarray(wp.transform_vector(X_ws, v)))
                out["normal"].append(np.asarray(wp.transform_vector(X_ws, nn)))
                out["distance"].append(d)
    res = {k: np.asarray(v) for k, v in out.items()}
    res["particle"] = res["particle"].astype(np.int32)
    res["shape"] = res["shape"].astype(np.int32)
    res.update(
        q=q, radius=radius, flags=flags, margin=np.float64(margin),
        shape_type=np.array([t for t, _, _, _ in shapes], dtype=np.int32),
        shape_transform=np.array([list(p) + list(r) for _, p, r, _ in shapes], dtype=np.float64),
        shape_scale=np.array([sc for _, _, _, sc in shapes], dtype=np.float64),
    )  # fmt: skip
    return res


GEO_HFIELD, GEO_CONE = 2, 9


def shape_contact_cases_cone_hfield(ns, seed=19):
    """Particle contacts against cones (``sdf_cone``/``sdf_cone_grad``, geometry/kernels.py:515-564) and
    heightfields (``sample_sdf_grad_heightfield``, utils/heightfield.py:178-205) through create_soft_contacts'
    frame handling, for shapes without a body. The heightfields' extents carry the shape scale as the reference
    builder bakes it (sim/builder.py:10698-10718): hx |sx|, hy |sy|, min_z sz, max_z sz; elevations are normalized
    to [0, 1] as ``Heightfield`` stores them (geometry/types.py:2128-2134). One grid has a single row and gives no
    contacts."""
    rng = np.random.default_rng(seed)

    def quat(axis, ang):
        return wp.quat_from_axis_angle(np.asarray(axis, dtype=float), ang)

    grids = []  # (raw elevations, hx, hy, min_z, max_z, scale)
    gx, gy = np.meshgrid(np.linspace(-1.0, 1.0, 17), np.linspace(-1.0, 1.0, 13))
    grids.append((np.sin(2.0 * gx) * np.cos(3.0 * gy), 0.8, 0.6, -0.05, 0.15, (1.0, 1.0, 1.0)))
    grids.append((rng.uniform(0.0, 1.0, (9, 7)), 0.3, 0.4, 0.0, 0.1, (1.5, -0.5, 2.0)))
    grids.append((rng.uniform(0.0, 1.0, (1, 5)), 0.3, 0.3, 0.0, 0.1, (1.0, 1.0, 1.0)))
    shapes = [  # type, position, rotation (x, y, z, w), scale (cones), heightfield index
        (GEO_CONE, (0.4, 0.3, 0.3), wp.quat_identity(), (0.25, 0.2, 0.0), -1),
        (GEO_CONE, (-0.5, 0.5, 0.35), quat((1.0, 0.3, 0.2), 2.2), (0.2, 0.3, 0.0), -1),
        (GEO_CONE, (0.5, -0.5, 0.25), quat((0.2, 1.0, 0.0), 0.8), (0.3, 0.0, 0.0), -1),
        (GEO_HFIELD, (0.0, 0.0, 0.1), quat((0.0, 0.0, 1.0), 0.3), (1.0, 1.0, 1.0), 0),
        (GEO_HFIELD, (-0.4, -0.4, 0.3), quat((1.0, 0.5, 0.0), 0.25), (1.5, -0.5, 2.0), 1),
        (GEO_HFIELD, (0.5, 0.6, 0.2), wp.quat_identity(), (1.0, 1.0, 1.0), 2),
    ]
    elevations, hdata, off = [], [], 0
    for raw, hx, hy, zmin, zmax, sc in grids:
        raw = np.asarray(raw, dtype=np.float32)
        lo, hi = float(raw.min()), float(raw.max())
        data = (raw - lo) / (hi - lo) if hi > lo else np.zeros_like(raw)
        hdata.append(types.SimpleNamespace(data_offset=off, nrow=raw.shape[0], ncol=raw.shape[1],
                                           hx=abs(hx * sc[0]), hy=abs(hy * sc[1]), min_z=zmin * sc[2],
                                           max_z=zmax * sc[2]))  # fmt: skip
        elevations.append(data.astype(np.float32).reshape(-1))
        off += data.size
    elev = np.concatenate(elevations).astype(np.float64)
    n = 6000
    q = np.stack([rng.uniform(-1.0, 1.0, n), rng.uniform(-1.0, 1.0, n), rng.uniform(-0.1, 0.7, n)], axis=1)
    radius = rng.uniform(0.005, 0.02, n)
    flags = np.where(rng.uniform(size=n) < 0.9, 1, 0).astype(np.int32)
    margin = 0.02
    out = {k: [] for k in ("particle", "shape", "body_pos", "body_vel", "normal", "distance")}
    for i in range(n):
        if not (flags[i] & 1):
            continue
        for s, (typ, pos, rot, sc, hk) in enumerate(shapes):
            X_ws = (np.asarray(pos, dtype=float), np.asarray(rot, dtype=float))
            x_local = wp.transform_point(wp.transform_inverse(X_ws), wp.vec3(*q[i]))
            scale = wp.vec3(*sc)
            d, nn, v = 1.0e6, wp.vec3(), wp.vec3()
            if typ == GEO_CONE:
                d = ns["sdf_cone"](x_local, scale[0], scale[1], 2)
                nn = ns["sdf_cone_grad"](x_local, scale[0], scale[1], 2)
            if typ == GEO_HFIELD:
                d, nn = ns["sample_sdf_grad_heightfield"](hdata[hk], elev, x_local)
            if d < margin + radius[i]:
                out["particle"].append(i)
                out["shape"].append(s)
                out["body_pos"].append(np.asarray(wp.transform_point(X_ws, x_local - nn * d)))
                out["body_vel"].append(np.asarray(wp.transform_vector(X_ws, v)))
                out["normal"].append(np.asarray(wp.transform_vector(X_ws, nn)))
                out["distance"].append(d)
    res = {k: np.asarray(v) for k, v in out.items()}
    res["particle"] = res["particle"].astype(np.int32)
    res["shape"] = res["shape"].astype(np.int32)
    res.update(
        q=q, radius=radius, flags=flags, margin=np.float64(margin),
        shape_type=np.array([t for t, _, _, _, _ in shapes], dtype=np.int32),
        shape_transform=np.array([list(p) + list(r) for _, p, r, _, _ in shapes], dtype=np.float64),
        shape_scale=np.array([sc for _, _, _, sc, _ in shapes], dtype=np.float64),
        shape_heightfield_index=np.array([k for _, _, _, _, k in shapes], dtype=np.int32),
        heightfields=np.array([[h.data_offset, h.nrow, h.ncol, h.hx, h.hy, h.min_z, h.max_z] for h in hdata]),
        elevations=elev.astype(np.float32),
    )  # fmt: skip
    return res


def create_soft_contacts_cases(ns, seed=23):
    """The reference's ``create_soft_contacts`` kernel (geometry/kernels.py:1001-1140) run as-is, one serial launch
    over every (particle, shape) thread, so the contact list comes in thread order (particle-major). Three worlds
    with their own shapes, global shapes, a shape without COLLIDE_PARTICLES, particles in every world and global
    ones, inactive particles; planes, sphere, box, capsule, cylinder, cone, ellipsoid and a heightfield."""
    rng = np.random.default_rng(seed)

    def quat(axis, ang):
        return wp.quat_from_axis_angle(np.asarray(axis, dtype=float), ang)

    gx, gy = np.meshgrid(np.linspace(-1.0, 1.0, 9), np.linspace(-1.0, 1.0, 7))
    raw = (0.1 * np.sin(2.0 * gx) * np.cos(3.0 * gy)).astype(np.float32)
    elev = ((raw - raw.min()) / (raw.max() - raw.min())).astype(np.float32).reshape(-1)
    hfd = types.SimpleNamespace(data_offset=0, nrow=7, ncol=9, hx=0.5, hy=0.4, min_z=0.0, max_z=0.12)
    shapes = [  # type, position, rotation, scale, world, flags
        (GEO_PLANE, (0.0, 0.0, 0.0), wp.quat_identity(), (0.0, 0.0, 0.0), -1, 4),
        (GEO_SPHERE, (0.2, 0.1, 0.25), wp.quat_identity(), (0.2, 0.0, 0.0), 0, 4),
        (GEO_BOX, (-0.2, 0.0, 0.25), quat((0.3, 1.0, 0.2), 0.7), (0.2, 0.15, 0.1), 1, 4),
        (GEO_CAPSULE, (0.0, 0.2, 0.3), quat((1.0, 0.0, 0.3), 1.1), (0.1, 0.2, 0.0), 2, 4),
        (GEO_CONE, (0.1, -0.2, 0.3), quat((0.2, 1.0, 0.0), 0.8), (0.25, 0.2, 0.0), 0, 4),
        (GEO_CYLINDER, (0.0, 0.0, 0.3), quat((0.0, 1.0, 1.0), 0.5), (0.15, 0.1, 0.0), -1, 0),
        (GEO_ELLIPSOID, (-0.1, -0.1, 0.45), quat((1.0, 1.0, 0.0), 0.9), (0.25, 0.2, 0.15), -1, 4),
        (GEO_HFIELD, (0.0, 0.0, 0.02), quat((0.0, 0.0, 1.0), 0.3), (1.0, 1.0, 1.0), 2, 4),
        (GEO_PLANE, (0.3, 0.3, 0.2), quat((1.0, 0.2, 0.0), 0.4), (0.6, 0.4, 0.0), 1, 4),
    ]
    n = 2400
    q = np.stack([rng.uniform(-0.6, 0.6, n), rng.uniform(-0.6, 0.6, n), rng.uniform(-0.05, 0.6, n)], axis=1)
    radius = rng.uniform(0.005, 0.02, n)
    flags = np.where(rng.uniform(size=n) < 0.9, 1, 0).astype(np.int32)
    pworld = rng.integers(-1, 3, n).astype(np.int32)
    S, margin, cmax = len(shapes), 0.02, n * len(shapes)
    shape_type = np.array([sh[0] for sh in shapes], dtype=np.int32)
    shape_world = np.array([sh[4] for sh in shapes], dtype=np.int32)
    shape_flags = np.array([sh[5] for sh in shapes], dtype=np.int32)
    xforms = [(np.asarray(sh[1], dtype=float), np.asarray(sh[2], dtype=float)) for sh in shapes]
    scales = [wp.vec3(*sh[3]) for sh in shapes]
    count, tids = [0], [0] * (n * S)
    out_p, out_s = [0] * cmax, [0] * cmax
    out_bp, out_bv, out_n = [None] * cmax, [None] * cmax, [None] * cmax
    hf_index = np.array([0 if t == GEO_HFIELD else -1 for t in shape_type], dtype=np.int32)
    wp.launch(ns["create_soft_contacts"], n * S, [wp.vec3(*x) for x in q], radius, flags, pworld, [],
              xforms, [-1] * S, shape_type, scales, [0] * S, shape_world, margin, cmax, S, shape_flags, hf_index,
              [hfd], elev.astype(np.float64), count, out_p, out_s, out_bp, out_bv, out_n, tids)  # fmt: skip
    k = count[0]
    return dict(
        q=q, radius=radius, flags=flags, particle_world=pworld, margin=np.float64(margin), shape_type=shape_type,
        shape_world=shape_world, shape_flags=shape_flags,
        shape_transform=np.array([list(sh[1]) + list(sh[2]) for sh in shapes], dtype=np.float64),
        shape_scale=np.array([sh[3] for sh in shapes], dtype=np.float64), shape_heightfield_index=hf_index,
        heightfields=np.array([[0, 7, 9, 0.5, 0.4, 0.0, 0.12]]), elevations=elev,
        particle=np.array(out_p[:k], dtype=np.int32), shape=np.array(out_s[:k], dtype=np.int32),
        body_pos=np.array([np.asarray(v) for v in out_bp[:k]]), body_vel=np.array([np.asarray(v) for v in out_bv[:k]]),
        normal=np.array([np.asarray(v) for v in out_n[:k]]),
    )  # fmt: skip


def run_create_soft_contacts(ns, q, radius, flags, shapes, body_q, margin):
    """The reference's ``create_soft_contacts`` kernel run as-is (serially, in thread order) for global particles
    against ``shapes`` = [(type, position, rotation, scale, body)] (transforms in the body's frame) with the body
    transforms ``body_q`` = [(p, q xyzw)]: the contacts as (particle, shape, body_pos, body_vel, normal)."""
    n, S = len(q), len(shapes)
    cmax = n * S
    count, tids = [0], [0] * (n * S)
    out_p, out_s = [0] * cmax, [0] * cmax
    out_bp, out_bv, out_n = [None] * cmax, [None] * cmax, [None] * cmax
    xforms = [(np.asarray(sh[1], dtype=float), np.asarray(sh[2], dtype=float)) for sh in shapes]
    wp.launch(ns["create_soft_contacts"], n * S, [wp.vec3(*x) for x in q], radius, flags, [-1] * n,
              [(np.asarray(p, dtype=float), np.asarray(r, dtype=float)) for p, r in body_q], xforms,
              [sh[4] for sh in shapes], [sh[0] for sh in shapes], [wp.vec3(*sh[3]) for sh in shapes], [0] * S,
              [-1] * S, margin, cmax, S, [4] * S, [-1] * S, [], np.zeros(1), count, out_p, out_s, out_bp, out_bv,
              out_n, tids)  # fmt: skip
    k = count[0]
    return [(out_p[i], out_s[i], np.asarray(out_bp[i]), np.asarray(out_bv[i]), np.asarray(out_n[i])) for i in range(k)]


def create_soft_contacts_body_cases(ns, seed=29):
    """``create_soft_contacts`` with shapes on two bodies (geometry/kernels.py:1045-1056, 1128-1140): each shape's
    world frame is body_q[body] times its own transform; contact points come out in the body's frame and normals in
    world. A static ground plane and sphere, box, capsule, cylinder, cone and ellipsoid on rotated, displaced
    bodies; 1600 seeded global particles, some inactive."""
    rng = np.random.default_rng(seed)

    def quat(axis, ang):
        return np.asarray(wp.quat_from_axis_angle(np.asarray(axis, dtype=float), ang), dtype=float)

    body_q = [(np.array([0.1, -0.05, 0.2]), quat((0.3, 0.2, 1.0), 0.6)),
              (np.array([-0.15, 0.1, 0.3]), quat((1.0, -0.4, 0.2), 1.2))]  # fmt: skip
    shapes = [  # type, position, rotation, scale, body
        (GEO_PLANE, (0.0, 0.0, 0.0), quat((0.0, 0.0, 1.0), 0.0), (0.0, 0.0, 0.0), -1),
        (GEO_SPHERE, (0.05, 0.0, 0.02), quat((0.0, 0.0, 1.0), 0.0), (0.12, 0.0, 0.0), 0),
        (GEO_BOX, (0.0, 0.1, -0.05), quat((0.2, 1.0, 0.3), 0.5), (0.1, 0.08, 0.06), 0),
        (GEO_CAPSULE, (0.05, -0.05, 0.0), quat((1.0, 0.0, 0.2), 0.9), (0.05, 0.12, 0.0), 1),
        (GEO_ELLIPSOID, (-0.05, 0.05, 0.05), quat((0.0, 1.0, 1.0), 0.4), (0.1, 0.07, 0.05), 1),
        (GEO_CYLINDER, (0.1, 0.0, 0.1), quat((1.0, 1.0, 0.0), 0.3), (0.06, 0.08, 0.0), 1),
        (GEO_CONE, (-0.1, -0.1, -0.05), quat((0.2, 1.0, 0.0), 0.8), (0.08, 0.1, 0.0), 0),
    ]
    n, margin = 1600, 0.02
    q = np.stack([rng.uniform(-0.45, 0.45, n), rng.uniform(-0.45, 0.45, n), rng.uniform(-0.05, 0.55, n)], axis=1)
    radius = rng.uniform(0.005, 0.02, n)
    flags = np.where(rng.uniform(size=n) < 0.9, 1, 0).astype(np.int32)
    c = run_create_soft_contacts(ns, q, radius, flags, shapes, body_q, margin)
    return dict(
        q=q, radius=radius, flags=flags, margin=np.float64(margin),
        shape_type=np.array([sh[0] for sh in shapes], dtype=np.int32),
        shape_transform=np.array([list(sh[1]) + list(sh[2]) for sh in shapes], dtype=np.float64),
        shape_scale=np.array([sh[3] for sh in shapes], dtype=np.float64),
        shape_body=np.array([sh[4] for sh in shapes], dtype=np.int32),
        body_q=np.array([list(p) + list(r) for p, r in body_q], dtype=np.float64),
        particle=np.array([x[0] for x in c], dtype=np.int32), shape=np.array([x[1] for x in c], dtype=np.int32),
        body_pos=np.array([x[2] for x in c]).reshape(-1, 3), body_vel=np.array([x[3] for x in c]).reshape(-1, 3),
        normal=np.array([x[4] for x in c]).reshape(-1, 3),
    )  # fmt: skip


def body_motion(p0, axis, w, v, dt):
    """Pose of a body moving at constant linear velocity v and angular velocity w about a fixed axis from (p0, I):
    motion(s) -> ([(p, q) at step s], [(p, q) at step s + 1], [(v, w axis)]) for one body."""
    axis = np.asarray(axis, dtype=float) / np.linalg.norm(axis)

    def pose(t):
        return (np.asarray(p0, dtype=float) + np.asarray(v, dtype=float) * t,
                np.asarray(wp.quat_from_axis_angle(axis, w * t), dtype=float))  # fmt: skip

    return lambda s: (pose(s * dt), pose((s + 1) * dt), np.concatenate([np.asarray(v, dtype=float), axis * w]))


def soft_cases(ns, seed=13):
    """Per-element goldens of the volumetric Neo-Hookean tetrahedron and of the spring."""
    rng = np.random.default_rng(seed)
    tet, spr = [], []
    for i in range(64):
        rest = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]) * rng.uniform(0.02, 0.2)
        rest += rng.normal(scale=0.01, size=(4, 3))
        Dm = (rest[1:] - rest[0]).T
        if np.linalg.det(Dm) <= 0.0:
            rest[[1, 2]] = rest[[2, 1]]
            Dm = (rest[1:] - rest[0]).T
        X = rest @ (np.eye(3) + rng.normal(scale=0.2, size=(3, 3))).T + rng.normal(size=3)
        Xp = X + rng.normal(scale=1e-3, size=(4, 3))
        mu, lam = rng.uniform(1e2, 1e5), rng.uniform(0.0, 1e5)
        damping = 0.0 if i % 2 == 0 else rng.uniform(1e-4, 1e-2)
        dt, order = 1.0 / 600.0, i % 4
        f, H = ns["evaluate_volumetric_neo_hookean_force_and_hessian"](
            0, order, wp.vec_array(Xp), wp.vec_array(X), wp.array2d([[0, 1, 2, 3]], int), wp.mat33(np.linalg.inv(Dm)),
            mu, lam, damping, dt)  # fmt: skip
        tet.append(np.concatenate([X.ravel(), Xp.ravel(), np.linalg.inv(Dm).ravel(), [mu, lam, damping, dt, order], f.a,
                                   H.a.ravel()]))  # fmt: skip
    for i in range(32):
        X = rng.normal(scale=0.1, size=(2, 3))
        Xa = X + rng.normal(scale=1e-3, size=(2, 3))
        rest, ke, kd, dt = rng.uniform(0.05, 0.3), rng.uniform(1.0, 1e4), [0.0, 1e-2][i % 2], 1.0 / 600.0
        v0, v1, f0, f1, H = ns["evaluate_spring_force_and_hessian_both_vertices"](
            0, dt, wp.vec_array(X), wp.vec_array(Xa), wp.scalar_array([0, 1], int), wp.scalar_array([rest]),
            wp.scalar_array([ke]), wp.scalar_array([kd]))  # fmt: skip
        spr.append(np.concatenate([X.ravel(), Xa.ravel(), [rest, ke, kd, dt], f0.a, f1.a, H.a.ravel()]))
    return {"tet": np.array(tet), "spring": np.array(spr)}


def rot_z(deg):
    return wp.quat_from_axis_angle(wp.vec3(0.0, 0.0, 1.0), math.radians(deg))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("VBD_REFERENCE_ROOT"),
                    help="root of the reference checkout (default: $VBD_REFERENCE_ROOT)")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    if not args.ref:
        ap.error("name the reference checkout with --ref or VBD_REFERENCE_ROOT")
    ns = load_reference(args.ref)

    np.savez_compressed(os.path.join(args.out, "elements.npz"), **element_cases(ns))
    print("elements.npz written")

    # Hanging grid above the ground, two top corners pinned, membrane and bending damping on,
    # drifting sideways into the ground so that penetration, damping and both friction regimes occur.
    mu, lam = lame(1.0e4, 0.3, 1.0e-3)
    dim = 7
    rot = wp.quat_from_axis_angle(wp.vec3(1.0, 0.0, 0.0), math.pi * 0.5)
    b = scene_grid(
        ns, dim=dim, cell=1.0 / dim, pos=(0.0, 0.0, 0.004), rot=rot, vel=(0.3, 0.0, -0.5), mass=0.2 / (dim + 1) ** 2,
        mu=mu, lam=lam, tri_kd=1e-2, edge_ke=5e-3, edge_kd=1e-3, radius=5e-3,
        pinned=[(dim + 1) * dim, (dim + 1) * (dim + 1) - 1],
    )  # fmt: skip
    # The rotation maps grid y to world z: particles of the bottom row start 4 mm above the
    # ground, inside the contact margin.
    out = run_scene(
        ns, "grid_ground", b, gravity=(0.0, 0.0, -9.81), soft=(1.0e3, 10.0, 0.5), shapes=[(2.5e3, 100.0, 1.0)],
        contact_fn=lambda q, r, f: plane_contacts(q, r, f, margin=0.01), dt=1.0 / 600.0, iterations=4, substeps=3,
        seed=1, f_ext_scale=1e-4,
    )  # fmt: skip
    np.savez_compressed(os.path.join(args.out, "step_grid_ground.npz"), **out)

    # Same grid lying flat and dropped on a static sphere; AVBD penalty ramp (beta > 0) on.
    b = scene_grid(
        ns, dim=6, cell=0.1, pos=(-0.3, -0.3, 0.205), rot=wp.quat_identity(), vel=(0.0, 0.0, -1.0), mass=1e-3,
        mu=mu, lam=lam, tri_kd=0.0, edge_ke=1e-4, edge_kd=0.0, radius=5e-3, pinned=[],
    )  # fmt: skip
    out = run_scene(
        ns, "grid_sphere", b, gravity=(0.0, 0.0, -9.81), soft=(1.0e4, 1.0, 0.4), shapes=[(1.0e4, 1.0, 0.6)],
        contact_fn=lambda q, r, f: sphere_contacts(q, r, f, 0.01, np.zeros(3), 0.2), dt=1.0 / 600.0, iterations=5,
        substeps=3, seed=2, beta=1.0e5,
    )  # fmt: skip
    np.savez_compressed(os.path.join(args.out, "step_grid_sphere.npz"), **out)

    # The non-flat fixture of test_cloth.py:551-609 (complex rest angles), y-up gravity of -1000.
    vs = np.array(_complex_rest_angle_mesh(args.ref)[0], dtype=np.float64)
    fs = _complex_rest_angle_mesh(args.ref)[1]
    b = FakeBuilder(ns)
    b.add_cloth_mesh(
        pos=wp.vec3(0.0, 2.0, 0.0), rot=wp.quat_identity(), scale=1.0, vel=wp.vec3(0.0, 0.0, 0.0),
        vertices=[wp.vec3(*v) for v in vs], indices=fs, density=0.02, tri_ke=1e3, tri_ka=1e3, tri_kd=1e-2,
        edge_ke=1e3, edge_kd=1e-3,
    )  # fmt: skip
    b.particle_flags[1] = 0
    out = run_scene(
        ns, "complex_rest_angle", b, gravity=(0.0, -1000.0, 0.0), soft=(1.0e4, 1e-2, 0.5), shapes=[],
        contact_fn=None, dt=1.0 / 600.0, iterations=5, substeps=3, seed=3,
    )  # fmt: skip
    np.savez_compressed(os.path.join(args.out, "step_complex_rest_angle.npz"), **out)

    np.savez_compressed(os.path.join(args.out, "selfcontact_elements.npz"), **selfcontact_cases(ns))
    print("selfcontact_elements.npz written")

    np.savez_compressed(os.path.join(args.out, "soft_elements.npz"), **soft_cases(ns))
    np.savez_compressed(os.path.join(args.out, "soft_contact_shapes.npz"), **shape_contact_cases(ns))
    print("soft_contact_shapes.npz written")
    np.savez_compressed(os.path.join(args.out, "soft_contact_cone_hfield.npz"), **shape_contact_cases_cone_hfield(ns))
    print("soft_contact_cone_hfield.npz written")
    np.savez_compressed(os.path.join(args.out, "create_soft_contacts.npz"), **create_soft_contacts_cases(ns))
    print("create_soft_contacts.npz written")
    np.savez_compressed(os.path.join(args.out, "create_soft_contacts_bodies.npz"), **create_soft_contacts_body_cases(ns))
    print("create_soft_contacts_bodies.npz written")

    # A flat grid pressed onto a box and a sphere carried by two bodies that an external rigid solver moves
    # (translating and turning) under it, over a static ground plane: contacts generated by create_soft_contacts
    # from state_in.body_q, the step reading state_out.body_q, state_in.body_q and state_out.body_qd.
    dt_b = 1.0 / 600.0
    b = scene_grid(
        ns, dim=7, cell=0.05, pos=(-0.175, -0.175, 0.204), rot=wp.quat_identity(), vel=(0.05, 0.0, -0.6), mass=1e-3,
        mu=mu, lam=lam, tri_kd=0.0, edge_ke=1e-4, edge_kd=0.0, radius=5e-3, pinned=[],
    )  # fmt: skip
    moving = [body_motion((0.0, 0.0, 0.1), (0.0, 0.0, 1.0), 3.0, (0.4, 0.1, 0.5), dt_b),
              body_motion((0.1, 0.1, 0.1), (1.0, 1.0, 0.0), -2.0, (-0.3, 0.2, 0.8), dt_b)]  # fmt: skip
    body_shapes = [  # type, position, rotation, scale, body
        (GEO_PLANE, (0.0, 0.0, 0.0), np.array([0.0, 0.0, 0.0, 1.0]), (0.0, 0.0, 0.0), -1),
        (GEO_BOX, (0.0, -0.05, 0.05), np.asarray(wp.quat_from_axis_angle(np.array([0.0, 0.0, 1.0]), 0.3)),
         (0.12, 0.1, 0.05), 0),
        (GEO_SPHERE, (0.0, 0.0, 0.0), np.array([0.0, 0.0, 0.0, 1.0]), (0.1, 0.0, 0.0), 1),
    ]  # fmt: skip

    def motion(s):
        parts = [m_(s) for m_ in moving]
        return [p[0] for p in parts], [p[1] for p in parts], np.stack([p[2] for p in parts])

    out = run_scene(
        ns, "grid_bodies", b, gravity=(0.0, 0.0, -9.81), soft=(1.0e4, 1.0e-2, 0.5),
        shapes=[(2.5e3, 1.0, 0.8), (5.0e3, 1.0, 0.6), (4.0e3, 2.0, 0.4)],
        contact_fn=lambda q, r, f, bq: run_create_soft_contacts(ns, q, r, f, body_shapes, bq, 0.01), dt=dt_b,
        iterations=5, substeps=3, seed=5,
        bodies=dict(shape_body=[sh[4] for sh in body_shapes], body_com=[(0.01, 0.0, 0.0), (0.0, 0.0, 0.0)],
                    motion=motion),
    )  # fmt: skip
    out["shape_type"] = np.array([sh[0] for sh in body_shapes], dtype=np.int32)
    out["shape_transform"] = np.array([list(sh[1]) + list(sh[2]) for sh in body_shapes], dtype=np.float64)
    out["shape_scale"] = np.array([sh[3] for sh in body_shapes], dtype=np.float64)
    np.savez_compressed(os.path.join(args.out, "step_grid_bodies.npz"), **out)
    print("soft_elements.npz written")

    # Volumetric: a 3 x 2 x 2-cell tetrahedral block (add_soft_grid, 5 tetrahedra per cell, damped), 4 mm
    # above the ground and moving down and sideways, hung from a fixed anchor particle by three springs and
    # braced by one diagonal spring.
    b = SoftBuilder(ns)
    b.add_soft_grid(
        pos=wp.vec3(0.0, 0.0, 0.004), rot=wp.quat_identity(), vel=wp.vec3(0.2, 0.0, -0.8), dim_x=3, dim_y=2,
        dim_z=2, cell_x=0.05, cell_y=0.05, cell_z=0.05, density=500.0, k_mu=2.0e4, k_lambda=3.0e4, k_damp=1.0e-3,
        particle_radius=5e-3,
    )  # fmt: skip
    nv = len(b.particle_q)
    anchor = b.add_particle(wp.vec3(0.075, 0.05, 0.4), wp.vec3(0.0, 0.0, 0.0), 0.0, 5e-3)
    for corner in (nv - 1, nv - 4, nv - 12):
        b.add_spring(anchor, corner, 2.0e2, 1.0e-2, 0.0)
    b.add_spring(0, nv - 1, 5.0e2, 0.0, 0.0)
    out = run_scene(
        ns, "soft_block", b, gravity=(0.0, 0.0, -9.81), soft=(1.0e4, 1.0, 0.5), shapes=[(1.0e4, 1.0, 0.6)],
        contact_fn=lambda q, r, f: plane_contacts(q, r, f, margin=0.01), dt=1.0 / 600.0, iterations=5, substeps=3,
        seed=6,
    )  # fmt: skip
    np.savez_compressed(os.path.join(args.out, "step_soft_block.npz"), **out)

    # Self-contact: a sheet pinned at its corners and a second sheet, turned by 17 degrees about z,
    # falling onto it from 15 mm. Vertex noise of 2 mm keeps edge pairs away from the parallel case.
    b = FakeBuilder(ns)
    mass = 0.2 * 0.01
    b.add_cloth_grid(
        pos=wp.vec3(-0.3, -0.3, 0.0), rot=wp.quat_identity(), vel=wp.vec3(0.0, 0.0, 0.0), dim_x=6, dim_y=6,
        cell_x=0.1, cell_y=0.1, mass=mass, tri_ke=mu, tri_ka=lam, tri_kd=1e-3, edge_ke=1e-3, edge_kd=0.0,
        particle_radius=5e-3,
    )  # fmt: skip
    for p in (0, 6, 42, 48):
        b.particle_flags[p] = 0
    rz = rot_z(17.0)
    c = wp.transform_vector((np.zeros(3), rz), wp.vec3(0.3, 0.3, 0.0))
    b.add_cloth_grid(
        pos=wp.vec3(-c[0], -c[1], 0.015), rot=rz, vel=wp.vec3(0.0, 0.0, -2.0), dim_x=6, dim_y=6, cell_x=0.1,
        cell_y=0.1, mass=mass, tri_ke=mu, tri_ka=lam, tri_kd=1e-3, edge_ke=1e-3, edge_kd=0.0, particle_radius=5e-3,
    )  # fmt: skip
    rng = np.random.default_rng(21)
    q0 = np.array(b.particle_q) + rng.normal(scale=2e-3, size=(len(b.particle_q), 3))
    out = run_scene(
        ns, "sc_two_layers", b, gravity=(0.0, 0.0, -9.81), soft=(1.0e2, 1.0e-3, 0.4), shapes=[], contact_fn=None,
        dt=1.0 / 600.0, iterations=4, substeps=3, seed=4, q_start=q0,
        self_contact=dict(radius=0.02, margin=0.035, relaxation=0.85, interval=0, ring=2),
    )  # fmt: skip
    np.savez_compressed(os.path.join(args.out, "step_selfcontact_layers.npz"), **out)

    # Self-contact: a sheet folded onto itself (upper half 16 mm above the lower half, moving down at
    # 1.5 m/s), dt = 1/100 so that the isotropic displacement bound acts; 3-ring filter, rest-shape
    # exclusion radius, collision detection every second iteration.
    b = FakeBuilder(ns)
    b.add_cloth_grid(
        pos=wp.vec3(0.0, 0.0, 0.0), rot=wp.quat_identity(), vel=wp.vec3(0.0, 0.0, 0.0), dim_x=8, dim_y=8, cell_x=0.05,
        cell_y=0.05, mass=0.2 * 0.0025, tri_ke=mu, tri_ka=lam, tri_kd=0.0, edge_ke=1e-3, edge_kd=1e-4,
        particle_radius=5e-3,
    )  # fmt: skip
    q0 = np.array(b.particle_q)
    qd0 = np.zeros_like(q0)
    upper = q0[:, 0] > 0.2 + 1e-9
    q0[upper, 0] = 0.4 - q0[upper, 0]
    q0[upper, 2] = 0.016
    qd0[upper, 2] = -1.5
    rng = np.random.default_rng(22)
    q0 += rng.normal(scale=1.5e-3, size=q0.shape)
    out = run_scene(
        ns, "sc_fold", b, gravity=(0.0, 0.0, -9.81), soft=(2.0e3, 1.0e-2, 0.6), shapes=[], contact_fn=None,
        dt=1.0 / 100.0, iterations=4, substeps=3, seed=5, q_start=q0, qd_start=qd0,
        self_contact=dict(radius=0.012, margin=0.02, relaxation=0.85, interval=2, ring=3, rest_exclusion=0.06),
    )  # fmt: skip
    np.savez_compressed(os.path.join(args.out, "step_selfcontact_fold.npz"), **out)


def _complex_rest_angle_mesh(ref):
    """Vertex/face lists of ``set_up_complex_rest_angle_bending_experiment`` read from the reference test."""
    path = os.path.join(ref, "newton/tests/test_cloth.py")
    with open(path) as f:
        tree = ast.parse(f.read())
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == "set_up_complex_rest_angle_bending_experiment":
            vals = {}
            for sub in ast.walk(node):
                if isinstance(sub, ast.Assign) and isinstance(sub.targets[0], ast.Name) and sub.targets[0].id in ("vs", "fs"):
                    if sub.targets[0].id not in vals:
                        vals[sub.targets[0].id] = ast.literal_eval(sub.value)
            return vals["vs"], vals["fs"]
    raise RuntimeError("fixture not found")


if __name__ == "__main__":
    main()
