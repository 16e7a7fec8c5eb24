"""Generate golden vectors for the cloth VBD path by executing the reference's own code.

Run in a container that has the reference checkout (read-only) at ``/root/reference``::

    python tests/golden/make_golden.py [--ref /root/reference] [--out tests/golden]

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
            mod = ast.Module(body=[strip(node)], type_ignores=[])
            exec(compile(mod, path, "exec"), ns)
            found.add(node.name)
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
    _lift(os.path.join(ref, "newton/_src/utils/mesh.py"), set(), ns, classes={"MeshAdjacency": {"*"}})
    _lift(
        os.path.join(ref, "newton/_src/sim/builder.py"),
        set(),
        ns,
        classes={"ModelBuilder": {"add_triangles", "add_edges", "add_cloth_grid", "add_cloth_mesh"}},
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


def greedy_coloring(n, tri_indices, edge_indices, edge_props):
    """Greedy coloring of the particle graph of ``construct_particle_graph`` (graph_coloring.py:199-236)."""
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
        self.adj = types.SimpleNamespace(
            v_adj_faces=wp.scalar_array(f_adj, int),
            v_adj_faces_offsets=wp.scalar_array(f_off, int),
            v_adj_edges=wp.scalar_array(e_adj, int),
            v_adj_edges_offsets=wp.scalar_array(e_off, int),
        )
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


def ref_step(sc: RefScene, q_in, qd_in, f_ext, contacts, dt, iterations, friction_epsilon=1e-2, beta=0.0):
    """One ``SolverVBD.step`` without self-contact and without rigid bodies (static shapes only)."""
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

    # _initialize_rigid_bodies -> init_body_particle_contacts (solver_vbd.py:2119-2149)
    wp.launch(
        ns["init_body_particle_contacts"], cmax, cnt, c_shape, sc.soft_ke, sc.soft_kd, sc.soft_mu,
        sc.shape_ke, sc.shape_kd, sc.shape_mu, k_start, pen_k, mat_kd, mat_mu, mat_ke,
    )  # fmt: skip

    # _initialize_particles (solver_vbd.py:1731-1766)
    pos_prev_cd = wp.vec_array(wp.to_numpy(state_in_q))
    disp = wp.vec_array(np.zeros((n, 3)))
    wp.launch(
        ns["forward_step"], n, dt, sc.gravity, q_prev, state_in_q, state_in_qd, sc.inv_mass, particle_f,
        sc.flags, inertia, disp,
    )  # fmt: skip
    ts = wp.scalar_array(np.ones(n))

    def truncate():
        ts.items = [1.0] * n
        wp.launch(ns["apply_truncation_ts"], n, pos_prev_cd, disp, ts, wp.inf, disp, state_in_q)

    truncate()
    for _it in range(iterations):
        # _solve_rigid_body_iteration with no bodies: dual update only (solver_vbd.py:2339-2376)
        wp.launch(
            ns["update_duals_body_particle_contacts"], cmax, cnt, c_particle, c_shape, c_body_pos, c_normal,
            state_in_q, sc.radius, sc.shape_body, sc.empty, mat_ke, beta, pen_k,
        )  # fmt: skip
        forces = wp.vec_array(np.zeros((n, 3)))
        hessians = wp.mat33_array(np.zeros((n, 3, 3)))
        for color in range(len(sc.groups)):
            wp.launch(
                ns["accumulate_particle_body_contact_force_and_hessian"], cmax, dt, color, q_prev, state_in_q,
                sc.particle_colors, friction_epsilon, sc.radius, c_particle, cnt, cmax, pen_k, mat_kd, mat_mu,
                sc.shape_mu, sc.shape_body, sc.empty, None, sc.empty, sc.empty, c_shape, c_body_pos, c_body_vel,
                c_normal, forces, hessians,
            )  # fmt: skip
            group = wp.scalar_array(sc.groups[color], int)
            wp.launch(
                ns["solve_elasticity"], len(sc.groups[color]), dt, group, q_prev, state_in_q, sc.mass, inertia,
                sc.flags, sc.tri_indices, sc.tri_poses, sc.tri_materials, sc.tri_areas, sc.edge_indices,
                sc.edge_rest_angle, sc.edge_rest_length, sc.edge_bending_properties, sc.empty, sc.empty,
                sc.empty, sc.adj, forces, hessians, disp,
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
              friction_epsilon=1e-2, f_ext_scale=0.0):  # fmt: skip
    m = b.arrays()
    colors, groups = greedy_coloring(len(m["particle_q"]), m["tri_indices"], m["edge_indices"], m["edge_bending_properties"])
    sc = RefScene(ns, m, groups, colors, gravity, soft, shapes)
    n = sc.n
    rng = np.random.default_rng(seed)
    q = m["particle_q"].copy()
    qd = m["particle_qd"].copy()
    out = {f"model_{k}": v for k, v in m.items()}
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
    for s in range(substeps):
        f_ext = rng.normal(0.0, 1.0, size=(n, 3)) * f_ext_scale
        contacts = contact_fn(q, m["particle_radius"], m["particle_flags"]) if contact_fn else []
        cnt, cp, cs, cbp, cbv, cn = contacts_to_arrays(contacts, cmax)
        out[f"s{s}_q_in"], out[f"s{s}_qd_in"], out[f"s{s}_f_ext"] = q.copy(), qd.copy(), f_ext
        out[f"s{s}_contact_count"], out[f"s{s}_contact_particle"], out[f"s{s}_contact_shape"] = cnt, cp, cs
        out[f"s{s}_contact_body_pos"], out[f"s{s}_contact_body_vel"], out[f"s{s}_contact_normal"] = cbp, cbv, cn
        q_in_after, q_out, qd_out = ref_step(sc, q, qd, f_ext, contacts, dt, iterations, friction_epsilon, beta)
        out[f"s{s}_q_in_after"], out[f"s{s}_q_out"], out[f"s{s}_qd_out"] = q_in_after, q_out, qd_out
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
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
