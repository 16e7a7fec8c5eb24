"""Shared test helpers: models from golden arrays, scene builders and oracle adapters."""

from __future__ import annotations

import os

import numpy as np
import torch

from newton_chysx_b200 import sim

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def model_from_golden(g, device="cuda") -> sim.Model:
    """A Model with the golden fixture's arrays (float32), colors and contact materials."""
    m = sim.Model()
    dev = torch.device(device)
    m.device = dev

    def t(a, dt):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)

    f32, i32 = torch.float32, torch.int32
    n = len(g["model_particle_mass"])
    m.particle_count = n
    m.tri_count = len(g["model_tri_indices"])
    m.edge_count = len(g["model_edge_indices"])
    m.particle_q = t(g["model_particle_q"], f32)
    m.particle_qd = t(g["model_particle_qd"], f32)
    m.particle_mass = t(g["model_particle_mass"], f32)
    m.particle_inv_mass = t(g["model_particle_inv_mass"], f32)
    m.particle_radius = t(g["model_particle_radius"], f32)
    m.particle_flags = t(g["model_particle_flags"], i32)
    m.tri_indices = t(g["model_tri_indices"], i32)
    m.tri_poses = t(g["model_tri_poses"], f32)
    m.tri_materials = t(g["model_tri_materials"], f32)
    m.tri_areas = t(g["model_tri_areas"], f32)
    m.edge_indices = t(g["model_edge_indices"], i32)
    m.edge_rest_angle = t(g["model_edge_rest_angle"], f32)
    m.edge_rest_length = t(g["model_edge_rest_length"], f32)
    m.edge_bending_properties = t(g["model_edge_bending_properties"], f32)
    co, cp = g["color_offsets"], g["color_particles"]
    m.particle_color_groups = [t(cp[co[c]:co[c + 1]], i32) for c in range(len(co) - 1)]
    m.particle_colors = t(g["particle_colors"], i32)
    m.gravity = t(np.asarray(g["gravity"]).reshape(1, 3), f32)
    soft = g["soft"]
    m.soft_contact_ke, m.soft_contact_kd, m.soft_contact_mu = float(soft[0]), float(soft[1]), float(soft[2])
    shapes = np.asarray(g["shapes"]).reshape(-1, 3)
    S = len(shapes)
    m.shape_count = S
    m.shape_material_ke = t(shapes[:, 0], f32)
    m.shape_material_kd = t(shapes[:, 1], f32)
    m.shape_material_mu = t(shapes[:, 2], f32)
    m.shape_body = t(-np.ones(S), i32)
    if "shape_body" in g:  # shapes on bodies that an external rigid solver moves
        m.shape_body = t(g["shape_body"], i32)
        m.body_com = t(np.asarray(g["body_com"]).reshape(-1, 3), f32)
        m.body_count = len(m.body_com)
    m.world_particle_start = None
    if "model_spring_indices" in g:
        m.spring_count = len(g["model_spring_rest_length"])
        m.spring_indices = t(np.asarray(g["model_spring_indices"]).reshape(-1), i32)
        m.spring_rest_length = t(g["model_spring_rest_length"], f32)
        m.spring_stiffness = t(g["model_spring_stiffness"], f32)
        m.spring_damping = t(g["model_spring_damping"], f32)
    if "model_tet_indices" in g:
        m.tet_count = len(g["model_tet_indices"])
        m.tet_indices = t(g["model_tet_indices"], i32)
        m.tet_poses = t(g["model_tet_poses"], f32)
        m.tet_materials = t(g["model_tet_materials"], f32)
    return m


def golden_solver_kw(g) -> dict:
    """SolverVBD keywords a golden fixture needs: its bodies are moved by an external rigid solver."""
    return dict(integrate_with_external_rigid_solver=True) if "shape_body" in g else {}


def golden_body_states(g, s, st_in, st_out, device="cuda"):
    """Substep s's body poses on the states (state_in.body_q, state_out.body_q, state_out.body_qd), if any."""
    if "shape_body" not in g:
        return
    dev = torch.device(device)
    st_in.body_q = torch.as_tensor(g[f"s{s}_body_q_in"], dtype=torch.float32, device=dev)
    st_out.body_q = torch.as_tensor(g[f"s{s}_body_q_out"], dtype=torch.float32, device=dev)
    st_in.body_qd = torch.zeros((len(st_in.body_q), 6), dtype=torch.float32, device=dev)
    st_out.body_qd = torch.as_tensor(g[f"s{s}_body_qd_out"], dtype=torch.float32, device=dev)


def golden_body_contacts_kw(g, s, fp32=False) -> dict:
    """make_contacts keywords of substep s's bodies for the oracle (float32-rounded with fp32, as the GPU reads
    them): the step reads state_out.body_q, state_in.body_q as the previous pose and state_out.body_qd."""
    if "shape_body" not in g:
        return {}

    def r(a):
        a = np.asarray(a, dtype=np.float64)
        return a.astype(np.float32).astype(np.float64) if fp32 else a

    return dict(shape_body=g["shape_body"], body_q=r(g[f"s{s}_body_q_out"]), body_q_prev=r(g[f"s{s}_body_q_in"]),
                body_qd=r(g[f"s{s}_body_qd_out"]), body_com=r(g["body_com"]))  # fmt: skip


def contacts_from_golden(g, s, device="cuda") -> sim.Contacts:
    cp = g[f"s{s}_contact_particle"]
    c = sim.Contacts(len(cp), device)
    c.soft_contact_count.fill_(int(g[f"s{s}_contact_count"]))
    c.soft_contact_particle.copy_(torch.as_tensor(cp, dtype=torch.int32))
    c.soft_contact_shape.copy_(torch.as_tensor(g[f"s{s}_contact_shape"], dtype=torch.int32))
    c.soft_contact_body_pos.copy_(torch.as_tensor(g[f"s{s}_contact_body_pos"], dtype=torch.float32))
    c.soft_contact_body_vel.copy_(torch.as_tensor(g[f"s{s}_contact_body_vel"], dtype=torch.float32))
    c.soft_contact_normal.copy_(torch.as_tensor(g[f"s{s}_contact_normal"], dtype=torch.float32))
    return c


def oracle_model_dict(model: sim.Model, friction_epsilon=1e-2, beta=0.0) -> dict:
    """Arrays of a product Model in the oracle's dict form (float32 values widened to float64)."""
    from oracle import vbd_oracle as orc

    def h(x):
        return x.detach().cpu().numpy()

    n = model.particle_count
    fo, fa, eo, ea = orc.build_adjacency(n, h(model.tri_indices), h(model.edge_indices))
    groups = [h(g) for g in model.particle_color_groups]
    colors = np.zeros(n, dtype=np.int32)
    for c, g in enumerate(groups):
        colors[g] = c
    S = model.shape_count
    shapes = np.zeros((max(S, 1), 3))
    if S:
        shapes = np.stack([h(model.shape_material_ke), h(model.shape_material_kd), h(model.shape_material_mu)], 1)
    d = dict(
        particle_mass=h(model.particle_mass), particle_inv_mass=h(model.particle_inv_mass),
        particle_radius=h(model.particle_radius), particle_flags=h(model.particle_flags),
        tri_indices=h(model.tri_indices), tri_poses=h(model.tri_poses), tri_materials=h(model.tri_materials),
        tri_areas=h(model.tri_areas), edge_indices=h(model.edge_indices), edge_rest_angle=h(model.edge_rest_angle),
        edge_rest_length=h(model.edge_rest_length), edge_bending_properties=h(model.edge_bending_properties),
        adj_face_offsets=fo, adj_faces=fa, adj_edge_offsets=eo, adj_edges=ea, particle_colors=colors,
        color_offsets=np.concatenate([[0], np.cumsum([len(g) for g in groups])]).astype(np.int32),
        color_particles=np.concatenate(groups).astype(np.int32), gravity=h(model.gravity)[0],
        soft=np.array([model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu]), shapes=shapes,
        friction_epsilon=friction_epsilon, beta=beta,
    )  # fmt: skip
    if getattr(model, "spring_count", 0):
        d.update(spring_indices=h(model.spring_indices), spring_rest_length=h(model.spring_rest_length),
                 spring_stiffness=h(model.spring_stiffness), spring_damping=h(model.spring_damping))  # fmt: skip
    if getattr(model, "tet_count", 0):
        d.update(tet_indices=h(model.tet_indices), tet_poses=h(model.tet_poses), tet_materials=h(model.tet_materials))
    return d


def cloth_grid_builder(n=32, side=1.0, E=1e4, nu=0.3, h=1e-3, density=0.2, bend=1e-4, radius=5e-3, hanging=True,
                       height=0.05, pin_top_corners=True, up_axis="Z"):  # fmt: skip
    """The plain-VBD scene: an n x n vertex sheet of `side` metres, StVK-like Lame from (E, nu, h)."""
    mu = E * h / (2.0 * (1.0 + nu))
    lam = E * h * nu / (1.0 - nu * nu)
    b = sim.ModelBuilder(up_axis=up_axis, gravity=-9.81)
    cell = side / (n - 1)
    mass = density * side * side / (n * n)
    rot = sim.quat_from_axis_angle((1.0, 0.0, 0.0), np.pi * 0.5) if hanging else sim.quat_identity()
    b.add_cloth_grid(pos=(0.0, 0.0, height), rot=rot, vel=(0.0, 0.0, 0.0), dim_x=n - 1, dim_y=n - 1, cell_x=cell,
                     cell_y=cell, mass=mass, tri_ke=mu, tri_ka=lam, tri_kd=0.0, edge_ke=bend, edge_kd=0.0,
                     particle_radius=radius)  # fmt: skip
    if pin_top_corners:
        flags = b.particle_flags
        flags[n * (n - 1)] &= ~int(sim.ParticleFlags.ACTIVE)
        flags[n * n - 1] &= ~int(sim.ParticleFlags.ACTIVE)
        b.set_particle_flags(flags)
    b.color(include_bending=True)
    return b


def _outward(v, tris, inside_point_fn):
    """Flip triangles whose normal points toward `inside_point_fn(centroid)` (a point inside the solid)."""
    a, b, c = v[tris[:, 0]], v[tris[:, 1]], v[tris[:, 2]]
    n = np.cross(b - a, c - a)
    cen = (a + b + c) / 3.0
    flip = np.einsum("ij,ij->i", n, cen - inside_point_fn(cen)) < 0.0
    tris = tris.copy()
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return tris


def box_mesh(hx, hy, hz):
    """A closed box of half extents (hx, hy, hz): 8 vertices, 12 triangles wound counter-clockwise from outside."""
    v = np.array([[(-hx, hx)[i & 1], (-hy, hy)[(i >> 1) & 1], (-hz, hz)[(i >> 2) & 1]] for i in range(8)])
    tris = []
    for k in range(3):
        for side in (0, 1):
            ids = [i for i in range(8) if ((i >> k) & 1) == side]  # 4 corners, in bit order
            tris += [[ids[0], ids[1], ids[3]], [ids[0], ids[3], ids[2]]]
    return v, _outward(v, np.array(tris), lambda c: np.zeros_like(c))


def icosphere(radius=1.0, subdivisions=2):
    t = (1.0 + 5.0**0.5) / 2.0
    v = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t], [t, 0, -1],
         [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]  # fmt: skip
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6],
         [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
         [8, 6, 7], [9, 8, 1]]  # fmt: skip
    v = [np.asarray(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    for _ in range(subdivisions):
        mid, nf = {}, []

        def m(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                mid[key] = len(v) - 1
            return mid[key]

        for a, b, c in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = nf
    v = np.array(v) * radius
    return v, _outward(v, np.array(f), lambda c: np.zeros_like(c))


def torus_mesh(R=0.3, r=0.1, nu=24, nv=12):
    """A closed torus around the Z axis (tube radius r at distance R): non-convex, genus one."""
    u, w = np.meshgrid(np.arange(nu) * 2 * np.pi / nu, np.arange(nv) * 2 * np.pi / nv, indexing="ij")
    v = np.stack([(R + r * np.cos(w)) * np.cos(u), (R + r * np.cos(w)) * np.sin(u), r * np.sin(w)], -1).reshape(-1, 3)
    tris = []
    for i in range(nu):
        for j in range(nv):
            a, b = i * nv + j, ((i + 1) % nu) * nv + j
            c, d = ((i + 1) % nu) * nv + (j + 1) % nv, i * nv + (j + 1) % nv
            tris += [[a, b, c], [a, c, d]]

    def tube_centre(c):
        ang = np.arctan2(c[:, 1], c[:, 0])
        return np.stack([R * np.cos(ang), R * np.sin(ang), np.zeros(len(c))], -1)

    return v, _outward(v, np.array(tris), tube_centre)
