"""GPU parity of particle self-contact (vertex-triangle and edge-edge contact, detection, truncation).

Tolerances (positions in metres):
  * FP32 kernels vs the float64 reference goldens: 1e-4 after each substep;
  * FP64 kernels vs the FP64 oracle on the same float32 model arrays: 1e-9 per substep, 1e-7 over a
    multi-substep trajectory;
  * detection: the same pairs in the same slots as the reference's detection kernels (goldens) and the
    oracle's brute force; minimum distances to 1e-6 (float32 arithmetic against float64).
"""

import numpy as np
import pytest
import torch

from newton_chysx_b200 import SolverVBD, sim
from newton_chysx_b200.collision import TriMeshCollisionDetector, build_contact_filters
from oracle import vbd_oracle as orc
from tests.helpers import contacts_from_golden, load_golden, model_from_golden, oracle_model_dict

pytestmark = pytest.mark.gpu

SCENES = ["step_selfcontact_layers.npz", "step_selfcontact_fold.npz"]


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _sc_kwargs(g):
    return dict(
        particle_enable_self_contact=True, particle_self_contact_radius=float(g["sc_radius"]),
        particle_self_contact_margin=float(g["sc_margin"]),
        particle_conservative_bound_relaxation=float(g["sc_relaxation"]),
        particle_collision_detection_interval=int(g["sc_interval"]),
        particle_topological_contact_filter_threshold=int(g["sc_ring"]),
        particle_rest_shape_contact_exclusion_radius=float(g.get("sc_rest_exclusion", 0.0)),
    )  # fmt: skip


def _solver(g, model, **kw):
    return SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                     **_sc_kwargs(g), **kw)  # fmt: skip


def _step(solver, q, qd, f, dt, dtype=torch.float32):
    st_in, st_out = sim.State(), sim.State()
    st_in.particle_q, st_in.particle_qd, st_in.particle_f = _t(q, dtype), _t(qd, dtype), _t(f, dtype)
    st_out.particle_q = torch.zeros_like(st_in.particle_q)
    st_out.particle_qd = torch.zeros_like(st_in.particle_qd)
    solver.step(st_in, st_out, None, None, dt)
    torch.cuda.synchronize()
    return st_in, st_out


def _oracle(model, g_or_kw):
    d = oracle_model_dict(model, 1e-2, 0.0)
    d["soft"] = d["soft"].astype(np.float32).astype(np.float64)  # the C ABI carries them as float
    return orc.Model(d)


def _oracle_sc(model, kw, vertex_buffer=32, edge_buffer=64):
    vt, ee = build_contact_filters(model.particle_count, model.tri_indices, model.edge_indices,
                                   kw["particle_topological_contact_filter_threshold"])  # fmt: skip
    return orc.SelfContact(
        model.particle_q.cpu().numpy().astype(np.float64), radius=kw["particle_self_contact_radius"],
        margin=kw["particle_self_contact_margin"], relaxation=kw["particle_conservative_bound_relaxation"],
        interval=kw["particle_collision_detection_interval"],
        rest_exclusion=kw["particle_rest_shape_contact_exclusion_radius"], vt_filter=vt, ee_filter=ee,
        vertex_buffer=vertex_buffer, edge_buffer=edge_buffer,
    )  # fmt: skip


@pytest.mark.parametrize("name", SCENES)
@pytest.mark.parametrize("lanes", [1, 4])
def test_fp32_selfcontact_step_matches_reference_goldens(name, lanes):
    g = load_golden(name)
    model = model_from_golden(g)
    solver = _solver(g, model, lanes_per_vertex=lanes)
    assert solver.schedule == "per_color" and solver.layout == "csr" and solver.lanes_per_vertex == lanes
    for s in range(int(g["substeps"])):
        st_in, st_out = _step(solver, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], float(g["dt"]))
        q = st_out.particle_q.cpu().numpy()
        assert np.abs(q - g[f"s{s}_q_out"]).max() <= 1e-4, (name, s)
        assert np.array_equal(st_in.particle_q.cpu().numpy(), q)
        nv, ne, flags = solver.self_contact_counts()
        assert nv > 0 and ne > 0 and flags == 0
    assert solver.device_errors() & ~4 == 0


@pytest.mark.parametrize("name", SCENES)
def test_fp64_selfcontact_step_matches_fp64_oracle(name):
    g = load_golden(name)
    model = model_from_golden(g)
    solver = _solver(g, model, precision="fp64")
    om, osc = _oracle(model, g), _oracle_sc(model, _sc_kwargs(g))
    for s in range(int(g["substeps"])):
        _, st_out = _step(solver, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], float(g["dt"]), torch.float64)
        _, q_o, qd_o = orc.step(om, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], None, float(g["dt"]),
                                int(g["iterations"]), 64, self_contact=osc)  # fmt: skip
        assert np.abs(st_out.particle_q.cpu().numpy() - q_o).max() <= 1e-9, (name, s)
        assert np.abs(st_out.particle_qd.cpu().numpy() - qd_o).max() <= 1e-9 / float(g["dt"])


@pytest.mark.parametrize("name", SCENES)
def test_detector_matches_reference_detection(name):
    """TriMeshCollisionDetector buffers at the step's start positions == the reference kernels' buffers."""
    g = load_golden(name)
    model = model_from_golden(g)
    det = TriMeshCollisionDetector(model, vertex_collision_buffer_pre_alloc=32, edge_collision_buffer_pre_alloc=64,
                                   vertex_triangle_filtering_list=g["sc_vt_filter"],
                                   vertex_triangle_filtering_list_offsets=g["sc_vt_filter_offsets"],
                                   edge_filtering_list=g["sc_ee_filter"],
                                   edge_filtering_list_offsets=g["sc_ee_filter_offsets"])  # fmt: skip
    for s in range(int(g["substeps"])):
        det.refit(_t(g[f"s{s}_q_in"]))
        kw = dict(min_query_radius=float(g.get("sc_rest_exclusion", 0.0)), min_distance_filtering_ref_pos=model.particle_q)
        det.vertex_triangle_collision_detection(float(g["sc_margin"]), **kw)
        det.edge_edge_collision_detection(float(g["sc_margin"]), **kw)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(det.vertex_colliding_triangles.cpu().numpy(), g[f"s{s}_cd0_vt"])
        np.testing.assert_array_equal(det.vertex_colliding_triangles_count.cpu().numpy(), g[f"s{s}_cd0_vt_count"])
        np.testing.assert_array_equal(det.edge_colliding_edges.cpu().numpy(), g[f"s{s}_cd0_ee"])
        np.testing.assert_array_equal(det.edge_colliding_edges_count.cpu().numpy(), g[f"s{s}_cd0_ee_count"])
        assert np.abs(det.vertex_colliding_triangles_min_dist.cpu().numpy() - g[f"s{s}_cd0_vt_min"]).max() <= 1e-6
        assert np.abs(det.edge_colliding_edges_min_dist.cpu().numpy() - g[f"s{s}_cd0_ee_min"]).max() <= 1e-6
        assert det.resize_flags.sum().item() == 0


def _crumpled(n=48, seed=3, layers=2):
    """Stacked, turned and noisy sheets: many vertex-triangle and edge-edge proximities."""
    b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    for k in range(layers):
        rot = sim.quat_from_axis_angle((0.0, 0.0, 1.0), 0.3 * k)
        b.add_cloth_grid(pos=(-0.5, -0.5, 0.004 * k), rot=rot, vel=(0.0, 0.0, -0.5 * k), dim_x=n - 1, dim_y=n - 1,
                         cell_x=1.0 / (n - 1), cell_y=1.0 / (n - 1), mass=2e-4, tri_ke=5.0, tri_ka=5.0, tri_kd=0.0,
                         edge_ke=1e-4, edge_kd=0.0, particle_radius=2e-3)  # fmt: skip
    b.color(include_bending=True)
    model = b.finalize("cuda")
    rng = np.random.default_rng(seed)
    q = model.particle_q.cpu().numpy() + rng.normal(scale=1.5e-3, size=(model.particle_count, 3))
    return model, q.astype(np.float32)


@pytest.mark.parametrize("vb,eb", [(32, 64), (2, 3)])
def test_detector_matches_brute_force(vb, eb):
    """Grid detection == the oracle's brute force (all pairs), including buffer overflow (lowest ids kept)."""
    model, q = _crumpled()
    margin = 6e-3
    vt, ee = build_contact_filters(model.particle_count, model.tri_indices, model.edge_indices, 2)
    det = TriMeshCollisionDetector(model, vertex_collision_buffer_pre_alloc=vb, edge_collision_buffer_pre_alloc=eb,
                                   vertex_triangle_filtering_list=vt[0], vertex_triangle_filtering_list_offsets=vt[1],
                                   edge_filtering_list=ee[0], edge_filtering_list_offsets=ee[1])  # fmt: skip
    det.refit(_t(q))
    det.vertex_triangle_collision_detection(margin)
    det.edge_edge_collision_detection(margin)
    torch.cuda.synchronize()
    om = _oracle(model, None)
    osc = orc.SelfContact(np.zeros((model.particle_count, 3)), radius=margin, margin=margin, vt_filter=vt,
                          ee_filter=ee, vertex_buffer=vb, edge_buffer=eb)  # fmt: skip
    ref = orc.collide(om, osc, q.astype(np.float64), precision=32, nthreads=orc.max_threads())
    got_vt = det.vertex_colliding_triangles.cpu().numpy()
    got_ee = det.edge_colliding_edges.cpu().numpy()
    assert ref["vt_count"].sum() > model.particle_count // 4 and ref["ee_count"].sum() > 0
    np.testing.assert_array_equal(det.vertex_colliding_triangles_count.cpu().numpy(), ref["vt_count"])
    np.testing.assert_array_equal(det.edge_colliding_edges_count.cpu().numpy(), ref["ee_count"])
    np.testing.assert_array_equal(got_vt, ref["vt"])
    np.testing.assert_array_equal(got_ee, ref["ee"])
    assert np.abs(det.vertex_colliding_triangles_min_dist.cpu().numpy() - ref["vt_min"]).max() <= 1e-6
    overflow = vb < 32
    assert bool(det.resize_flags[0].item()) == overflow and bool(det.resize_flags[2].item()) == overflow


def _layers_scene(n=12):
    model, q = _crumpled(n=n, seed=5)
    qd = np.zeros_like(q)
    qd[model.particle_count // 2 :, 2] = -0.5
    kw = dict(particle_enable_self_contact=True, particle_self_contact_radius=2e-3, particle_self_contact_margin=3.5e-3,
              particle_conservative_bound_relaxation=0.85, particle_collision_detection_interval=0,
              particle_topological_contact_filter_threshold=2, particle_rest_shape_contact_exclusion_radius=0.0)  # fmt: skip
    return model, q, qd, kw


def test_fp64_selfcontact_trajectory_matches_oracle():
    model, q, qd, kw = _layers_scene()
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e2, 1.0e-4, 0.3
    solver = SolverVBD(model, iterations=5, precision="fp64", **kw)
    om, osc = _oracle(model, None), _oracle_sc(model, kw)
    dt = 1.0 / 600.0
    qg, qdg = q.astype(np.float64), qd.astype(np.float64)
    qo, qdo = qg.copy(), qdg.copy()
    f = np.zeros_like(qg)
    for _ in range(8):
        _, st_out = _step(solver, qg, qdg, f, dt, torch.float64)
        qg, qdg = st_out.particle_q.cpu().numpy(), st_out.particle_qd.cpu().numpy()
        _, qo, qdo = orc.step(om, qo, qdo, f, None, dt, 5, 64, self_contact=osc)
    assert np.abs(qg - qo).max() <= 1e-7
    assert solver.self_contact_counts()[0] > 0


def test_selfcontact_graph_capture_and_determinism():
    model, q, qd, kw = _layers_scene(24)
    solver = SolverVBD(model, iterations=4, **kw)
    dt = 1.0 / 600.0

    def run(steps):
        s0, s1 = model.state(), model.state()
        s0.particle_q.copy_(_t(q))
        s0.particle_qd.copy_(_t(qd))
        for _ in range(steps):
            solver.step(s0, s1, None, None, dt)
            s0, s1 = s1, s0
        torch.cuda.synchronize()
        return s0.particle_q.clone()

    a, b = run(3), run(3)
    assert torch.equal(a, b)  # no atomics in the sums: bitwise repeatable
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(_t(q))
    s0.particle_qd.copy_(_t(qd))
    solver.step(s0, s1, None, None, dt)  # sizes every buffer before capture
    s0.particle_q.copy_(_t(q))
    s0.particle_qd.copy_(_t(qd))
    graph = torch.cuda.CUDAGraph()
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        with torch.cuda.graph(graph, stream=stream):
            solver.step(s0, s1, None, None, dt)
            solver.step(s1, s0, None, None, dt)
    torch.cuda.current_stream().wait_stream(stream)
    s0.particle_q.copy_(_t(q))
    s0.particle_qd.copy_(_t(qd))
    graph.replay()
    solver.step(s0, s1, None, None, dt)
    torch.cuda.synchronize()
    assert torch.equal(s1.particle_q, a)
    assert torch.isfinite(a).all()


def test_selfcontact_launch_constraints():
    """Self-contact runs with the csr layout; the persistent schedule needs a fixed AVBD penalty (rigid_avbd_beta
    0); the margin may not be below the radius."""
    from newton_chysx_b200 import _lib

    model, q, qd, kw = _layers_scene(8)
    assert SolverVBD(model, **kw).schedule == "per_color"  # one world
    assert SolverVBD(model, schedule="persistent", **kw).schedule == "persistent"
    with pytest.raises(ValueError):
        SolverVBD(model, layout="ell", **kw)
    with pytest.raises(ValueError):
        SolverVBD(model, **dict(kw, particle_self_contact_margin=1e-3))
    with pytest.raises(_lib.VbdError, match="unsupported"):
        SolverVBD(model, schedule="persistent", rigid_avbd_beta=1.0e3, **kw)


def _point_triangle_distance(p, a, b, c):
    """|p - closest point of triangle abc| (float64, vectorised): the closest point of the plane, clamped into the
    triangle through its edges when it falls outside."""
    ab, ac, ap = b - a, c - a, p - a
    n = np.cross(ab, ac)
    nn = np.einsum("ij,ij->i", n, n)
    q = p - n * (np.einsum("ij,ij->i", ap, n) / nn)[:, None]

    def inside(u, v, w):
        return np.einsum("ij,ij->i", np.cross(v - u, q - u), n) >= 0.0

    def seg(u, v):
        d = v - u
        t = np.clip(np.einsum("ij,ij->i", p - u, d) / np.einsum("ij,ij->i", d, d), 0.0, 1.0)
        return np.linalg.norm(p - (u + d * t[:, None]), axis=1)

    plane = np.linalg.norm(p - q, axis=1)
    edges = np.minimum(np.minimum(seg(a, b), seg(b, c)), seg(c, a))
    return np.where(inside(a, b, c) & inside(b, c, a) & inside(c, a, b), plane, edges)


def _check_triangle_side(det, tri, q, pairs, T, tb, margin):
    """The detector's triangle -> colliding vertices buffers against the pair set (vertex, triangle): per triangle
    the count of its pairs, its tb smallest vertex ids in increasing order (-1 after), and the smallest pair
    distance (margin when none) to 1e-6."""
    got = det.triangle_colliding_vertices.cpu().numpy().reshape(T, tb)
    cnt = det.triangle_colliding_vertices_count.cpu().numpy()
    mind = det.triangle_colliding_vertices_min_dist.cpu().numpy()
    by_tri = {}
    for v, t in pairs:
        by_tri.setdefault(int(t), []).append(int(v))
    want_cnt = np.zeros(T, dtype=np.int64)
    want_min = np.full(T, margin)
    for t, vs in by_tri.items():
        vs = sorted(vs)
        want_cnt[t] = len(vs)
        row = np.full(tb, -1)
        row[: min(tb, len(vs))] = vs[:tb]
        np.testing.assert_array_equal(got[t], row)
        qv = q[vs].astype(np.float64)
        abc = [np.repeat(q[tri[t, k]][None].astype(np.float64), len(vs), 0) for k in range(3)]
        want_min[t] = _point_triangle_distance(qv, *abc).min()
    np.testing.assert_array_equal(cnt, want_cnt)
    empty = want_cnt == 0
    assert np.all(got[empty] == -1)
    assert np.abs(mind - want_min).max() <= 1e-6
    overflow = bool(np.any(want_cnt > tb))
    assert bool(det.resize_flags[1].item()) == overflow
    return overflow


@pytest.mark.parametrize("name", SCENES)
def test_detector_records_triangle_contacting_vertices(name):
    """record_triangle_contacting_vertices: the reference records every vertex-triangle pair on the triangle's side
    as well (geometry/kernels.py:1373-1384). The golden scenes' vertex buffers (the reference's own detection, no
    overflow) hold every pair, so they give each triangle's colliding vertices and count."""
    g = load_golden(name)
    model = model_from_golden(g)
    tb = 16
    det = TriMeshCollisionDetector(model, record_triangle_contacting_vertices=True,
                                   triangle_collision_buffer_pre_alloc=tb, vertex_collision_buffer_pre_alloc=32,
                                   edge_collision_buffer_pre_alloc=64,
                                   vertex_triangle_filtering_list=g["sc_vt_filter"],
                                   vertex_triangle_filtering_list_offsets=g["sc_vt_filter_offsets"],
                                   edge_filtering_list=g["sc_ee_filter"],
                                   edge_filtering_list_offsets=g["sc_ee_filter_offsets"])  # fmt: skip
    tri = g["model_tri_indices"]
    margin = float(g["sc_margin"])
    seen = 0
    for s in range(int(g["substeps"])):
        q = g[f"s{s}_q_in"].astype(np.float32)
        det.refit(_t(q))
        kw = dict(min_query_radius=float(g.get("sc_rest_exclusion", 0.0)), min_distance_filtering_ref_pos=model.particle_q)
        det.vertex_triangle_collision_detection(margin, **kw)
        torch.cuda.synchronize()
        vt = g[f"s{s}_cd0_vt"].reshape(-1, 2)
        assert np.all(g[f"s{s}_cd0_vt_count"] <= 32)  # the reference kept every pair
        pairs = [(int(v), int(t)) for v, t in vt if v >= 0]
        seen += len(pairs)
        _check_triangle_side(det, tri, q, pairs, model.tri_count, tb, margin)
    assert seen > 0


@pytest.mark.parametrize("tb", [16, 2])
def test_detector_triangle_buffers_match_brute_force(tb):
    """Triangle buffers on a crumpled two-layer sheet against the oracle's brute-force pairs; with 2 slots per
    triangle the buffers overflow, keep the smallest vertex ids and raise resize flag 1."""
    model, q = _crumpled()
    margin = 6e-3
    vt, ee = build_contact_filters(model.particle_count, model.tri_indices, model.edge_indices, 2)
    det = TriMeshCollisionDetector(model, record_triangle_contacting_vertices=True,
                                   triangle_collision_buffer_pre_alloc=tb, vertex_collision_buffer_pre_alloc=32,
                                   vertex_triangle_filtering_list=vt[0], vertex_triangle_filtering_list_offsets=vt[1],
                                   edge_filtering_list=ee[0], edge_filtering_list_offsets=ee[1])  # fmt: skip
    det.refit(_t(q))
    det.vertex_triangle_collision_detection(margin)
    torch.cuda.synchronize()
    om = _oracle(model, None)
    osc = orc.SelfContact(np.zeros((model.particle_count, 3)), radius=margin, margin=margin, vt_filter=vt,
                          ee_filter=ee, vertex_buffer=32, edge_buffer=64)  # fmt: skip
    ref = orc.collide(om, osc, q.astype(np.float64), precision=32, nthreads=orc.max_threads())
    assert np.all(ref["vt_count"] <= 32)
    pairs = [(int(v), int(t)) for v, t in ref["vt"].reshape(-1, 2) if v >= 0]
    assert len(pairs) > model.particle_count // 4
    overflow = _check_triangle_side(det, model.tri_indices.cpu().numpy(), q, pairs, model.tri_count, tb, margin)
    assert overflow == (tb == 2)


def _two_worlds(g, offset=(4.0, 0.0, 0.0)):
    """The golden scene twice, as worlds 0 and 1 of one model, the second moved by `offset` (far beyond the contact
    margin, so the worlds never touch): the reference's add_world union with each world its own instance."""
    m = model_from_golden(g)
    V = m.particle_count
    off = torch.tensor(offset, dtype=torch.float32, device="cuda")
    cat = torch.cat
    m.particle_q = cat([m.particle_q, m.particle_q + off])
    m.particle_qd = cat([m.particle_qd, m.particle_qd])
    for k in ("particle_mass", "particle_inv_mass", "particle_radius", "particle_flags", "tri_poses", "tri_materials",
              "tri_areas", "edge_rest_angle", "edge_rest_length", "edge_bending_properties"):  # fmt: skip
        setattr(m, k, cat([getattr(m, k), getattr(m, k)]))
    m.tri_indices = cat([m.tri_indices, m.tri_indices + V])
    e2 = m.edge_indices.clone()
    e2[e2 >= 0] += V
    m.edge_indices = cat([m.edge_indices, e2])
    m.particle_color_groups = [cat([c, c + V]) for c in m.particle_color_groups]
    m.particle_colors = cat([m.particle_colors, m.particle_colors])
    m.particle_count, m.tri_count, m.edge_count = 2 * V, 2 * m.tri_count, 2 * m.edge_count
    m.world_count = 2
    m.world_particle_start = np.array([0, V, 2 * V], dtype=np.int32)
    return m, V, np.asarray(offset)


def _two_world_inputs(g, s, V, offset, dtype=np.float64):
    q = np.concatenate([g[f"s{s}_q_in"], g[f"s{s}_q_in"] + offset]).astype(dtype)
    qd = np.concatenate([g[f"s{s}_qd_in"], g[f"s{s}_qd_in"]]).astype(dtype)
    f = np.concatenate([g[f"s{s}_f_ext"], g[f"s{s}_f_ext"]]).astype(dtype)
    c1 = contacts_from_golden(g, s)
    n = int(c1.soft_contact_count.item())
    c = sim.Contacts(2 * max(c1.soft_contact_max, 1), "cuda")
    c.soft_contact_count.fill_(2 * n)
    for name in ("soft_contact_shape", "soft_contact_body_pos", "soft_contact_body_vel", "soft_contact_normal"):
        a = getattr(c1, name)[:n]
        getattr(c, name)[: 2 * n] = torch.cat([a, a])
    p = c1.soft_contact_particle[:n]
    c.soft_contact_particle[: 2 * n] = torch.cat([p, p + V])
    return q, qd, f, c


@pytest.mark.parametrize("name", SCENES)
def test_persistent_self_contact_two_worlds_match_reference_goldens(name):
    """Self-contact on a model of two worlds runs one world per CTA (persistent schedule, the detection keeping
    pairs within a world): each world follows the reference's goldens of its scene, within 1e-4 m per substep."""
    g = load_golden(name)
    model, V, offset = _two_worlds(g)
    solver = _solver(g, model)
    assert solver.schedule == "persistent" and solver.layout == "csr"
    for s in range(int(g["substeps"])):
        q, qd, f, c = _two_world_inputs(g, s, V, offset)
        st_in, st_out = sim.State(), sim.State()
        st_in.particle_q, st_in.particle_qd, st_in.particle_f = _t(q), _t(qd), _t(f)
        st_out.particle_q = torch.zeros_like(st_in.particle_q)
        st_out.particle_qd = torch.zeros_like(st_in.particle_qd)
        solver.step(st_in, st_out, None, c if model.shape_count else None, float(g["dt"]))
        torch.cuda.synchronize()
        out = st_out.particle_q.cpu().numpy().astype(np.float64)
        ref = g[f"s{s}_q_out"]
        assert np.abs(out[:V] - ref).max() <= 1e-4, (name, s)
        assert np.abs(out[V:] - offset - ref).max() <= 1e-4, (name, s)
        qd_out = st_out.particle_qd.cpu().numpy()
        assert np.abs(qd_out[:V] - g[f"s{s}_qd_out"]).max() <= 1e-4 / float(g["dt"])
    nv, ne, flags = solver.self_contact_counts()
    assert nv + ne > 0 and flags == 0
    assert solver.device_errors() & ~4 == 0


@pytest.mark.parametrize("name", SCENES)
def test_persistent_self_contact_fp64_matches_per_color_fp64(name):
    """FP64: the persistent schedule on two worlds against the per-color schedule on the same model, which the tests
    above hold to the FP64 oracle; the worlds are apart, so both find the same pairs."""
    g = load_golden(name)
    model, V, offset = _two_worlds(g)
    outs = []
    for schedule in ("persistent", "per_color"):
        solver = _solver(g, model, schedule=schedule, precision="fp64")
        assert solver.schedule == schedule
        res = []
        for s in range(int(g["substeps"])):
            q, qd, f, c = _two_world_inputs(g, s, V, offset)
            st_in, st_out = _step_with(solver, q, qd, f, c if model.shape_count else None, float(g["dt"]))
            res.append(st_out.particle_q.cpu().numpy())
        outs.append(res)
    for a, b in zip(*outs, strict=True):
        assert np.abs(a - b).max() <= 1e-9


def _step_with(solver, q, qd, f, contacts, dt):
    st_in, st_out = sim.State(), sim.State()
    st_in.particle_q, st_in.particle_qd, st_in.particle_f = (_t(a, torch.float64) for a in (q, qd, f))
    st_out.particle_q = torch.zeros_like(st_in.particle_q)
    st_out.particle_qd = torch.zeros_like(st_in.particle_qd)
    solver.step(st_in, st_out, None, contacts, dt)
    torch.cuda.synchronize()
    return st_in, st_out


def test_persistent_self_contact_batch_matches_per_color():
    """Four crumpled two-layer sheets of different sizes as worlds, detection every second iteration: each substep of
    the persistent schedule (pairs within a world) against the per-color schedule (all pairs; the worlds are apart,
    so the same ones) from the same input state, FP32, within the 1e-4 m of the FP32 parity tests: the two kernels
    compile the same solve separately, so their multiply-adds may fuse differently, and the barrier-driven contact
    solves of these sheets amplify that rounding to ~1e-5 m (the FP64 versions agree to 1e-9 m, above)."""
    b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    rng = np.random.default_rng(11)
    for k, n in enumerate((12, 20, 9, 16)):
        w = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
        for layer in range(2):
            rot = sim.quat_from_axis_angle((0.0, 0.0, 1.0), 0.3 * layer)
            w.add_cloth_grid(pos=(3.0 * k - 0.5, -0.5, 0.004 * layer), rot=rot, vel=(0.0, 0.0, -0.5 * layer),
                             dim_x=n - 1, dim_y=n - 1, cell_x=1.0 / (n - 1), cell_y=1.0 / (n - 1), mass=2e-4,
                             tri_ke=5.0, tri_ka=5.0, tri_kd=0.0, edge_ke=1e-4, edge_kd=0.0, particle_radius=2e-3)  # fmt: skip
        w.color(include_bending=True)
        b.add_world(w)
    model = b.finalize("cuda")
    q0 = model.particle_q.cpu().numpy() + rng.normal(scale=1.0e-3, size=(model.particle_count, 3))
    # the same lane split in both (the persistent default), so that each vertex sums its terms in the same order
    kw = dict(particle_enable_self_contact=True, particle_self_contact_radius=2e-3, particle_self_contact_margin=3.5e-3,
              particle_collision_detection_interval=2, lanes_per_vertex=4)  # fmt: skip
    pers = SolverVBD(model, iterations=6, schedule="persistent", **kw)
    ref = SolverVBD(model, iterations=6, schedule="per_color", **kw)
    s0, s1, t0, t1 = model.state(), model.state(), model.state(), model.state()
    s0.particle_q.copy_(torch.as_tensor(q0, dtype=torch.float32))
    worst, pairs = 0.0, 0
    for _ in range(6):
        t0.particle_q.copy_(s0.particle_q)
        t0.particle_qd.copy_(s0.particle_qd)
        pers.step(t0, t1, None, None, 1.0 / 600.0)
        ref.step(s0, s1, None, None, 1.0 / 600.0)
        torch.cuda.synchronize()
        assert pers.self_contact_counts()[:2] == ref.self_contact_counts()[:2]
        pairs += sum(ref.self_contact_counts()[:2])
        worst = max(worst, (t1.particle_q - s1.particle_q).abs().max().item())
        s0, s1 = s1, s0
    assert pairs > 0 and torch.isfinite(s0.particle_q).all()
    assert worst <= 1e-4, worst
