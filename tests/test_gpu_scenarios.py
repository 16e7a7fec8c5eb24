"""Scenario tests on the GPU: the reference's known-answer cloth tests (test_cloth.py) and
multi-substep trajectories against the FP64 oracle."""

import numpy as np
import pytest
import torch

from newton_chysx_b200 import CollisionPipeline, SolverVBD, sim
from oracle import vbd_oracle as orc
from tests.helpers import cloth_grid_builder, load_golden, oracle_model_dict

pytestmark = pytest.mark.gpu


def _run(model, solver, frames, substeps, dt, pipeline=None):
    s0, s1 = model.state(), model.state()
    contacts = pipeline.contacts() if pipeline else None
    for _ in range(frames):
        for _ in range(substeps):
            s0.clear_forces()
            if pipeline:
                pipeline.collide(s0, contacts)
            solver.step(s0, s1, None, contacts, dt)
            s0, s1 = s1, s0
    torch.cuda.synchronize()
    return s0


def _hanging_scene():
    b = cloth_grid_builder(n=32)
    b.add_ground_plane()
    model = b.finalize("cuda")
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e3, 10.0, 0.5
    return model


def _gpu_trajectory(model, frames, precision, schedule):
    """Frames of 10 substeps x 10 iterations with ground contacts regenerated every substep."""
    solver = SolverVBD(model, iterations=10, schedule=schedule, precision=precision)
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    dt = 1.0 / 600.0
    dtype = torch.float64 if precision == "fp64" else torch.float32
    s0, s1 = model.state(), model.state()
    if precision == "fp64":
        for s in (s0, s1):
            s.particle_q, s.particle_qd, s.particle_f = (t.double() for t in (s.particle_q, s.particle_qd, s.particle_f))
    contacts = pipe.contacts()
    out = []
    for _ in range(frames):
        for _ in range(10):
            pipe.collide(s0 if dtype == torch.float32 else _f32_state(s0), contacts)
            solver.step(s0, s1, None, contacts, dt)
            s0, s1 = s1, s0
        out.append(s0.particle_q.cpu().numpy().astype(np.float64))
    return out


def _f32_state(s):
    t = sim.State()
    t.particle_q = s.particle_q.float()
    return t


def _oracle_trajectory(model, frames, precision):
    om = orc.Model(oracle_model_dict(model))
    q = model.particle_q.cpu().numpy().astype(np.float64)
    qd = model.particle_qd.cpu().numpy().astype(np.float64)
    r, fl = model.particle_radius.cpu().numpy(), model.particle_flags.cpu().numpy()
    out = []
    for _ in range(frames):
        for _ in range(10):
            qc = q.astype(np.float32).astype(np.float64)  # contacts from float32 positions, as on the GPU
            cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(qc, r, fl, model.shape_type, model.shape_transform,
                                                             model.shape_scale, 0.01)  # fmt: skip
            c = orc.make_contacts(cnt, p, s, bp, bv, nn)
            _, q, qd = orc.step(om, q, qd, None, c, 1.0 / 600.0, 10, precision=precision, nthreads=orc.max_threads())
        out.append(q.copy())
    return out


@pytest.mark.parametrize("schedule", ["per_color", "persistent"])
def test_hanging_cloth_fp64_trajectory_matches_fp64_oracle(schedule):
    """32x32 hanging sheet (E=1e4, nu=0.3, h=1e-3, bending 1e-4), two top corners pinned, ground
    contact with friction, 12 frames of 10 substeps x 10 iterations: the FP64 kernels follow the FP64
    oracle through first contact."""
    model = _hanging_scene()
    gpu = _gpu_trajectory(model, 12, "fp64", schedule)
    ref = _oracle_trajectory(model, 12, 64)
    assert max(np.abs(a - b).max() for a, b in zip(gpu, ref, strict=True)) <= 1e-7


@pytest.mark.parametrize("schedule", ["per_color", "persistent"])
def test_hanging_cloth_fp32_error_vs_fp64(schedule):
    """FP32 position error against the FP64 oracle: <= 1e-4 m (cloth side 1 m) while the sheet falls
    (frames 0-4). After the ground contact starts (frame 5) stick/slip friction, regularised over
    eps_u = 1e-2 dt, amplifies FP32 rounding to the millimetre level; the reference's own FP32
    arithmetic (the FP32 oracle) shows the same error, so the GPU must stay within 1.5x of it."""
    model = _hanging_scene()
    gpu = _gpu_trajectory(model, 12, "fp32", schedule)
    ref64 = _oracle_trajectory(model, 12, 64)
    ref32 = _oracle_trajectory(model, 12, 32)
    err = [np.abs(a - b).max() for a, b in zip(gpu, ref64, strict=True)]
    err_ref = [np.abs(a - b).max() for a, b in zip(ref32, ref64, strict=True)]
    assert max(err[:5]) <= 1e-4, err
    assert max(err) <= 1.5 * max(err_ref) + 1e-4, (err, err_ref)


FULL_FRAMES = 120  # the plain-VBD scene's horizon: 120 frames of 10 substeps x 10 iterations


def _per_substep_errors(precision, schedule):
    """Along the GPU's own trajectory of the whole 120-frame horizon of the hanging-sheet scene in `precision`,
    the first substep of every frame against the FP64 oracle's substep from the same state (contacts from the
    same FP32 positions): max vertex |x_gpu - x_oracle|_2 per frame."""
    model = _hanging_scene()
    solver = SolverVBD(model, iterations=10, schedule=schedule, precision=precision)
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    om = orc.Model(oracle_model_dict(model))
    r, fl = model.particle_radius.cpu().numpy(), model.particle_flags.cpu().numpy()
    s0, s1 = model.state(), model.state()
    if precision == "fp64":
        for s in (s0, s1):
            s.particle_q, s.particle_qd, s.particle_f = (t.double() for t in (s.particle_q, s.particle_qd, s.particle_f))
    samples = []
    for _ in range(FULL_FRAMES):
        for k in range(10):
            if k == 0:
                q_in = s0.particle_q.cpu().numpy().astype(np.float64)
                qd_in = s0.particle_qd.cpu().numpy().astype(np.float64)
            pipe.collide(s0 if precision != "fp64" else _f32_state(s0), contacts)
            solver.step(s0, s1, None, contacts, 1.0 / 600.0)
            if k == 0:
                samples.append((q_in, qd_in, s1.particle_q.cpu().numpy().astype(np.float64)))
            s0, s1 = s1, s0
    assert solver.device_errors() == 0
    err = []
    for q_in, qd_in, q_gpu in samples:
        qc = q_in.astype(np.float32).astype(np.float64)
        cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(qc, r, fl, model.shape_type, model.shape_transform,
                                                         model.shape_scale, 0.01)  # fmt: skip
        _, q_ref, _ = orc.step(om, q_in, qd_in, None, orc.make_contacts(cnt, p, s, bp, bv, nn), 1.0 / 600.0, 10,
                               precision=64, nthreads=orc.max_threads())  # fmt: skip
        err.append(float(np.linalg.norm(q_gpu - q_ref, axis=1).max()))
    return err


@pytest.mark.parametrize("schedule", ["per_color", "persistent"])
def test_hanging_cloth_fp64_per_substep_full_horizon(schedule):
    """The whole 120-frame horizon (1,200 substeps: the fall, first contact at frame 5 and stick/slip friction
    on the ground to the end): at every frame the FP64 step equals the FP64 oracle's step from the same state.
    Whole trajectories are not compared past the first frames: from the frame-10 state two FP64 runs that differ
    by 1e-10 m part by centimetres within ten frames (the contact set and the friction regime switch on
    thresholds), in the oracle against itself as well."""
    err = _per_substep_errors("fp64", schedule)
    assert max(err) <= 1e-9, max(err)


def test_hanging_cloth_fp32_per_substep_full_horizon():
    """Along the GPU's own FP32 trajectory of the 120-frame horizon, every frame's first FP32 substep against the
    FP64 oracle's substep from the same FP32 state: <= 1e-4 m (cloth side 1 m) in the fall, at first contact and
    through the friction phase."""
    err = _per_substep_errors("fp32", "per_color")
    assert max(err) <= 1e-4, max(err)
    assert max(err[5:]) > 0.0  # contact frames were compared, not an idle sheet


def test_cloth_on_a_moving_body_matches_oracle():
    """A 16 x 16 sheet (0.5 m) dropped onto a box carried by a body that turns (3 rad/s about z) and rises
    (0.2 m/s) under it, moved by the test as an external rigid solver would: contacts from
    ``CollisionPipeline.collide`` at ``state_in.body_q``, the step with ``integrate_with_external_rigid_solver=True``
    reading ``state_out.body_q``, ``state_in.body_q`` and ``state_out.body_qd``. Along the FP64 trajectory, every
    substep against the FP64 oracle's substep from the same state, contacts and body poses: FP64 <= 1e-9 m, the
    mixed mode (contact vertices in FP64) <= 1e-4 m. FP32 is held to 1e-3 m only: the contact damping
    kd ke / dt = 2.3e6 N/m against the sheet's ~1 N/m tangential stiffness cost FP32 1.6e-4 m along its own
    trajectory."""
    b = cloth_grid_builder(n=16, side=0.5, hanging=False, height=0.262, pin_top_corners=False)
    body = b.add_body(xform=((0.25, 0.25, 0.1), sim.quat_identity()))
    b.add_shape_box(body=body, xform=((0.0, 0.0, 0.05), sim.quat_from_axis_angle((0.0, 0.0, 1.0), 0.2)), hx=0.15,
                    hy=0.12, hz=0.1, cfg=sim.ShapeConfig(ke=5.0e3, kd=1.0, mu=0.6))  # fmt: skip
    b.add_ground_plane()
    model = b.finalize("cuda")
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e4, 1.0e-2, 0.5
    solvers = {p: SolverVBD(model, iterations=10, precision=p, integrate_with_external_rigid_solver=True)
               for p in ("fp32", "mixed", "fp64")}  # fmt: skip
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    c = pipe.contacts()
    om = orc.Model(oracle_model_dict(model))
    sb = model._shape_body_host
    com = model.body_com.cpu().numpy().astype(np.float64)
    dt, w, v = 1.0 / 600.0, 3.0, np.array([0.0, 0.0, 0.2])

    def pose(t):
        return np.concatenate([np.array([0.25, 0.25, 0.1]) + v * t, sim.quat_from_axis_angle((0.0, 0.0, 1.0), w * t)])

    q = model.particle_q.cpu().numpy().astype(np.float64)
    qd = model.particle_qd.cpu().numpy().astype(np.float64)
    err = {p: [] for p in solvers}
    touching = 0
    for k in range(40):
        X0 = pose(k * dt).astype(np.float32)[None]
        X1 = pose((k + 1) * dt).astype(np.float32)[None]
        body_qd = np.concatenate([v, [0.0, 0.0, w]]).astype(np.float32)[None]
        view = sim.State()
        view.particle_q = torch.as_tensor(q.astype(np.float32), device="cuda")
        view.body_q = torch.as_tensor(X0, device="cuda")
        pipe.collide(view, c)  # contacts from the FP32 positions, for every precision
        cnt = int(c.soft_contact_count.item())
        touching += int((sb[c.soft_contact_shape[:cnt].cpu().numpy()] == 0).sum())
        oc = orc.make_contacts(cnt, c.soft_contact_particle.cpu().numpy(), c.soft_contact_shape.cpu().numpy(),
                               c.soft_contact_body_pos.cpu().numpy(), c.soft_contact_body_vel.cpu().numpy(),
                               c.soft_contact_normal.cpu().numpy(), shape_body=sb, body_q=X1.astype(np.float64),
                               body_q_prev=X0.astype(np.float64), body_qd=body_qd.astype(np.float64),
                               body_com=com)  # fmt: skip
        out = {}
        for p, solver in solvers.items():
            dtype = torch.float64 if p == "fp64" else torch.float32
            s_in, s_out = sim.State(), sim.State()
            src_q = q if p == "fp64" else q.astype(np.float32)
            src_qd = qd if p == "fp64" else qd.astype(np.float32)
            s_in.particle_q = torch.as_tensor(src_q, dtype=dtype, device="cuda")
            s_in.particle_qd = torch.as_tensor(src_qd, dtype=dtype, device="cuda")
            s_in.particle_f = torch.zeros_like(s_in.particle_q)
            s_out.particle_q, s_out.particle_qd = torch.zeros_like(s_in.particle_q), torch.zeros_like(s_in.particle_q)
            s_in.body_q, s_out.body_q = torch.as_tensor(X0, device="cuda"), torch.as_tensor(X1, device="cuda")
            s_in.body_qd = torch.zeros_like(torch.as_tensor(body_qd, device="cuda"))
            s_out.body_qd = torch.as_tensor(body_qd, device="cuda")
            solver.step(s_in, s_out, None, c, dt)
            out[p] = (s_out.particle_q.cpu().numpy().astype(np.float64), s_out.particle_qd.cpu().numpy())
            _, q_ref, _ = orc.step(om, np.asarray(src_q, np.float64), np.asarray(src_qd, np.float64), None, oc, dt, 10,
                                   precision=64, nthreads=orc.max_threads())  # fmt: skip
            err[p].append(float(np.linalg.norm(out[p][0] - q_ref, axis=1).max()))
        q, qd = out["fp64"][0], out["fp64"][1].astype(np.float64)
    assert all(s.device_errors() == 0 for s in solvers.values())
    assert touching > 0  # the body's box was in contact
    assert max(err["fp64"]) <= 1e-9, max(err["fp64"])
    assert max(err["mixed"]) <= 1e-4, max(err["mixed"])
    assert max(err["fp32"]) <= 1e-3, max(err["fp32"])


def test_free_fall_matches_kinematics():
    """test_cloth.py:1093-1114: an unconstrained sheet falls as 1/2 g t^2 with no horizontal drift."""
    b = cloth_grid_builder(n=16, hanging=False, pin_top_corners=False, height=4.0, up_axis="Y")
    model = b.finalize("cuda")
    model.set_gravity((0.0, -1000.0, 0.0))
    solver = SolverVBD(model, iterations=5)
    q0 = model.particle_q.cpu().numpy()
    frames, substeps, dt = 5, 10, 1.0 / 600.0
    s = _run(model, solver, frames, substeps, dt)
    diff = s.particle_q.cpu().numpy() - q0
    t = frames * substeps * dt
    # implicit Euler: y_n = -g dt^2 n (n+1) / 2
    n = frames * substeps
    expected = -1000.0 * dt * dt * n * (n + 1) / 2
    assert np.abs(diff[:, 1] - expected).max() < 2e-1
    assert np.abs(diff[:, [0, 2]]).max() < 1e-1
    assert abs(expected) > 0.5 * 1000.0 * t * t * 0.9


def test_bending_converges_to_rest_angles():
    """test_cloth.py:980-1000: without gravity a bent sheet keeps its rest dihedral angles (<= 0.01 rad)."""
    g = load_golden("step_complex_rest_angle.npz")
    vs = g["model_particle_q"] - np.array([0.0, 2.0, 0.0])
    b = sim.ModelBuilder(up_axis="Y")
    b.add_cloth_mesh(pos=(0.0, 2.0, 0.0), rot=sim.quat_identity(), scale=1.0, vel=(0.0, 0.0, 0.0), vertices=vs,
                     indices=g["model_tri_indices"].reshape(-1), density=0.02, tri_ke=1e2, tri_ka=1e2, tri_kd=0.0,
                     edge_ke=1e-1, edge_kd=0.0)  # fmt: skip
    flags = b.particle_flags
    flags[1] = 0
    b.set_particle_flags(flags)
    b.color(include_bending=True)
    model = b.finalize("cuda")
    model.set_gravity((0.0, 0.0, 0.0))
    solver = SolverVBD(model, iterations=5)
    s = _run(model, solver, 50, 10, 1.0 / 600.0)
    q = s.particle_q.cpu().numpy().astype(np.float64)
    rest = model.edge_rest_angle.cpu().numpy()
    worst = 0.0
    for k, (i, j, a, c) in enumerate(model.edge_indices.cpu().numpy()):
        if i < 0 or j < 0:
            continue
        n1 = np.cross(q[a] - q[i], q[c] - q[i])
        n2 = np.cross(q[c] - q[j], q[a] - q[j])
        n1 /= np.linalg.norm(n1)
        n2 /= np.linalg.norm(n2)
        e = (q[c] - q[a]) / np.linalg.norm(q[c] - q[a])
        ang = np.arctan2(np.dot(np.cross(n1, n2), e), np.clip(np.dot(n1, n2), -1, 1))
        worst = max(worst, abs(ang - rest[k]))
    assert worst <= 0.01, worst


def test_schedules_and_lane_counts_agree():
    b = cloth_grid_builder(n=24)
    b.add_ground_plane()
    model = b.finalize("cuda")
    results = []
    for schedule, lanes, shared, layout in [("per_color", 1, "auto", "ell"), ("per_color", 1, "auto", "csr"),
                                            ("per_color", 8, "auto", "csr"), ("persistent", 1, "on", "ell"),
                                            ("persistent", 1, "off", "ell"), ("persistent", 16, "on", "csr"),
                                            ("persistent", 2, "off", "csr"), ("persistent", 1, "on", "ell16"),
                                            ("persistent", 1, "off", "ell16"), ("persistent", 1, "on", "ring"),
                                            ("persistent", 1, "off", "ring")]:
        solver = SolverVBD(model, iterations=10, schedule=schedule, lanes_per_vertex=lanes, positions_in_shared=shared,
                           layout=layout)  # fmt: skip
        s = _run(model, solver, 3, 10, 1.0 / 600.0, CollisionPipeline(model))
        results.append(s.particle_q.cpu().numpy())
    for r in results[1:]:
        assert np.abs(r - results[0]).max() <= 1e-5


def test_batched_worlds_match_single_instances():
    """A multi-world model solved by the persistent kernel (one CTA per world) equals each world
    solved alone: instances are independent and keep their relative color order."""
    sizes = [5, 17, 9, 24, 12]
    top = sim.ModelBuilder()
    singles = []
    for k, n in enumerate(sizes):
        b = cloth_grid_builder(n=n, E=10.0 ** (3 + k % 3), bend=10.0 ** (-5 + k % 3))
        top.add_world(b)
        singles.append(b)
    model = top.finalize("cuda")
    solver = SolverVBD(model, iterations=10, schedule="persistent")
    assert solver.shared_bytes == 12 * max(n * n for n in sizes)
    s = _run(model, solver, 2, 10, 1.0 / 600.0)
    q = s.particle_q.cpu().numpy()
    assert solver.layout == "ell16"
    for shared, layout in [("off", "ell"), ("on", "csr"), ("off", "csr"), ("off", "ell16"), ("off", "ring"),
                           ("on", "ring")]:
        s_g = _run(model, SolverVBD(model, iterations=10, schedule="persistent", positions_in_shared=shared,
                                    layout=layout), 2, 10, 1.0 / 600.0)  # fmt: skip
        assert np.abs(s_g.particle_q.cpu().numpy() - q).max() <= 1e-5
    start = 0
    for b in singles:
        m1 = b.finalize("cuda")
        s1 = _run(m1, SolverVBD(m1, iterations=10, schedule="per_color"), 2, 10, 1.0 / 600.0)
        n = m1.particle_count
        assert np.abs(q[start:start + n] - s1.particle_q.cpu().numpy()).max() <= 1e-5
        start += n


def test_cuda_graph_capture_replays_the_step():
    b = cloth_grid_builder(n=16)
    b.add_ground_plane()
    model = b.finalize("cuda")
    pipe = CollisionPipeline(model)
    solver = SolverVBD(model, iterations=5)
    s_eager = _run(model, solver, 2, 4, 1.0 / 600.0, pipe)
    s0, s1 = model.state(), model.state()
    contacts = pipe.contacts()
    solver.step(s0, s1, None, contacts, 1.0 / 600.0)  # sizes contact buffers before capture
    s0.assign(model.state())
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        with torch.cuda.graph(graph, stream=stream):
            for k in range(4):
                a, c = (s0, s1) if k % 2 == 0 else (s1, s0)
                pipe.collide(a, contacts)
                solver.step(a, c, None, contacts, 1.0 / 600.0)
    torch.cuda.current_stream().wait_stream(stream)
    s0.assign(model.state())
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()
    assert np.abs(s0.particle_q.cpu().numpy() - s_eager.particle_q.cpu().numpy()).max() <= 1e-6


def test_soft_contacts_match_oracle():
    rng = np.random.default_rng(0)
    b = sim.ModelBuilder()
    q = rng.uniform(-0.4, 0.4, size=(500, 3))
    q[:, 2] = rng.uniform(-0.01, 0.05, size=500)
    b.add_particles(q, (0, 0, 0), np.ones(500), radius=5e-3)
    b.add_ground_plane()
    b.add_shape_sphere(xform=(0.1, 0.0, 0.0), radius=0.2)
    b.set_coloring([np.arange(500)])
    model = b.finalize("cuda")
    state = model.state()
    c = model.contacts()
    model.collide(state, c, soft_contact_margin=0.01)
    torch.cuda.synchronize()
    n = int(c.soft_contact_count.item())
    got = sorted(zip(c.soft_contact_particle.cpu().numpy()[:n].tolist(), c.soft_contact_shape.cpu().numpy()[:n].tolist()))
    cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(
        model.particle_q.cpu().numpy(), model.particle_radius.cpu().numpy(), model.particle_flags.cpu().numpy(),
        model.shape_type, model.shape_transform, model.shape_scale, 0.01,
    )  # fmt: skip
    want = sorted(zip(p[:cnt].tolist(), s[:cnt].tolist()))
    assert n == cnt and got == want


def test_nonfinite_input_is_flagged_not_trapped():
    b = cloth_grid_builder(n=8)
    model = b.finalize("cuda")
    solver = SolverVBD(model, iterations=2)
    s0, s1 = model.state(), model.state()
    s0.particle_q[20, 0] = float("nan")
    solver.step(s0, s1, None, None, 1.0 / 600.0)
    assert solver.device_errors() & 1
    assert solver.device_errors() == 0  # cleared by the read
