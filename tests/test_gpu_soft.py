"""GPU parity for springs and tetrahedra: the CUDA step against the reference's own kernel code (golden
soft block, float64) and against the FP64 oracle.

Tolerances (positions in metres; the block is 15 cm across):
  * FP32 kernels vs the float64 reference goldens: 1e-4 after each substep.
  * FP64 kernels vs the FP64 oracle on the same float32 model arrays: 1e-9.
"""

import numpy as np
import pytest
import torch

from newton_chysx_b200 import SolverVBD, _lib, sim
from oracle import vbd_oracle as orc
from tests.helpers import contacts_from_golden, load_golden, model_from_golden, oracle_model_dict
from tests.test_soft_builder import soft_block_builder

pytestmark = pytest.mark.gpu

GOLDEN = "step_soft_block.npz"
# (schedule, lanes per vertex, positions in shared memory)
LAUNCH = [("per_color", 1, "auto"), ("per_color", 4, "auto"), ("per_color", 32, "auto"), ("persistent", 1, "on"),
          ("persistent", 8, "on"), ("persistent", 4, "off")]  # fmt: skip


def _state(arr, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype, device="cuda")


def _substep(solver, g, s, dtype=torch.float32, contacts=True):
    st_in, st_out = sim.State(), sim.State()
    st_in.particle_q = _state(g[f"s{s}_q_in"], dtype)
    st_in.particle_qd = _state(g[f"s{s}_qd_in"], dtype)
    st_in.particle_f = _state(g[f"s{s}_f_ext"], dtype)
    st_out.particle_q = torch.zeros_like(st_in.particle_q)
    st_out.particle_qd = torch.zeros_like(st_in.particle_qd)
    solver.step(st_in, st_out, None, contacts_from_golden(g, s) if contacts else None, float(g["dt"]))
    torch.cuda.synchronize()
    return st_in, st_out


def _oracle_step(om, g, s, q, qd, f, contacts=True):
    oc = None
    if contacts:
        oc = orc.make_contacts(g[f"s{s}_contact_count"], g[f"s{s}_contact_particle"], g[f"s{s}_contact_shape"],
                               g[f"s{s}_contact_body_pos"], g[f"s{s}_contact_body_vel"], g[f"s{s}_contact_normal"])  # fmt: skip
    _, q_o, qd_o = orc.step(om, q, qd, f, oc, float(g["dt"]), int(g["iterations"]), precision=64)
    return q_o, qd_o


@pytest.mark.parametrize("schedule,lanes,shared", LAUNCH)
def test_fp32_soft_block_matches_reference_goldens(schedule, lanes, shared):
    g = load_golden(GOLDEN)
    model = model_from_golden(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                       schedule=schedule, lanes_per_vertex=lanes, positions_in_shared=shared)  # fmt: skip
    assert solver.layout == "csr" and solver.schedule == schedule and solver.lanes_per_vertex == lanes
    for s in range(int(g["substeps"])):
        st_in, st_out = _substep(solver, g, s)
        q_out = st_out.particle_q.cpu().numpy()
        assert np.abs(q_out - g[f"s{s}_q_out"]).max() <= 1e-4, (s, np.abs(q_out - g[f"s{s}_q_out"]).max())
        assert np.array_equal(st_in.particle_q.cpu().numpy(), q_out)
        qd = st_out.particle_qd.cpu().numpy()
        assert np.abs(qd - g[f"s{s}_qd_out"]).max() <= 1e-4 / float(g["dt"])
    assert solver.device_errors() & ~4 == 0


@pytest.mark.parametrize("schedule", ["per_color", "persistent"])
def test_fp64_soft_block_matches_fp64_oracle(schedule):
    g = load_golden(GOLDEN)
    model = model_from_golden(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                       precision="fp64", schedule=schedule)  # fmt: skip
    om = orc.Model(oracle_model_dict(model, float(g["friction_epsilon"]), float(g["beta"])))
    for s in range(int(g["substeps"])):
        _, st_out = _substep(solver, g, s, torch.float64)
        q_o, qd_o = _oracle_step(om, g, s, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"])
        assert np.abs(st_out.particle_q.cpu().numpy() - q_o).max() <= 1e-9
        assert np.abs(st_out.particle_qd.cpu().numpy() - qd_o).max() <= 1e-9 / float(g["dt"])


def _same_color_model(g):
    """The golden block recolored the reference's way (springs are not graph edges) with the anchor put in the
    color of one of its spring partners, so that spring's ends share a color."""
    model = model_from_golden(g)
    n = model.particle_count
    groups = sim.color_particles(n, g["model_tri_indices"], g["model_tri_materials"], g["model_edge_indices"],
                                 g["model_edge_bending_properties"], tet_indices=g["model_tet_indices"],
                                 tet_materials=g["model_tet_materials"])  # fmt: skip
    colors = np.zeros(n, dtype=np.int32)
    for c, grp in enumerate(groups):
        colors[grp] = c
    anchor, partner = g["model_spring_indices"][0]
    colors[anchor] = colors[partner]
    groups = [np.nonzero(colors == c)[0].astype(np.int32) for c in range(colors.max() + 1)]
    model.particle_color_groups = [torch.as_tensor(grp, device="cuda") for grp in groups if len(grp)]
    sp = g["model_spring_indices"]
    assert (colors[sp[:, 0]] == colors[sp[:, 1]]).any()
    return model


@pytest.mark.parametrize("schedule", ["per_color", "persistent"])
def test_same_color_springs_match_oracle(schedule):
    """Springs whose ends share a color are summed from the positions before the color's solve, as the
    reference's accumulate_spring_force_and_hessian does; the FP64 oracle does the same."""
    g = load_golden(GOLDEN)
    model = _same_color_model(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                       precision="fp64", schedule=schedule)  # fmt: skip
    om = orc.Model(oracle_model_dict(model, float(g["friction_epsilon"]), float(g["beta"])))
    for s in range(int(g["substeps"])):
        _, st_out = _substep(solver, g, s, torch.float64)
        q_o, _ = _oracle_step(om, g, s, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"])
        assert np.abs(st_out.particle_q.cpu().numpy() - q_o).max() <= 1e-9
    solver32 = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                         schedule=schedule)  # fmt: skip
    _, st_out = _substep(solver32, g, 0)
    q_o, _ = _oracle_step(om, g, 0, g["s0_q_in"], g["s0_qd_in"], g["s0_f_ext"])
    assert np.abs(st_out.particle_q.cpu().numpy() - q_o).max() <= 1e-4


def test_builder_worlds_persistent_matches_oracle():
    """Two soft blocks as worlds from the builder (soft grid, springs, coloring with tets), one CTA per world on
    the persistent schedule, against the FP64 oracle over the whole model, for two substeps."""
    inner = soft_block_builder()
    inner.color()
    b = sim.ModelBuilder()
    b.add_world(inner)
    b.add_world(inner)
    model = b.finalize("cuda")
    solver = SolverVBD(model, iterations=5, precision="fp64", schedule="persistent")
    assert solver.schedule == "persistent"
    om = orc.Model(oracle_model_dict(model))
    rng = np.random.default_rng(3)
    q = model.particle_q.double().cpu().numpy() + rng.normal(scale=2e-3, size=(model.particle_count, 3))
    qd = np.zeros_like(q)
    f = np.zeros_like(q)
    dt = 1.0 / 600.0
    for _ in range(2):
        st_in, st_out = sim.State(), sim.State()
        st_in.particle_q, st_in.particle_qd, st_in.particle_f = _state(q, torch.float64), _state(qd, torch.float64), _state(f, torch.float64)
        st_out.particle_q = torch.zeros_like(st_in.particle_q)
        st_out.particle_qd = torch.zeros_like(st_in.particle_qd)
        solver.step(st_in, st_out, None, None, dt)
        torch.cuda.synchronize()
        _, q_o, qd_o = orc.step(om, q, qd, f, None, dt, 5, precision=64)
        assert np.abs(st_out.particle_q.cpu().numpy() - q_o).max() <= 1e-9
        q, qd = q_o, qd_o


def test_soft_model_rejects_stencil_layouts():
    g = load_golden(GOLDEN)
    model = model_from_golden(g)
    for layout in ("ell", "ell16", "ring"):
        with pytest.raises(_lib.VbdError, match="unsupported"):
            SolverVBD(model, iterations=2, layout=layout, schedule="persistent")
    solver = SolverVBD(model, iterations=2)
    assert solver.layout == "csr"


def test_soft_adjoint_matches_fp64_central_differences():
    """The damped tetrahedral block hung by springs (the soft-body golden scene, 4 substeps, no ground contact):
    the recorded forward equals the solver's FP64 step (same-color springs at the color's start state, as the
    solver's pre-pass has them), and the adjoint in the initial velocity matches FP64 central differences along 6
    seeded directions, relative 1e-3."""
    from newton_chysx_b200.adjoint import DifferentiableVBD

    g = load_golden(GOLDEN)
    model = model_from_golden(g)
    iters, dt, substeps = int(g["iterations"]), float(g["dt"]), 4
    dsim = DifferentiableVBD(model, iterations=iters, precision="fp64")
    mu = model.tri_materials[:, 0].double().clone()
    lam = model.tri_materials[:, 1].double().clone()
    q0 = torch.as_tensor(g["s0_q_in"], dtype=torch.float64, device="cuda")
    qd0 = torch.as_tensor(g["s0_qd_in"], dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(9)
    target = q0 + torch.tensor(rng.normal(0.0, 0.01, size=q0.shape), dtype=torch.float64, device="cuda")

    def loss(v0):
        q, _ = dsim.rollout(q0, v0, mu, lam, dt, substeps)
        return ((q - target) ** 2).sum(dim=1).mean()

    with torch.no_grad():  # the differentiated forward is the solver's step
        q_ad, _ = dsim.rollout(q0, qd0, mu, lam, dt, substeps)
        solver = SolverVBD(model, iterations=iters, precision="fp64", schedule="per_color",
                           friction_epsilon=float(g["friction_epsilon"]))  # fmt: skip
        s0, s1 = sim.State(), sim.State()
        s0.particle_q, s0.particle_qd, s0.particle_f = q0.clone(), qd0.clone(), torch.zeros_like(q0)
        s1.particle_q, s1.particle_qd, s1.particle_f = (torch.zeros_like(q0) for _ in range(3))
        for _ in range(substeps):
            solver.step(s0, s1, None, None, dt)
            s0, s1 = s1, s0
        assert (q_ad - s0.particle_q).abs().max().item() <= 1e-9
    v0 = qd0.clone().requires_grad_(True)
    loss(v0).backward()
    gv = v0.grad.detach()
    assert gv.abs().max() > 0
    h, worst = 1e-4, 0.0
    for _ in range(6):
        dv = torch.tensor(rng.normal(size=qd0.shape), device="cuda", dtype=torch.float64)
        dv = dv / dv.norm()
        with torch.no_grad():
            fd = float(loss(qd0 + h * dv) - loss(qd0 - h * dv))
        ad = float((gv * (2.0 * h * dv)).sum())
        worst = max(worst, abs(ad - fd) / max(abs(fd), 1e-30))
    assert worst <= 1e-3, worst


def test_soft_step_graph_capture_replays_identically():
    g = load_golden(GOLDEN)
    model = _same_color_model(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]))
    st_in, st_out = sim.State(), sim.State()
    st_in.particle_q = _state(g["s0_q_in"])
    st_in.particle_qd = _state(g["s0_qd_in"])
    st_in.particle_f = _state(g["s0_f_ext"])
    st_out.particle_q = torch.zeros_like(st_in.particle_q)
    st_out.particle_qd = torch.zeros_like(st_in.particle_qd)
    q0 = st_in.particle_q.clone()
    solver.step(st_in, st_out, None, None, float(g["dt"]))
    torch.cuda.synchronize()
    eager = st_out.particle_q.clone()
    st_in.particle_q.copy_(q0)
    graph = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(graph, stream=s):
            solver.step(st_in, st_out, None, None, float(g["dt"]))
    torch.cuda.current_stream().wait_stream(s)
    st_in.particle_q.copy_(q0)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(st_out.particle_q, eager)


@pytest.mark.parametrize("lanes,shared", [(4, "auto"), (8, "auto"), (8, "off"), (1, "auto")])
def test_instance_per_warp_matches(lanes, shared):
    """One warp per instance on the persistent CSR kernel: the golden soft block in FP32 (1e-4) and FP64 (1e-9
    against the oracle), and a batch of builder blocks against one instance per CTA."""
    g = load_golden(GOLDEN)
    model = model_from_golden(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                       schedule="persistent", lanes_per_vertex=lanes, positions_in_shared=shared,
                       instance_per_warp=True)  # fmt: skip
    for s in range(int(g["substeps"])):
        _, st_out = _substep(solver, g, s)
        assert np.abs(st_out.particle_q.cpu().numpy() - g[f"s{s}_q_out"]).max() <= 1e-4
    solver64 = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                         precision="fp64", schedule="persistent", lanes_per_vertex=lanes, instance_per_warp=True)  # fmt: skip
    om = orc.Model(oracle_model_dict(model, float(g["friction_epsilon"]), float(g["beta"])))
    _, st_out = _substep(solver64, g, 0, torch.float64)
    q_o, _ = _oracle_step(om, g, 0, g["s0_q_in"], g["s0_qd_in"], g["s0_f_ext"])
    assert np.abs(st_out.particle_q.cpu().numpy() - q_o).max() <= 1e-9
    inner = soft_block_builder()
    inner.color()
    b = sim.ModelBuilder()
    for _ in range(20):
        b.add_world(inner)
    bm = b.finalize("cuda")
    runs = []
    for warp in (True, False):
        sv = SolverVBD(bm, iterations=5, schedule="persistent", lanes_per_vertex=lanes, positions_in_shared=shared,
                       instance_per_warp=warp)  # fmt: skip
        s0, s1 = bm.state(), bm.state()
        for _ in range(3):
            sv.step(s0, s1, None, None, 1.0 / 600.0)
            s0, s1 = s1, s0
        torch.cuda.synchronize()
        runs.append(s0.particle_q.clone())
    assert (runs[0] - runs[1]).abs().max().item() <= 1e-6


def test_instance_per_warp_needs_csr_persistent():
    g = load_golden(GOLDEN)
    model = model_from_golden(g)
    for kw in (dict(schedule="per_color"), dict(schedule="persistent", lanes_per_vertex=16)):
        with pytest.raises(_lib.VbdError, match="invalid argument"):
            SolverVBD(model, iterations=2, instance_per_warp=True, **kw)


def test_damped_soft_block_falls_freely():
    """The pattern of test_cloth.py:1026-1076 for volumetric elements: a tetrahedral block with tet damping and a
    spring between two of its corners, released at rest, falls as free particles (elastic and damping forces stay
    zero under a uniform translation). The spring is undamped: the reference's spring damping acts on each end's
    own displacement, h_d (x_prev - x) (particle_vbd_kernels.py:2288-2290), so a damped spring slows the fall
    (by 8.9 mm here in the oracle as on the GPU)."""
    b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    b.add_soft_grid(pos=(0.0, 0.0, 0.25), rot=sim.quat_identity(), vel=(0.0, 0.0, 0.0), dim_x=3, dim_y=2, dim_z=2,
                    cell_x=0.05, cell_y=0.05, cell_z=0.05, density=500.0, k_mu=2.0e4, k_lambda=3.0e4, k_damp=1.0e-2,
                    tri_ke=10.0, tri_ka=10.0, tri_kd=1e-2, edge_ke=1e-2, edge_kd=1e-3)  # fmt: skip
    b.add_spring(0, b.particle_count - 1, 100.0, 0.0, 0.0)
    b.color()
    model = b.finalize("cuda")
    solver = SolverVBD(model, iterations=5)
    s0, s1 = model.state(), model.state()
    q0 = s0.particle_q.clone()
    dt, n = 1.0 / 600.0, 60
    for _ in range(n):
        solver.step(s0, s1, None, None, dt)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    diff = (s0.particle_q - q0).cpu().numpy()
    expected = -9.81 * dt * dt * n * (n + 1) / 2  # implicit Euler
    # FP32 positions near z = 0.3 m round by up to 1.5e-8 m per substep; every particle moves alike, so the
    # rounding biases the velocity the same way each step and adds up to about n^2 / 2 * 1.5e-8 = 2.7e-5 m
    assert np.abs(diff[:, 2] - expected).max() <= 1e-4
    assert np.abs(diff[:, :2]).max() <= 1e-5
    assert solver.device_errors() & ~4 == 0
