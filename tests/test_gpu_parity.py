"""GPU parity: the CUDA step (through the C ABI) against the reference's own kernel code (golden
vectors) and against the CPU oracle.

Tolerances (positions in metres; the cloth side is 1 m, so these are relative to it):
  * FP32 kernels vs float64 reference goldens: 1e-4 after each substep (FP32 rounding plus the
    float32 rounding of the model arrays).
  * FP64 kernels vs the FP64 oracle on the same float32 model arrays: 1e-9.
"""

import numpy as np
import pytest
import torch

from newton_chysx_b200 import SolverVBD, _lib, sim
from oracle import vbd_oracle as orc
from tests.helpers import (cloth_grid_builder, contacts_from_golden, golden_body_contacts_kw, golden_body_states,
                           golden_solver_kw, load_golden, model_from_golden, oracle_model_dict)

pytestmark = pytest.mark.gpu

# step_grid_bodies: shapes on two bodies moved by an external rigid solver (integrate_with_external_rigid_solver)
FIXTURES = ["step_grid_ground.npz", "step_grid_sphere.npz", "step_complex_rest_angle.npz", "step_grid_bodies.npz"]
# (schedule, lanes per vertex, positions in shared memory, element layout)
LAUNCH = [("per_color", 1, "auto", "ell"), ("per_color", 1, "auto", "csr"), ("per_color", 4, "auto", "csr"),
          ("persistent", 1, "on", "ell"), ("persistent", 1, "off", "ell"), ("persistent", 1, "on", "csr"),
          ("persistent", 8, "on", "csr"), ("persistent", 32, "on", "csr"), ("persistent", 4, "off", "csr"),
          ("persistent", 1, "on", "ell16"), ("persistent", 1, "off", "ell16"), ("persistent", 1, "on", "ring"),
          ("persistent", 1, "off", "ring")]


def _state(arr, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype, device="cuda")


def _run_golden_substep(solver, g, s, dtype=torch.float32):
    st_in, st_out = sim.State(), sim.State()
    st_in.particle_q = _state(g[f"s{s}_q_in"], dtype)
    st_in.particle_qd = _state(g[f"s{s}_qd_in"], dtype)
    st_in.particle_f = _state(g[f"s{s}_f_ext"], dtype)
    st_out.particle_q = torch.zeros_like(st_in.particle_q)
    st_out.particle_qd = torch.zeros_like(st_in.particle_qd)
    golden_body_states(g, s, st_in, st_out)
    contacts = contacts_from_golden(g, s)
    solver.step(st_in, st_out, None, contacts, float(g["dt"]))
    torch.cuda.synchronize()
    return st_in, st_out


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("schedule,lanes,shared,layout", LAUNCH)
def test_fp32_step_matches_reference_goldens(name, schedule, lanes, shared, layout):
    g = load_golden(name)
    model = model_from_golden(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                       rigid_avbd_beta=float(g["beta"]), schedule=schedule, lanes_per_vertex=lanes,
                       positions_in_shared=shared, layout=layout, **golden_solver_kw(g))  # fmt: skip
    assert solver.schedule == schedule and solver.lanes_per_vertex == lanes and solver.layout == layout
    assert (solver.shared_bytes > 0) == (schedule == "persistent" and shared == "on")
    for s in range(int(g["substeps"])):
        st_in, st_out = _run_golden_substep(solver, g, s)
        q_out = st_out.particle_q.cpu().numpy()
        assert np.abs(q_out - g[f"s{s}_q_out"]).max() <= 1e-4
        # reference side effect: state_in.particle_q holds the solution too
        assert np.array_equal(st_in.particle_q.cpu().numpy(), q_out)
        qd = st_out.particle_qd.cpu().numpy()
        assert np.abs(qd - g[f"s{s}_qd_out"]).max() <= 1e-4 / float(g["dt"])
        # particles that are not ACTIVE never move (test_cloth.py:944-948)
        fixed = (g["model_particle_flags"] & 1) == 0
        assert np.array_equal(q_out[fixed], g[f"s{s}_q_in"][fixed].astype(np.float32))
    assert solver.device_errors() & ~4 == 0


@pytest.mark.parametrize("occ,shared", [(0, "off"), (3, "off"), (4, "off"), (0, "on")])
def test_paired_vertices_match_reference_goldens(occ, shared):
    """Two vertices per thread in paired FP32 instructions: the same substeps as the goldens and, up to the
    compiler's different fusing of multiplies and adds, as one vertex per thread."""
    g = load_golden("step_grid_sphere.npz")
    model = model_from_golden(g)
    kw = dict(iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
              rigid_avbd_beta=float(g["beta"]), schedule="persistent", layout="ell16", positions_in_shared=shared,
              min_blocks_per_sm=occ)  # fmt: skip
    paired = SolverVBD(model, pair_vertices=True, **kw)
    plain = SolverVBD(model, **kw)
    for s in range(int(g["substeps"])):
        _, out_s = _run_golden_substep(paired, g, s)
        _, out_p = _run_golden_substep(plain, g, s)
        q = out_s.particle_q.cpu().numpy()
        assert np.abs(q - g[f"s{s}_q_out"]).max() <= 1e-4
        assert (out_s.particle_q - out_p.particle_q).abs().max().item() <= 1e-5
    assert paired.device_errors() & ~4 == 0


@pytest.mark.parametrize("occ", [0, 4])
def test_paired_vertices_on_a_batch(occ):
    """Paired vertices on three instances of different sizes (color ranges longer than twice the block, odd
    lengths, so threads take several pairs and some a lone vertex), with ground contact, pinned corners and an
    inactive triangle, for five substeps, against one vertex per thread."""
    b = sim.ModelBuilder()
    for n in (24, 47, 72):
        b.add_world(cloth_grid_builder(n=n, hanging=False, height=0.01))
    b.add_ground_plane()
    mats = b.tri_materials
    mats[5, :2] = 0.0  # one triangle with mu = lambda = 0 (skipped by the sweep)
    b._tri_mat = [mats]
    model = b.finalize("cuda")
    kw = dict(iterations=10, schedule="persistent", layout="ell16", positions_in_shared="off", min_blocks_per_sm=occ)
    paired, plain = SolverVBD(model, pair_vertices=True, **kw), SolverVBD(model, **kw)
    pipe = sim.CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    runs = []
    for solver in (paired, plain):
        s0, s1 = model.state(), model.state()
        for _ in range(5):
            pipe.collide(s0, contacts)
            solver.step(s0, s1, None, contacts, 1.0 / 600.0)
            s0, s1 = s1, s0
        torch.cuda.synchronize()
        runs.append(s0.particle_q.clone())
    assert torch.isfinite(runs[0]).all()
    assert (runs[0] - runs[1]).abs().max().item() <= 1e-5
    assert paired.device_errors() & ~4 == 0


def test_paired_vertices_need_fp32_ell16_persistent():
    g = load_golden("step_grid_sphere.npz")
    model = model_from_golden(g)
    for kw in (dict(layout="ell"), dict(layout="csr"), dict(precision="mixed"), dict(schedule="per_color")):
        args = dict(dict(schedule="persistent", layout="ell16"), **kw)
        with pytest.raises(_lib.VbdError, match="invalid argument|unsupported"):
            SolverVBD(model, iterations=2, pair_vertices=True, **args)
    # the paired bending has no damping term
    damped = model_from_golden(load_golden("step_grid_ground.npz"))
    with pytest.raises(_lib.VbdError, match="unsupported"):
        SolverVBD(damped, iterations=2, pair_vertices=True, schedule="persistent", layout="ell16")


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("schedule,layout", [("per_color", "ell"), ("per_color", "csr"), ("persistent", "ell"),
                                             ("persistent", "csr"), ("persistent", "ell16"), ("persistent", "ring")])
def test_fp64_step_matches_fp64_oracle(name, schedule, layout):
    """Every layout in FP64 against the FP64 oracle; step_grid_ground and step_complex_rest_angle carry hinge
    damping, which the 16-bit stencil layout reads from its side array and the one-ring layout evaluates per
    damped hinge."""
    g = load_golden(name)
    model = model_from_golden(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), friction_epsilon=float(g["friction_epsilon"]),
                       rigid_avbd_beta=float(g["beta"]), precision="fp64", schedule=schedule, layout=layout,
                       **golden_solver_kw(g))  # fmt: skip
    om = orc.Model(oracle_model_dict(model, float(g["friction_epsilon"]), float(g["beta"])))
    for s in range(int(g["substeps"])):
        st_in, st_out = _run_golden_substep(solver, g, s, torch.float64)
        c = contacts_from_golden(g, s)
        oc = orc.make_contacts(int(c.soft_contact_count.item()), c.soft_contact_particle.cpu().numpy(),
                               c.soft_contact_shape.cpu().numpy(), c.soft_contact_body_pos.cpu().numpy(),
                               c.soft_contact_body_vel.cpu().numpy(), c.soft_contact_normal.cpu().numpy(),
                               **golden_body_contacts_kw(g, s, fp32=True))  # fmt: skip
        _, q_o, qd_o = orc.step(om, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], oc, float(g["dt"]),
                                int(g["iterations"]), precision=64)  # fmt: skip
        assert np.abs(st_out.particle_q.cpu().numpy() - q_o).max() <= 1e-9
        assert np.abs(st_out.particle_qd.cpu().numpy() - qd_o).max() <= 1e-9 / float(g["dt"])


@pytest.mark.parametrize("layout", ["ell", "csr"])
def test_mixed_precision_matches_and_reports_residuals(layout):
    g = load_golden("step_grid_ground.npz")
    model = model_from_golden(g)
    solver = SolverVBD(model, iterations=int(g["iterations"]), precision="mixed", fp64_solve_threshold=1.0,
                       layout=layout)  # fmt: skip
    st_in, st_out = _run_golden_substep(solver, g, 0)
    assert np.abs(st_out.particle_q.cpu().numpy() - g["s0_q_out"]).max() <= 1e-4
    res = solver.residuals()
    assert res.shape == (int(g["iterations"]),) and np.all(res > 0) and np.all(np.isfinite(res))
