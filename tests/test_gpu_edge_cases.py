"""Edge cases of the step on the GPU: models without triangles or hinges, springs only, every particle fixed,
zero iterations, an empty color group, more contacts on a particle than contact slots, and shape tables at and
beyond the 16-shape limit. Where a result is defined, the FP64 path is held to the FP64 oracle (1e-9)."""

import ctypes as C

import numpy as np
import pytest
import torch

from newton_chysx_b200 import SolverVBD, _lib, sim
from oracle import vbd_oracle as orc
from tests.helpers import cloth_grid_builder, oracle_model_dict

pytestmark = pytest.mark.gpu
DT = 1.0 / 600.0


def _states(model, q, qd, dtype):
    s0, s1 = sim.State(), sim.State()
    s0.particle_q = torch.as_tensor(q, dtype=dtype, device="cuda").contiguous()
    s0.particle_qd = torch.as_tensor(qd, dtype=dtype, device="cuda").contiguous()
    s0.particle_f = torch.zeros_like(s0.particle_q)
    s1.particle_q = torch.zeros_like(s0.particle_q)
    s1.particle_qd = torch.zeros_like(s0.particle_q)
    return s0, s1


def _fp64_vs_oracle(model, iterations, contacts_fn=None, substeps=2, **kw):
    solver = SolverVBD(model, iterations=iterations, precision="fp64", **kw)
    om = orc.Model(oracle_model_dict(model))
    q = model.particle_q.double().cpu().numpy()
    qd = model.particle_qd.double().cpu().numpy()
    for _ in range(substeps):
        s0, s1 = _states(model, q, qd, torch.float64)
        solver.step(s0, s1, None, None, DT)
        torch.cuda.synchronize()
        _, q_o, qd_o = orc.step(om, q, qd, None, None, DT, iterations, precision=64)
        assert np.abs(s1.particle_q.cpu().numpy() - q_o).max() <= 1e-9
        assert np.abs(s1.particle_qd.cpu().numpy() - qd_o).max() <= 1e-9 / DT
        q, qd = q_o, qd_o
    return q


def test_particles_only_fall_freely():
    b = sim.ModelBuilder()
    b.add_particles(np.random.default_rng(0).uniform(-1.0, 1.0, (50, 3)), (0.0, 0.0, 1.0), 0.1)
    b.color()
    model = b.finalize("cuda")
    assert model.tri_count == 0 and model.edge_count == 0 and len(model.particle_color_groups) == 1
    q = _fp64_vs_oracle(model, 5)
    # free fall: x = x0 + v0 t + g t^2 dt-discretised by implicit Euler: v_n = v0 + n g dt, x_n = x0 + dt sum v_k
    v1, v2 = 1.0 - 9.81 * DT, 1.0 - 2 * 9.81 * DT
    np.testing.assert_allclose(q[:, 2] - model.particle_q.double().cpu().numpy()[:, 2], DT * (v1 + v2), atol=1e-12)


def test_spring_chain_matches_oracle():
    """A chain of particles joined by springs only (no triangles): every spring's ends share the single color,
    so all springs go through the same-color pre-pass."""
    b = sim.ModelBuilder()
    n = 12
    b.add_particles([(0.1 * i, 0.0, 1.0) for i in range(n)], (0.0, 0.0, 0.0), 0.05)
    flags = b.particle_flags
    flags[0] = 0
    b.set_particle_flags(flags)
    b.add_springs(np.arange(n - 1), np.arange(1, n), 500.0, 0.5)
    b.color()
    model = b.finalize("cuda")
    assert len(model.particle_color_groups) == 1
    _fp64_vs_oracle(model, 6, substeps=3)


def test_all_fixed_particles_do_not_move():
    b = cloth_grid_builder(n=8)
    b.set_particle_flags(np.zeros(b.particle_count, dtype=np.int32))
    model = b.finalize("cuda")
    solver = SolverVBD(model, iterations=4)
    s0, s1 = model.state(), model.state()
    q0 = s0.particle_q.clone()
    s0.particle_qd.fill_(3.0)
    solver.step(s0, s1, None, None, DT)
    torch.cuda.synchronize()
    assert torch.equal(s1.particle_q, q0)
    assert torch.count_nonzero(s1.particle_qd) == 0
    assert solver.device_errors() == 0


def test_zero_iterations_is_the_inertial_prediction():
    b = cloth_grid_builder(n=8)
    model = b.finalize("cuda")
    _fp64_vs_oracle(model, 0)


def test_empty_color_group_is_skipped():
    b = cloth_grid_builder(n=8)
    groups = b.particle_color_groups
    b.particle_color_groups = groups[:1] + [np.zeros(0, dtype=np.int32)] + groups[1:]
    model = b.finalize("cuda")
    for schedule in ("per_color", "persistent"):
        _fp64_vs_oracle(model, 3, schedule=schedule)


def test_contact_slot_overflow_is_flagged():
    """More contacts on one particle than contact slots: the extra contacts are dropped and the device error
    word says so, without a trap."""
    b = sim.ModelBuilder()
    b.add_particles([(0.0, 0.0, 0.001)], (0.0, 0.0, 0.0), 1.0, radius=0.01)
    b.color()
    for _ in range(3):
        b.add_ground_plane()
    model = b.finalize("cuda")
    solver = SolverVBD(model, iterations=2, contact_slots=2)
    pipe = sim.CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    s0, s1 = model.state(), model.state()
    pipe.collide(s0, contacts)
    solver.step(s0, s1, None, contacts, DT)
    torch.cuda.synchronize()
    assert int(contacts.soft_contact_count.item()) == 3
    assert solver.device_errors() & 2
    assert torch.isfinite(s1.particle_q).all()


def test_shape_table_limit():
    lib = _lib.load()
    dev = torch.device("cuda")
    q = torch.zeros((4, 3), device=dev)
    r = torch.full((4,), 0.01, device=dev)
    fl = torch.ones(4, dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    out_i = torch.zeros(64 * 17, dtype=torch.int32, device=dev)
    out_f = torch.zeros((64 * 17, 3), device=dev)
    ip, fp = C.POINTER(C.c_int32), C.POINTER(C.c_float)
    for S, want in ((16, _lib.VBD_OK), (17, _lib.VBD_ERR_INVALID_ARGUMENT)):
        st = np.full(S, 1, dtype=np.int32)
        sx = np.tile(np.array([0, 0, 0, 0, 0, 0, 1], dtype=np.float32), (S, 1))
        ss = np.zeros((S, 3), dtype=np.float32)
        rc = lib.vbd_soft_contacts_shapes(4, q.data_ptr(), r.data_ptr(), fl.data_ptr(), S, st.ctypes.data_as(ip),
                                          sx.ctypes.data_as(fp), ss.ctypes.data_as(fp), 0.01, 64 * 17, cnt.data_ptr(),
                                          out_i.data_ptr(), out_i.data_ptr(), out_f.data_ptr(), out_f.data_ptr(),
                                          out_f.data_ptr(), None)  # fmt: skip
        assert rc == want
    torch.cuda.synchronize()
    bad = np.array([8], dtype=np.int32)  # MESH: no analytic SDF here
    rc = lib.vbd_soft_contacts_shapes(4, q.data_ptr(), r.data_ptr(), fl.data_ptr(), 1, bad.ctypes.data_as(ip),
                                      np.array([0, 0, 0, 0, 0, 0, 1], dtype=np.float32).ctypes.data_as(fp),
                                      np.zeros(3, dtype=np.float32).ctypes.data_as(fp), 0.01, 64, cnt.data_ptr(),
                                      out_i.data_ptr(), out_i.data_ptr(), out_f.data_ptr(), out_f.data_ptr(),
                                      out_f.data_ptr(), None)  # fmt: skip
    assert rc == _lib.VBD_ERR_UNSUPPORTED


@pytest.mark.parametrize("layout,schedule", [("csr", "per_color"), ("ell", "per_color"), ("ell", "persistent"),
                                             ("ell16", "persistent")])  # fmt: skip
def test_sliver_triangles_match_oracle(layout, schedule):
    """Triangles whose rest area is ~1e-6 of nominal (the precision stress sheet at 16 x 16): the stencil records
    carry mu and lambda times the area, which for slivers falls below the 1e-6 floor the reference applies to
    |lambda + mu|; the floor must act on the material values, as in the reference. FP64 against the FP64 oracle
    (1e-7: the slivers make the 3x3 blocks ill-conditioned, which amplifies the order of the sums)."""
    import bench

    b, sites = bench.build_precision_model(n=16, seed=4, sliver_fraction=0.05)
    assert len(sites) > 0
    model = b.finalize("cuda")
    solver = SolverVBD(model, iterations=5, precision="fp64", schedule=schedule, layout=layout)
    assert solver.layout == layout
    om = orc.Model(oracle_model_dict(model))
    q = model.particle_q.double().cpu().numpy()
    qd = np.zeros_like(q)
    for _ in range(3):
        s0, s1 = _states(model, q, qd, torch.float64)
        solver.step(s0, s1, None, None, DT)
        torch.cuda.synchronize()
        _, q_o, qd_o = orc.step(om, q, qd, None, None, DT, 5, precision=64)
        assert np.abs(s1.particle_q.cpu().numpy() - q_o).max() <= 1e-7
        q, qd = q_o, qd_o


def test_tiny_material_falls_back_to_csr():
    """A triangle with 0 < |lambda + mu| < 1e-6 needs the reference's floor on the material values: the stencil
    layouts refuse the model and the automatic choice takes CSR."""
    b = cloth_grid_builder(n=8)
    mats = b.tri_materials
    mats[3, :2] = (4.0e-7, 1.0e-7)
    b._tri_mat = [mats]
    model = b.finalize("cuda")
    with pytest.raises(_lib.VbdError, match="unsupported"):
        SolverVBD(model, iterations=2, schedule="persistent", layout="ell16")
    assert SolverVBD(model, iterations=2, schedule="persistent").layout == "csr"
    _fp64_vs_oracle(model, 3)
