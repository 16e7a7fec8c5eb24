"""The benchmarked kernel on the benchmark's instance distribution, against the FP64 oracle.

The batched benchmark steps 4,096 cloth instances whose grid sides are drawn from 16..128 vertices, with
Young's moduli log-uniform in [1e3, 1e6] Pa, bending stiffness log-uniform in [1e-5, 1e-3] and one to four
pinned corners, over a ground plane, through the 16-bit stencil persistent kernel. These tests run that
kernel, in each launch shape the autotuner chooses from, on a batch spanning the same ranges (sides 16, 37,
64, 101 and 128, each at both ends of the modulus and bending ranges), half of the instances falling freely
and half pressed 0.5 mm into the ground, and compare every substep with the FP64 oracle (the CPU restatement
of the reference step): from the same FP32 input, and along the trajectory. Tolerance: 1e-4 m (the cloth
side is 1 m)."""

import numpy as np
import pytest
import torch

from newton_chysx_b200 import CollisionPipeline, SolverVBD, sim
from oracle import vbd_oracle as orc
from tests.helpers import cloth_grid_builder, oracle_model_dict

pytestmark = pytest.mark.gpu

SIDES = (16, 37, 64, 101, 128)
SUBSTEPS = 8
DT = 1.0 / 600.0
TOL = 1e-4

SHAPES = {
    "occ3": dict(layout="ell16", min_blocks_per_sm=3),
    "occ4": dict(layout="ell16", min_blocks_per_sm=4),
    "occ2": dict(layout="ell16", min_blocks_per_sm=2),
    "paired": dict(layout="ell16", pair_vertices=True),
}


def _batch_model():
    top = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    k = 0
    for n in SIDES:
        for E, bend in ((1.0e3, 1.0e-3), (1.0e6, 1.0e-5)):
            height = 0.6 if k % 2 == 0 else 0.0045  # particle radius 5 mm: the second kind starts in contact
            b = cloth_grid_builder(n=n, E=E, bend=bend, hanging=False, height=height, pin_top_corners=False)
            corners = [0, n - 1, n * (n - 1), n * n - 1]
            flags = b.particle_flags
            for c in corners[: 1 + k % 4]:
                flags[c] &= ~int(sim.ParticleFlags.ACTIVE)
            b.set_particle_flags(flags)
            top.add_world(b)
            k += 1
    top.add_ground_plane()
    model = top.finalize("cuda")
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e3, 10.0, 0.5
    return model


@pytest.fixture(scope="module")
def batch():
    model = _batch_model()
    om = orc.Model(oracle_model_dict(model))
    r, fl = model.particle_radius.cpu().numpy(), model.particle_flags.cpu().numpy()

    def oracle_step(q, qd):
        qc = q.astype(np.float32).astype(np.float64)  # contacts from FP32 positions, as on the GPU
        cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(qc, r, fl, model.shape_type, model.shape_transform,
                                                         model.shape_scale, 0.01)  # fmt: skip
        c = orc.make_contacts(cnt, p, s, bp, bv, nn)
        _, q1, qd1 = orc.step(om, q, qd, None, c, DT, 10, precision=64, nthreads=orc.max_threads())
        return q1, qd1, cnt

    q = model.particle_q.cpu().numpy().astype(np.float64)
    qd = model.particle_qd.cpu().numpy().astype(np.float64)
    traj, contacts = [], []
    for _ in range(SUBSTEPS):
        q, qd, cnt = oracle_step(q, qd)
        traj.append(q.copy())
        contacts.append(cnt)
    return model, oracle_step, traj, contacts


@pytest.mark.parametrize("shape", list(SHAPES))
def test_benchmark_distribution_matches_fp64_oracle(batch, shape):
    model, oracle_step, traj64, contacts = batch
    assert min(contacts) > 0  # the pressed instances are in contact throughout
    solver = SolverVBD(model, iterations=10, schedule="persistent", **SHAPES[shape])
    assert solver.layout == "ell16" and solver.schedule == "persistent"
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    c = pipe.contacts()
    s0, s1 = model.state(), model.state()
    per_substep, along = [], []
    for k in range(SUBSTEPS):
        q_in = s0.particle_q.cpu().numpy().astype(np.float64)
        qd_in = s0.particle_qd.cpu().numpy().astype(np.float64)
        pipe.collide(s0, c)
        solver.step(s0, s1, None, c, DT)
        torch.cuda.synchronize()
        q_gpu = s1.particle_q.cpu().numpy().astype(np.float64)
        q_ref, _, _ = oracle_step(q_in, qd_in)
        per_substep.append(float(np.linalg.norm(q_gpu - q_ref, axis=1).max()))
        along.append(float(np.linalg.norm(q_gpu - traj64[k], axis=1).max()))
        s0, s1 = s1, s0
    assert solver.device_errors() == 0
    assert max(per_substep) <= TOL, per_substep
    assert max(along) <= TOL, along
