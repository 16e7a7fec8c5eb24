"""The hand-written VBD adjoint against FP64 central finite differences of the forward step.

The reference VBD has no gradient (its kernels are compiled with enable_backward=False), so finite
differences are the only check: directional derivatives along seeded random directions of the
per-triangle Young's moduli and of the initial velocity, relative tolerance 1e-3.
"""

import numpy as np
import pytest
import torch

from newton_chysx_b200.adjoint import DifferentiableVBD, lame_from_young
from tests.helpers import cloth_grid_builder

pytestmark = pytest.mark.gpu

NU, H = 0.3, 1.0e-3


def _setup(n, precision, iterations=5):
    b = cloth_grid_builder(n=n, hanging=True, pin_top_corners=True, height=1.0, bend=1e-3)
    model = b.finalize("cuda")
    sim = DifferentiableVBD(model, iterations=iterations, precision=precision)
    rng = np.random.default_rng(3)
    T = model.tri_count
    E = torch.tensor(10.0 ** rng.uniform(3.5, 4.5, size=T), dtype=torch.float64, device="cuda")
    q0 = model.particle_q.to(torch.float64)
    qd0 = torch.zeros_like(q0)
    target = q0 + torch.tensor(rng.normal(0.0, 0.05, size=q0.shape), dtype=torch.float64, device="cuda")
    return model, sim, E, q0, qd0, target


def _loss_ml(sim, mu, lam, qd0, q0, target, substeps, dt):
    q, _ = sim.rollout(q0.to(sim.dtype), qd0.to(sim.dtype), mu, lam, dt, substeps)
    return ((q.to(torch.float64) - target) ** 2).sum(dim=1).mean()


def _loss(sim, E, qd0, q0, target, substeps, dt):
    mu, lam = lame_from_young(E, NU, H)
    return _loss_ml(sim, mu, lam, qd0, q0, target, substeps, dt)


@pytest.mark.parametrize("n,substeps", [(8, 6), (16, 10)])
def test_adjoint_matches_fp64_central_differences(n, substeps):
    """Directional derivatives along 8 seeded directions of (per-triangle E, initial velocity)."""
    model, sim, E, q0, qd0, target = _setup(n, "fp64")
    dt = 1.0 / 600.0
    mu0, lam0 = lame_from_young(E, NU, H)
    mu = mu0.clone().requires_grad_(True)
    lam = lam0.clone().requires_grad_(True)
    v0 = qd0.clone().requires_grad_(True)
    _loss_ml(sim, mu, lam, v0, q0, target, substeps, dt).backward()
    gmu, glam, gv = mu.grad.detach(), lam.grad.detach(), v0.grad.detach()
    rng = np.random.default_rng(11)
    h = 1e-4
    worst = 0.0
    for _ in range(8):
        dE = torch.tensor(rng.normal(size=E.shape), device="cuda", dtype=torch.float64)
        dv = torch.tensor(rng.normal(size=qd0.shape), device="cuda", dtype=torch.float64)
        dE, dv = dE / dE.abs().max(), dv / dv.norm()
        with torch.no_grad():
            mu_p, lam_p = lame_from_young(E * (1.0 + h * dE), NU, H)
            mu_m, lam_m = lame_from_young(E * (1.0 - h * dE), NU, H)
            fd = float(_loss_ml(sim, mu_p, lam_p, qd0 + h * dv, q0, target, substeps, dt)
                       - _loss_ml(sim, mu_m, lam_m, qd0 - h * dv, q0, target, substeps, dt))  # fmt: skip
            # the model stores mu and lambda in float32: predict with the perturbation actually applied
            d_mu = mu_p.float().double() - mu_m.float().double()
            d_lam = lam_p.float().double() - lam_m.float().double()
            ad = float((gmu * d_mu).sum() + (glam * d_lam).sum() + (gv * (2.0 * h * dv)).sum())
        worst = max(worst, abs(ad - fd) / max(abs(fd), 1e-30))
    assert worst <= 1e-3, worst


def test_fp32_adjoint_tracks_fp64():
    model, sim64, E, q0, qd0, target = _setup(12, "fp64")
    sim32 = DifferentiableVBD(model, iterations=5, precision="fp32")
    dt = 1.0 / 600.0
    grads = []
    for sim in (sim64, sim32):
        Ev = E.clone().requires_grad_(True)
        v0 = qd0.clone().requires_grad_(True)
        _loss(sim, Ev, v0, q0, target, 6, dt).backward()
        grads.append((Ev.grad.double(), v0.grad.double()))
    for a, b in zip(grads[0], grads[1], strict=True):
        assert (a - b).norm() / a.norm() <= 5e-2  # FP32 adjoint: a few percent after 6 substeps


def test_adjoint_with_ground_contact_matches_fp64_central_differences():
    """A 10 x 10 sheet pressed 1 mm into the ground and sliding at 0.3 m/s, so that every vertex has its contact's
    penalty and IPC friction terms active (contact damping off: no term switches with the sign of the normal
    velocity). Six substeps whose contacts are generated along the nominal trajectory and then held fixed, as the
    adjoint differentiates the step for its contact set: directional derivatives in (per-triangle E, initial
    velocity) against FP64 central differences, relative 1e-3."""
    from newton_chysx_b200 import CollisionPipeline, sim

    b = cloth_grid_builder(n=10, hanging=False, height=0.004, pin_top_corners=False, bend=1e-3)
    b.add_ground_plane(cfg=sim.ShapeConfig(ke=2.5e3, kd=0.0, mu=0.6))
    model = b.finalize("cuda")
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e3, 0.0, 0.5
    dsim = DifferentiableVBD(model, iterations=5, precision="fp64")
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    rng = np.random.default_rng(5)
    T = model.tri_count
    E = torch.tensor(10.0 ** rng.uniform(3.5, 4.5, size=T), dtype=torch.float64, device="cuda")
    q0 = model.particle_q.to(torch.float64)
    qd0 = torch.zeros_like(q0)
    qd0[:, 0] = 0.3
    target = q0 + torch.tensor(rng.normal(0.0, 0.01, size=q0.shape), dtype=torch.float64, device="cuda")
    dt, substeps = 1.0 / 600.0, 6

    mu0, lam0 = lame_from_young(E, NU, H)
    dsim.set_materials(mu0, lam0)
    contacts = []
    with torch.no_grad():
        q, qd = q0, qd0
        for _ in range(substeps):
            view = sim.State()
            view.particle_q = q.float().contiguous()
            c = pipe.contacts()
            pipe.collide(view, c)
            contacts.append(c)
            q, qd = dsim.substep(q, qd, mu0, lam0, dt, contacts=c)
    counts = [int(k.soft_contact_count.item()) for k in contacts]
    assert min(counts) == model.particle_count  # every vertex in contact at every substep

    def loss(mu, lam, v0):
        dsim.set_materials(mu, lam)
        q, qd = q0, v0
        for k in range(substeps):
            q, qd = dsim.substep(q, qd, mu, lam, dt, contacts=contacts[k])
        return ((q - target) ** 2).sum(dim=1).mean()

    mu = mu0.clone().requires_grad_(True)
    lam = lam0.clone().requires_grad_(True)
    v0 = qd0.clone().requires_grad_(True)
    loss(mu, lam, v0).backward()
    gmu, glam, gv = mu.grad.detach(), lam.grad.detach(), v0.grad.detach()
    assert gv.abs().max() > 0
    h, worst = 1e-4, 0.0
    for _ in range(6):
        dE = torch.tensor(rng.normal(size=E.shape), device="cuda", dtype=torch.float64)
        dv = torch.tensor(rng.normal(size=qd0.shape), device="cuda", dtype=torch.float64)
        dE, dv = dE / dE.abs().max(), dv / dv.norm()
        with torch.no_grad():
            mu_p, lam_p = lame_from_young(E * (1.0 + h * dE), NU, H)
            mu_m, lam_m = lame_from_young(E * (1.0 - h * dE), NU, H)
            fd = float(loss(mu_p, lam_p, qd0 + h * dv) - loss(mu_m, lam_m, qd0 - h * dv))
            d_mu = mu_p.float().double() - mu_m.float().double()
            d_lam = lam_p.float().double() - lam_m.float().double()
            ad = float((gmu * d_mu).sum() + (glam * d_lam).sum() + (gv * (2.0 * h * dv)).sum())
        worst = max(worst, abs(ad - fd) / max(abs(fd), 1e-30))
    assert worst <= 1e-3, worst


def test_adjoint_with_damping_matches_fp64_central_differences():
    """A hanging 8 x 8 sheet with membrane damping (tri_kd 1e-2) and bending damping (edge_kd 1e-3), whose terms
    depend on the positions at the start of the substep as well: the adjoint in (per-triangle E, initial velocity)
    against FP64 central differences over 6 substeps, relative 1e-3."""
    from newton_chysx_b200 import sim

    n = 8
    mu_, lam_ = 1.0e4 * H / (2.0 * (1.0 + NU)), 1.0e4 * H * NU / (1.0 - NU * NU)
    b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    b.add_cloth_grid(pos=(0.0, 0.0, 1.0), rot=sim.quat_from_axis_angle((1.0, 0.0, 0.0), np.pi * 0.5),
                     vel=(0.0, 0.0, 0.0), dim_x=n - 1, dim_y=n - 1, cell_x=1.0 / (n - 1), cell_y=1.0 / (n - 1),
                     mass=0.2 / (n * n), tri_ke=mu_, tri_ka=lam_, tri_kd=1e-2, edge_ke=5e-3, edge_kd=1e-3,
                     particle_radius=5e-3)  # fmt: skip
    flags = b.particle_flags
    flags[n * (n - 1)] &= ~int(sim.ParticleFlags.ACTIVE)
    flags[n * n - 1] &= ~int(sim.ParticleFlags.ACTIVE)
    b.set_particle_flags(flags)
    b.color(include_bending=True)
    model = b.finalize("cuda")
    assert float(model.tri_materials[:, 2].min()) > 0 and float(model.edge_bending_properties[:, 1].min()) > 0
    dsim = DifferentiableVBD(model, iterations=5, precision="fp64")
    rng = np.random.default_rng(7)
    E = torch.tensor(10.0 ** rng.uniform(3.5, 4.5, size=model.tri_count), dtype=torch.float64, device="cuda")
    q0 = model.particle_q.to(torch.float64)
    qd0 = torch.tensor(rng.normal(0.0, 0.2, size=q0.shape), dtype=torch.float64, device="cuda")
    target = q0 + torch.tensor(rng.normal(0.0, 0.05, size=q0.shape), dtype=torch.float64, device="cuda")
    dt, substeps = 1.0 / 600.0, 6
    mu0, lam0 = lame_from_young(E, NU, H)
    mu = mu0.clone().requires_grad_(True)
    lam = lam0.clone().requires_grad_(True)
    v0 = qd0.clone().requires_grad_(True)
    _loss_ml(dsim, mu, lam, v0, q0, target, substeps, dt).backward()
    gmu, glam, gv = mu.grad.detach(), lam.grad.detach(), v0.grad.detach()
    h, worst = 1e-4, 0.0
    for _ in range(6):
        dE = torch.tensor(rng.normal(size=E.shape), device="cuda", dtype=torch.float64)
        dv = torch.tensor(rng.normal(size=qd0.shape), device="cuda", dtype=torch.float64)
        dE, dv = dE / dE.abs().max(), dv / dv.norm()
        with torch.no_grad():
            mu_p, lam_p = lame_from_young(E * (1.0 + h * dE), NU, H)
            mu_m, lam_m = lame_from_young(E * (1.0 - h * dE), NU, H)
            fd = float(_loss_ml(dsim, mu_p, lam_p, qd0 + h * dv, q0, target, substeps, dt)
                       - _loss_ml(dsim, mu_m, lam_m, qd0 - h * dv, q0, target, substeps, dt))  # fmt: skip
            d_mu = mu_p.float().double() - mu_m.float().double()
            d_lam = lam_p.float().double() - lam_m.float().double()
            ad = float((gmu * d_mu).sum() + (glam * d_lam).sum() + (gv * (2.0 * h * dv)).sum())
        worst = max(worst, abs(ad - fd) / max(abs(fd), 1e-30))
    assert worst <= 1e-3, worst

    # the differentiated forward is the solver's step (damping included): FP64, per-color schedule
    from newton_chysx_b200 import SolverVBD

    with torch.no_grad():
        q_ad, qd_ad = dsim.rollout(q0, qd0, mu0, lam0, dt, substeps)
        solver = SolverVBD(model, iterations=5, precision="fp64", schedule="per_color", layout="csr")
        s0, s1 = sim.State(), sim.State()
        s0.particle_q, s0.particle_qd = q0.clone(), qd0.clone()
        s0.particle_f = torch.zeros_like(q0)
        s1.particle_q, s1.particle_qd, s1.particle_f = (torch.zeros_like(q0) for _ in range(3))
        for _ in range(substeps):
            solver.step(s0, s1, None, None, dt)
            s0, s1 = s1, s0
    assert (q_ad - s0.particle_q).abs().max().item() <= 1e-9
