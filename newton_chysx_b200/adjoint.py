"""Differentiable VBD substeps: the hand-written adjoint of the C ABI behind ``torch.autograd``.

``vbd_step`` has a hand-written reverse, ``vbd_adjoint_step``. Its forward pass ``vbd_record_step``
keeps the positions at the start of every iteration (per-iteration checkpoints). The reverse pass
recomputes the per-color states of one iteration from its checkpoint and walks the colors backwards.
Gradients flow to the input positions and velocities and to the triangles' Lame coefficients
(``Model.tri_materials[:, 0:2]``), hence to anything they are computed from, e.g. per-triangle
Young's moduli. Membranes, hinges, tetrahedra and springs take part with their damping.

The reference VBD has no gradient: its kernels are built with ``enable_backward=False``
(``newton/_src/solvers/vbd/particle_vbd_kernels.py:27-28``). The check is against central finite
differences of the forward step (``tests/test_gpu_adjoint.py``, ``bench.py --workload adjoint``).
Particle-shape contacts against static shapes take part: each substep's contacts (``CollisionPipeline.collide``)
are kept with it, and the reverse differentiates the step for that contact set (points, normals and stiffness
held fixed) through the contacts' penalty, friction and damping terms in the position and in the substep's start
position. The AVBD penalty ramp must be off (``rigid_avbd_beta = 0``, the default).
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .sim import Contacts, Model
from .solver_vbd import SolverVBD, contacts_desc


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class DifferentiableVBD:
    """A ``SolverVBD`` set up for differentiation (per-color schedule, adjacency layout)."""

    def __init__(self, model: Model, iterations: int = 10, precision: str = "fp32"):
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be 'fp32' or 'fp64'")
        self.model = model
        self.solver = SolverVBD(model, iterations=iterations, precision=precision, schedule="per_color", layout="csr")
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.iterations = iterations
        self._lib = _lib.load()

    def set_materials(self, tri_mu: torch.Tensor, tri_lambda: torch.Tensor):
        """Writes the triangles' Lame coefficients into the model (float32) and re-packs it."""
        m = self.model
        with torch.no_grad():
            m.tri_materials[:, 0].copy_(tri_mu.detach().to(torch.float32))
            m.tri_materials[:, 1].copy_(tri_lambda.detach().to(torch.float32))
        self.solver.notify_model_changed()

    def substep(self, q, qd, tri_mu, tri_lambda, dt, particle_f=None, contacts: Contacts | None = None):
        """One differentiable substep; ``contacts``: this substep's particle-shape contacts (static shapes), copied
        for the reverse pass."""
        return _Substep.apply(self, q, qd, tri_mu, tri_lambda, float(dt), particle_f, self._keep(contacts))

    def rollout(self, q0, qd0, tri_mu, tri_lambda, dt, substeps, particle_f=None, pipeline=None):
        """``substeps`` differentiable substeps from (q0, qd0); returns the final (q, qd). With a
        ``CollisionPipeline`` each substep generates its contacts from its start positions."""
        self.set_materials(tri_mu, tri_lambda)
        q, qd = q0, qd0
        contacts = pipeline.contacts() if pipeline is not None else None
        for _ in range(substeps):
            c = None
            if pipeline is not None:
                view = _PositionsView(q.detach().to(torch.float32).contiguous())
                pipeline.collide(view, contacts)
                c = self._keep(contacts)
            q, qd = _Substep.apply(self, q, qd, tri_mu, tri_lambda, float(dt), particle_f, c)
        return q, qd

    def _keep(self, contacts):
        """A copy of the contact arrays (the pipeline rewrites its own every substep), or None."""
        if contacts is None or self.model.shape_count == 0:
            return None
        if bool((getattr(self.model, "_shape_body_host", None) is not None) and
                (self.model._shape_body_host >= 0).any()):  # fmt: skip
            raise NotImplementedError("differentiable contacts cover static shapes only")
        keep = Contacts(int(contacts.soft_contact_max), self.model.device)
        for name in ("soft_contact_count", "soft_contact_particle", "soft_contact_shape", "soft_contact_body_pos",
                     "soft_contact_body_vel", "soft_contact_normal"):  # fmt: skip
            getattr(keep, name).copy_(getattr(contacts, name))
        return keep


class _PositionsView:
    """The one state field contact generation reads."""

    def __init__(self, particle_q):
        self.particle_q = particle_q
        self.body_q = None


class _Substep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sim: DifferentiableVBD, q, qd, tri_mu, tri_lambda, dt, particle_f, contacts):
        n = sim.model.particle_count
        dev = sim.model.device
        q = q.detach().to(sim.dtype).contiguous()
        qd = qd.detach().to(sim.dtype).contiguous()
        f = None if particle_f is None else particle_f.detach().to(sim.dtype).contiguous()
        y = torch.empty((n, 3), dtype=sim.dtype, device=dev)
        ck = torch.empty((sim.iterations + 1, n, 3), dtype=sim.dtype, device=dev)
        q_out = torch.empty_like(q)
        qd_out = torch.empty_like(qd)
        stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        cdesc = contacts_desc(contacts, sim.model)
        rc = sim._lib.vbd_record_step(sim.solver._h, _p(q), _p(qd), _p(f), None if cdesc is None else C.byref(cdesc),
                                      dt, _p(y), _p(ck), _p(q_out), _p(qd_out), stream)  # fmt: skip
        _lib.check(rc, "vbd_record_step")
        ctx.sim = sim
        ctx.dt = dt
        ctx.contacts = contacts
        ctx.save_for_backward(q, y, ck)
        return q_out, qd_out

    @staticmethod
    def backward(ctx, g_q, g_qd):
        sim = ctx.sim
        q, y, ck = ctx.saved_tensors
        T = sim.model.tri_count
        dev = q.device
        aq = torch.empty_like(q)
        aqd = torch.empty_like(q)
        amu = torch.zeros(T, dtype=sim.dtype, device=dev)
        alam = torch.zeros(T, dtype=sim.dtype, device=dev)
        g_q = None if g_q is None else g_q.to(sim.dtype).contiguous()
        g_qd = None if g_qd is None else g_qd.to(sim.dtype).contiguous()
        stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        cdesc = contacts_desc(ctx.contacts, sim.model)
        rc = sim._lib.vbd_adjoint_step(sim.solver._h, _p(q), _p(y), _p(ck), None if cdesc is None else C.byref(cdesc),
                                       ctx.dt, _p(g_q), _p(g_qd), _p(aq), _p(aqd), _p(amu), _p(alam), stream)  # fmt: skip
        _lib.check(rc, "vbd_adjoint_step")
        return None, aq, aqd, amu, alam, None, None, None


def lame_from_young(E: torch.Tensor, nu: float, thickness: float, area: torch.Tensor | None = None):
    """Plane-stress membrane Lame coefficients times thickness: mu = E h / (2 (1 + nu)),
    lambda = E h nu / (1 - nu^2). (The reference consumes mu, lambda directly in tri_materials.)"""
    mu = E * (thickness / (2.0 * (1.0 + nu)))
    lam = E * (thickness * nu / (1.0 - nu * nu))
    return mu, lam
