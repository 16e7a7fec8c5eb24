"""Differentiable VBD substeps: the hand-written adjoint of the C ABI behind ``torch.autograd``.

``vbd_step`` has a hand-written reverse, ``vbd_adjoint_step``. Its forward pass ``vbd_record_step``
keeps the positions at the start of every iteration (per-iteration checkpoints). The reverse pass
recomputes the per-color states of one iteration from its checkpoint and walks the colors backwards.
Gradients flow to the input positions and velocities and to the triangles' Lame coefficients
(``Model.tri_materials[:, 0:2]``), hence to anything they are computed from, e.g. per-triangle
Young's moduli.

The reference VBD has no gradient: its kernels are built with ``enable_backward=False``
(``newton/_src/solvers/vbd/particle_vbd_kernels.py:27-28``). The check is against central finite
differences of the forward step (``tests/test_gpu_adjoint.py``, ``bench.py --workload adjoint``).
Particle-shape contacts are not differentiated.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .sim import Model
from .solver_vbd import SolverVBD


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

    def substep(self, q, qd, tri_mu, tri_lambda, dt, particle_f=None):
        return _Substep.apply(self, q, qd, tri_mu, tri_lambda, float(dt), particle_f)

    def rollout(self, q0, qd0, tri_mu, tri_lambda, dt, substeps, particle_f=None):
        """``substeps`` differentiable substeps from (q0, qd0); returns the final (q, qd)."""
        self.set_materials(tri_mu, tri_lambda)
        q, qd = q0, qd0
        for _ in range(substeps):
            q, qd = _Substep.apply(self, q, qd, tri_mu, tri_lambda, float(dt), particle_f)
        return q, qd


class _Substep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sim: DifferentiableVBD, q, qd, tri_mu, tri_lambda, dt, particle_f):
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
        rc = sim._lib.vbd_record_step(sim.solver._h, _p(q), _p(qd), _p(f), dt, _p(y), _p(ck), _p(q_out), _p(qd_out),
                                      stream)  # fmt: skip
        _lib.check(rc, "vbd_record_step")
        ctx.sim = sim
        ctx.dt = dt
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
        rc = sim._lib.vbd_adjoint_step(sim.solver._h, _p(q), _p(y), _p(ck), ctx.dt, _p(g_q), _p(g_qd), _p(aq), _p(aqd),
                                       _p(amu), _p(alam), stream)  # fmt: skip
        _lib.check(rc, "vbd_adjoint_step")
        return None, aq, aqd, amu, alam, None, None


def lame_from_young(E: torch.Tensor, nu: float, thickness: float, area: torch.Tensor | None = None):
    """Plane-stress membrane Lame coefficients times thickness: mu = E h / (2 (1 + nu)),
    lambda = E h nu / (1 - nu^2). (The reference consumes mu, lambda directly in tri_materials.)"""
    mu = E * (thickness / (2.0 * (1.0 + nu)))
    lam = E * (thickness * nu / (1.0 - nu * nu))
    return mu, lam
