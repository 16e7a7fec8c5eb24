"""Launch-shape autotuner for ``SolverVBD``.

Times a few substeps of each candidate configuration on the caller's model (or a representative
subset of it) and returns the fastest as ``SolverVBD`` keyword arguments. The candidates cover what
changes the speed of the sweep on a B200:

* the element layout: ``ell16`` / ``ell`` (per-incidence stencil records with 16-bit or 32-bit vertex
  ids, one lane per vertex) or ``csr`` (adjacency + element records) with 1, 2 or 4 lanes per vertex;
* the persistent kernel's register budget (``min_blocks_per_sm``: 2, 3, 4 CTAs of 256 threads per SM,
  or the compiler's choice), whether an instance's positions live in shared memory, and whether the ell16
  kernel pairs two vertices per thread in paired FP32 instructions (``pair_vertices``), and whether the csr
  kernel gives each warp its own instance (``instance_per_warp``);
* the block size of the per-color schedule.

Each candidate is a separate solver on the same model; results do not depend on the choice beyond
FP32 rounding (``tests/test_gpu_scenarios.py::test_schedules_and_lane_counts_agree``).
"""

from __future__ import annotations

import itertools

import torch

from .sim import CollisionPipeline, Model
from .solver_vbd import SolverVBD


def candidates(model: Model, schedule: str):
    if schedule == "persistent":
        out = []
        for layout in ("ell16", "ell"):
            for occ in (0, 2, 3, 4):
                out.append(dict(layout=layout, lanes_per_vertex=1, positions_in_shared="off", min_blocks_per_sm=occ))
                if layout == "ell16":
                    out.append(dict(layout=layout, lanes_per_vertex=1, positions_in_shared="off", min_blocks_per_sm=occ,
                                    pair_vertices=True))  # fmt: skip
            out.append(dict(layout=layout, lanes_per_vertex=1, positions_in_shared="on"))
        for lanes, shared in itertools.product((1, 2, 4), ("off", "on")):
            out.append(dict(layout="csr", lanes_per_vertex=lanes, positions_in_shared=shared))
        for lanes in (2, 4, 8):
            out.append(dict(layout="csr", lanes_per_vertex=lanes, instance_per_warp=True))
        return out
    out = []
    for block in (64, 128, 256):
        out.append(dict(layout="ell", lanes_per_vertex=1, block_size=block))
        for lanes in (2, 4, 8):
            out.append(dict(layout="csr", lanes_per_vertex=lanes, block_size=block))
    return out


def tune(model: Model, schedule: str = "persistent", iterations: int = 10, dt: float = 1.0 / 600.0, substeps: int = 3,
         contact_margin: float | None = 0.01, verbose: bool = False, **solver_kwargs) -> dict:  # fmt: skip
    """Returns the fastest candidate's keyword arguments (plus ``schedule``) for this model."""
    pipe = CollisionPipeline(model, soft_contact_margin=contact_margin) if contact_margin is not None else None
    contacts = pipe.contacts() if pipe else None
    best, best_ms = None, float("inf")
    for cand in candidates(model, schedule):
        try:
            solver = SolverVBD(model, iterations=iterations, schedule=schedule, **cand, **solver_kwargs)
        except Exception:  # a shape this device cannot run (e.g. shared memory too small)
            continue
        s0, s1 = model.state(), model.state()
        for k in range(2):  # warm-up
            if pipe:
                pipe.collide(s0, contacts)
            solver.step(s0, s1, None, contacts, dt)
            s0, s1 = s1, s0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = 0.0
        for _ in range(substeps):
            if pipe:
                pipe.collide(s0, contacts)
            e0.record()
            solver.step(s0, s1, None, contacts, dt)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            s0, s1 = s1, s0
        if verbose:
            print(f"  {cand}: {ms / substeps:.3f} ms")
        if ms < best_ms:
            best, best_ms = cand, ms
        del solver
    if best is None:
        raise RuntimeError("no candidate configuration could run")
    return dict(best, schedule=schedule)
