"""The precision-stress configuration amplifies rounding in the reference's own arithmetic.

On the stress sheet (per-triangle E log-uniform in [1e5, 1e8] Pa, 0.1 % sliver triangles, 30 iterations,
dt = 1/600 s), two FP64 runs of the oracle whose initial positions differ by 1e-12 m drift apart by orders
of magnitude within a few frames. Position differences between FP32 (or mixed) and FP64 trajectories are
therefore bounded below by this sensitivity, and the meaningful accuracy figure of a precision mode is the
error of one substep from a common state (``bench.py --workload precision`` reports both). Runs on the CPU.
"""

import numpy as np

import bench
from oracle import vbd_oracle as orc
from tests.helpers import oracle_model_dict


def test_fp64_runs_of_the_stress_sheet_diverge_from_a_1e12_perturbation():
    b, _ = bench.build_precision_model(n=24, seed=4, sliver_fraction=1e-3)
    m = b.finalize("cpu")
    om = orc.Model(oracle_model_dict(m))
    q0 = m.particle_q.numpy().astype(np.float64)

    def run(perturb):
        q = q0 + perturb * np.random.default_rng(1).normal(size=q0.shape)
        qd = np.zeros_like(q)
        for _ in range(40):
            _, q, qd = orc.step(om, q, qd, None, None, 1.0 / 600.0, 30, 64, orc.max_threads())
        return q

    a, b2 = run(0.0), run(1e-12)
    spread = np.linalg.norm(a - b2, axis=1).max()
    assert np.all(np.isfinite(a)) and spread > 1e-12 * 1e4, spread
