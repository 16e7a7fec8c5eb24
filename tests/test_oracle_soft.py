"""Oracle springs and tetrahedra against goldens from the reference's own code (float64).

``tests/golden/make_golden.py`` runs ``evaluate_volumetric_neo_hookean_force_and_hessian`` with the reference's
9x9 assembly, ``evaluate_spring_force_and_hessian_both_vertices``, the spring accumulation kernel and
``solve_elasticity``'s tetrahedron loop on a falling tetrahedral block hung by springs; the FP64 oracle
(closed-form vertex blocks) must agree to near machine precision.
"""

import os

import numpy as np
import pytest

from oracle import vbd_oracle as orc


def _load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, name)))


def test_tetrahedron_elements(golden_dir):
    for r in _load(golden_dir, "soft_elements.npz")["tet"]:
        X, Xp, Dinv = r[:12], r[12:24], r[24:33]
        mu, lam, damping, dt, order = r[33:38]
        f_ref, H_ref = r[38:41], r[41:50].reshape(3, 3)
        f, H = orc.tet_element(64, order, X, Xp, Dinv, mu, lam, damping, dt)
        scale = max(np.abs(f_ref).max(), np.abs(H_ref).max(), 1e-30)
        assert np.abs(f - f_ref).max() <= 1e-10 * scale and np.abs(H - H_ref).max() <= 1e-10 * scale
        f32, H32 = orc.tet_element(32, order, X, Xp, Dinv, mu, lam, damping, dt)
        assert np.abs(f32 - f_ref).max() <= 2e-3 * scale and np.abs(H32 - H_ref).max() <= 2e-3 * scale


def test_spring_elements(golden_dir):
    for r in _load(golden_dir, "soft_elements.npz")["spring"]:
        X, Xa = r[:6], r[6:12]
        rest, ke, kd, dt = r[12:16]
        f0, f1, H = orc.spring_element(64, X, Xa, rest, ke, kd, dt)
        scale = max(np.abs(r[16:22]).max(), np.abs(r[22:31]).max(), 1e-30)
        assert np.abs(f0 - r[16:19]).max() <= 1e-12 * scale and np.abs(f1 - r[19:22]).max() <= 1e-12 * scale
        assert np.abs(H - r[22:31].reshape(3, 3)).max() <= 1e-12 * scale


def _model(g):
    m = {k[len("model_"):]: v for k, v in g.items() if k.startswith("model_")}
    for k in ("adj_face_offsets", "adj_faces", "adj_edge_offsets", "adj_edges", "adj_tet_offsets", "adj_tets",
              "particle_colors", "color_offsets", "color_particles", "gravity", "soft", "shapes", "beta",
              "friction_epsilon"):  # fmt: skip
        m[k] = g[k]
    return m


def test_tet_adjacency_matches_reference_fill_order(golden_dir):
    g = _load(golden_dir, "step_soft_block.npz")
    to, ta = orc.build_tet_adjacency(len(g["model_particle_mass"]), g["model_tet_indices"])
    np.testing.assert_array_equal(to, g["adj_tet_offsets"])
    np.testing.assert_array_equal(ta, g["adj_tets"])


@pytest.mark.parametrize("precision,tol", [(64, 1e-10), (32, 1e-4)])
def test_soft_block_step(golden_dir, precision, tol):
    g = _load(golden_dir, "step_soft_block.npz")
    model = orc.Model(_model(g))
    for s in range(int(g["substeps"])):
        c = orc.make_contacts(g[f"s{s}_contact_count"], g[f"s{s}_contact_particle"], g[f"s{s}_contact_shape"],
                              g[f"s{s}_contact_body_pos"], g[f"s{s}_contact_body_vel"], g[f"s{s}_contact_normal"])  # fmt: skip
        _, q_out, qd_out = orc.step(model, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], c, float(g["dt"]),
                                    int(g["iterations"]), precision)  # fmt: skip
        assert np.abs(q_out - g[f"s{s}_q_out"]).max() <= tol, (s, np.abs(q_out - g[f"s{s}_q_out"]).max())


def _nh_energy(x, Dinv, mu, lam):
    """Stable Neo-Hookean energy of one tetrahedron with the reference's Lame shift (lambda_nh = lambda + mu,
    alpha = 1 + mu / lambda_nh): V (mu / 2 (tr F^T F - 3) + lambda_nh / 2 (det F - alpha)^2), whose gradient is
    the first Piola stress mu F + lambda_nh (det F - alpha) cof F that the element code assembles."""
    D = Dinv.reshape(3, 3)
    V = 1.0 / (np.linalg.det(D) * 6.0)
    F = np.stack([x[1] - x[0], x[2] - x[0], x[3] - x[0]], axis=1) @ D
    lnh = lam + mu
    alpha = 1.0 + mu / lnh
    return V * (0.5 * mu * (np.sum(F * F) - 3.0) + 0.5 * lnh * (np.linalg.det(F) - alpha) ** 2)


def test_tetrahedron_force_is_the_energy_gradient():
    """The finite-difference pattern of the reference's test_tet_energy (test_softbody.py:378-470): the force on
    each vertex equals minus the derivative of the element energy (central differences, FP64), and the vertex
    Hessian block is symmetric positive semi-definite."""
    rng = np.random.default_rng(42)
    for _ in range(30):
        rest = rng.standard_normal((4, 3))
        if np.linalg.det((rest[1:] - rest[0]).T) < 0:
            rest[[0, 1]] = rest[[1, 0]]
        Dinv = np.linalg.inv((rest[1:] - rest[0]).T)
        mu, lam = abs(rng.standard_normal()) + 0.1, abs(rng.standard_normal()) + 0.1
        x = rest + 0.3 * rng.standard_normal((4, 3))
        for order in range(4):
            f, H = orc.tet_element(64, order, x.reshape(-1), x.reshape(-1), Dinv.reshape(-1), mu, lam, 0.0, 1e-3)
            g = np.zeros(3)
            h = 1e-6
            for k in range(3):
                xp, xm = x.copy(), x.copy()
                xp[order, k] += h
                xm[order, k] -= h
                g[k] = (_nh_energy(xp, Dinv, mu, lam) - _nh_energy(xm, Dinv, mu, lam)) / (2 * h)
            assert np.abs(f + g).max() <= 1e-6 * max(1.0, np.abs(g).max())
            H = np.asarray(H).reshape(3, 3)
            assert np.abs(H - H.T).max() <= 1e-12 * max(1.0, np.abs(H).max())
            assert np.linalg.eigvalsh(0.5 * (H + H.T)).min() >= -1e-9 * max(1.0, np.abs(H).max())


def test_spring_force_is_the_energy_gradient():
    rng = np.random.default_rng(7)
    for _ in range(30):
        x = rng.standard_normal((2, 3))
        rest, ke = abs(rng.standard_normal()) + 0.1, abs(rng.standard_normal()) * 100.0 + 1.0
        f0, f1, _ = orc.spring_element(64, x.reshape(-1), x.reshape(-1), rest, ke, 0.0, 1e-3)

        def energy(y):
            return 0.5 * ke * (np.linalg.norm(y[0] - y[1]) - rest) ** 2

        for end, f in ((0, f0), (1, f1)):
            g = np.zeros(3)
            for k in range(3):
                yp, ym = x.copy(), x.copy()
                yp[end, k] += 1e-6
                ym[end, k] -= 1e-6
                g[k] = (energy(yp) - energy(ym)) / 2e-6
            assert np.abs(np.asarray(f) + g).max() <= 1e-6 * max(1.0, np.abs(g).max())
