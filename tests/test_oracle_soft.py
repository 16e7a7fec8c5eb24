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
