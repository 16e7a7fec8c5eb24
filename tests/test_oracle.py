"""The CPU oracle against golden vectors produced by the reference's own kernel code.

``tests/golden/make_golden.py`` executes the reference's ``@wp.func``/``@wp.kernel`` bodies in
float64; the oracle's FP64 mode must agree to near machine precision (these are identical
formulas), and its FP32 mode to FP32 rounding.
"""

import os

import numpy as np
import pytest

from oracle import vbd_oracle as orc
from tests.helpers import golden_body_contacts_kw


def _load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, name)))


def test_membrane_elements(golden_dir):
    rows = _load(golden_dir, "elements.npz")["membrane"]
    for r in rows:
        X, Xp, pose = r[0:9], r[9:18], r[18:22]
        area, mu, lam, damping, dt, order = r[22:28]
        f_ref, H_ref = r[28:31], r[31:40].reshape(3, 3)
        f, H = orc.element("membrane", 64, order, X, Xp, pose, area, mu, lam, damping, dt)
        scale = max(np.abs(f_ref).max(), np.abs(H_ref).max(), 1e-30)
        assert np.abs(f - f_ref).max() <= 1e-11 * scale
        assert np.abs(H - H_ref).max() <= 1e-11 * scale
        f32, H32 = orc.element("membrane", 32, order, X, Xp, pose, area, mu, lam, damping, dt)
        assert np.abs(f32 - f_ref).max() <= 2e-4 * scale
        assert np.abs(H32 - H_ref).max() <= 2e-4 * scale


def test_bending_elements(golden_dir):
    rows = _load(golden_dir, "elements.npz")["bending"]
    boundaries = 0
    for r in rows:
        X, Xp = r[0:12], r[12:24]
        rest_angle, rest_len, ke, kd, dt, order, boundary = r[24:31]
        f_ref, H_ref = r[31:34], r[34:43].reshape(3, 3)
        boundaries += int(boundary)
        f, H = orc.element("bending", 64, order, X, Xp, boundary, rest_angle, rest_len, ke, kd, dt)
        scale = max(np.abs(f_ref).max(), np.abs(H_ref).max(), 1e-30)
        assert np.abs(f - f_ref).max() <= 1e-10 * scale
        assert np.abs(H - H_ref).max() <= 1e-10 * scale
    assert boundaries > 0


def test_contact_elements(golden_dir):
    rows = _load(golden_dir, "elements.npz")["contact"]
    for r in rows:
        pen, n, rel = r[0], r[1:4], r[4:7]
        ke, kd, mu, eps, dt = r[7:12]
        f_ref, H_ref = r[12:15], r[15:24].reshape(3, 3)
        f, H = orc.element("contact", 64, pen, n, rel, ke, kd, mu, eps, dt)
        scale = max(np.abs(f_ref).max(), np.abs(H_ref).max(), 1e-30)
        assert np.abs(f - f_ref).max() <= 1e-11 * scale
        assert np.abs(H - H_ref).max() <= 1e-11 * scale


def _model_from_golden(g):
    m = {k[len("model_"):]: v for k, v in g.items() if k.startswith("model_")}
    for k in ("adj_face_offsets", "adj_faces", "adj_edge_offsets", "adj_edges", "particle_colors", "color_offsets",
              "color_particles", "gravity", "soft", "shapes", "beta", "friction_epsilon"):
        m[k] = g[k]
    return m


STEP_FIXTURES = ["step_grid_ground.npz", "step_grid_sphere.npz", "step_complex_rest_angle.npz", "step_grid_bodies.npz"]


@pytest.mark.parametrize("name", STEP_FIXTURES)
def test_adjacency_matches_reference_fill_order(golden_dir, name):
    g = _load(golden_dir, name)
    n = len(g["model_particle_mass"])
    fo, fa, eo, ea = orc.build_adjacency(n, g["model_tri_indices"], g["model_edge_indices"])
    np.testing.assert_array_equal(fo, g["adj_face_offsets"])
    np.testing.assert_array_equal(fa, g["adj_faces"])
    np.testing.assert_array_equal(eo, g["adj_edge_offsets"])
    np.testing.assert_array_equal(ea, g["adj_edges"])


@pytest.mark.parametrize("name", STEP_FIXTURES)
@pytest.mark.parametrize("precision,tol", [(64, 1e-10), (32, 1e-4)])
def test_step_matches_reference(golden_dir, name, precision, tol):
    g = _load(golden_dir, name)
    model = orc.Model(_model_from_golden(g))
    for s in range(int(g["substeps"])):
        contacts = orc.make_contacts(
            g[f"s{s}_contact_count"], g[f"s{s}_contact_particle"], g[f"s{s}_contact_shape"],
            g[f"s{s}_contact_body_pos"], g[f"s{s}_contact_body_vel"], g[f"s{s}_contact_normal"],
            **golden_body_contacts_kw(g, s),
        )  # fmt: skip
        q_after, q_out, qd_out = orc.step(
            model, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], contacts, float(g["dt"]),
            int(g["iterations"]), precision=precision,
        )  # fmt: skip
        # positions in metres: absolute tolerance; velocity tolerance scaled by 1/dt
        assert np.abs(q_out - g[f"s{s}_q_out"]).max() <= tol
        assert np.abs(q_after - g[f"s{s}_q_in_after"]).max() <= tol
        assert np.abs(qd_out - g[f"s{s}_qd_out"]).max() <= tol / float(g["dt"])
