"""The oracle's self-contact restatement against goldens from the reference's own code.

``tests/golden/make_golden.py`` runs the reference's self-contact functions (pair terms, division
planes, detection kernels, n-ring filters, accumulation and truncation kernels) in float64 through the
Warp stand-in. The FP64 oracle must agree to near machine precision, and its detection must record the
same pairs in the same slots.
"""

import os

import numpy as np
import pytest

from oracle import vbd_oracle as orc

RADIUS, KE, KD, MU, EPS, DT = 0.02, 1.0e4, 1.0e-3, 0.4, 1.0e-2, 1.0 / 600.0


def _load(golden_dir, name):
    return dict(np.load(os.path.join(golden_dir, name)))


def _close(a, b, rel):
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(np.asarray(a) - np.asarray(b)).max() <= rel * scale


def test_barrier_norm(golden_dir):
    for dis, dEdD, d2E in _load(golden_dir, "selfcontact_elements.npz")["norm"]:
        a, b = orc.sc_norm(dis, RADIUS, KE)
        assert abs(a - dEdD) <= 1e-12 * max(abs(dEdD), 1e-30)
        assert abs(b - d2E) <= 1e-12 * max(abs(d2E), 1e-30)


def test_triangle_closest_point(golden_dir):
    for r in _load(golden_dir, "selfcontact_elements.npz")["closest"]:
        x = r[:12].reshape(4, 3)
        c, bary, feat = orc.tri_closest(*x)
        assert feat == int(r[18])
        assert np.abs(c - r[12:15]).max() <= 1e-12
        assert np.abs(bary - r[15:18]).max() <= 1e-12


def test_vertex_triangle_pairs(golden_dir):
    g = _load(golden_dir, "selfcontact_elements.npz")
    rows, closest = g["vt"], g["closest"]
    hits = 0
    for r, c in zip(rows, closest, strict=True):
        X, Xa, hit_ref = r[:12], r[12:24], bool(r[24])
        dist = np.linalg.norm(X[9:12] - c[12:15])
        f_ref, H_ref = r[25:37].reshape(4, 3), r[37:73].reshape(4, 3, 3)
        hit, f, H = orc.sc_pair("vt", 64, X, Xa, RADIUS, KE, KD, MU, EPS, DT)
        assert hit == hit_ref
        hits += hit
        if hit:
            assert _close(f, f_ref, 1e-10) and _close(H, H_ref, 1e-10)
            if dist > 1e-3:  # below that, FP32 rounding of the positions is a visible part of the distance
                _, f32, H32 = orc.sc_pair("vt", 32, X, Xa, RADIUS, KE, KD, MU, EPS, DT)
                assert _close(f32, f_ref, 2e-3) and _close(H32, H_ref, 2e-3)
    assert 0 < hits < len(rows)


def test_edge_edge_pairs(golden_dir):
    rows = _load(golden_dir, "selfcontact_elements.npz")["ee"]
    hits = 0
    for r in rows:
        X, Xa, hit_ref = r[:12], r[12:24], bool(r[24])
        f_ref = np.stack([r[25:28], r[28:31]])
        H_ref = np.stack([r[31:40].reshape(3, 3), r[40:49].reshape(3, 3)])
        st = orc.edge_closest(*X.reshape(4, 3), 1e-5)
        assert np.abs(st - r[49:52]).max() <= 1e-12
        hit, f, H = orc.sc_pair("ee", 64, X, Xa, RADIUS, KE, KD, MU, EPS, DT, 1e-5)
        assert hit == hit_ref
        hits += hit
        if hit:
            assert _close(f, f_ref, 1e-10) and _close(H, H_ref, 1e-10)
    assert 0 < hits < len(rows)


@pytest.mark.parametrize("kind", ["vt", "ee"])
def test_division_planes(golden_dir, kind):
    rows = _load(golden_dir, "selfcontact_elements.npz")[f"{kind}_plane"]
    cut = 0
    for r in rows:
        X, dX = r[:12], r[12:24]
        dummy_ref, n_ref, d_ref, t_ref = r[24:28] != 0.0, r[28:31], r[31:34], r[34:38]
        if kind == "vt":  # stored as (a, b, c, p); the plane routine takes (v, t1, t2, t3)
            X = X.reshape(4, 3)[[3, 0, 1, 2]].ravel()
            dX = dX.reshape(4, 3)[[3, 0, 1, 2]].ravel()
        dummy, n, d, t = orc.sc_plane(kind, 64, X, dX)
        np.testing.assert_array_equal(dummy, dummy_ref)
        # a normal from a short closest-point vector carries its rounding, relatively enlarged
        assert np.abs(n - n_ref).max() <= 1e-9 and np.abs(d - d_ref).max() <= 1e-9
        assert np.abs(t - t_ref).max() <= 1e-8
        cut += int(np.sum(~dummy & (t < 1.0)))
    assert cut > 0


SCENES = ["step_selfcontact_layers.npz", "step_selfcontact_fold.npz"]


def _scene(g):
    m = {k[len("model_"):]: v for k, v in g.items() if k.startswith("model_")}
    for k in ("adj_face_offsets", "adj_faces", "adj_edge_offsets", "adj_edges", "particle_colors", "color_offsets",
              "color_particles", "gravity", "soft", "shapes", "beta", "friction_epsilon"):
        m[k] = g[k]
    vt = (g["sc_vt_filter"], g["sc_vt_filter_offsets"]) if "sc_vt_filter" in g else None
    ee = (g["sc_ee_filter"], g["sc_ee_filter_offsets"]) if "sc_ee_filter" in g else None
    sc = orc.SelfContact(
        g["model_particle_q"], radius=float(g["sc_radius"]), margin=float(g["sc_margin"]),
        relaxation=float(g["sc_relaxation"]), interval=int(g["sc_interval"]),
        rest_exclusion=float(g.get("sc_rest_exclusion", 0.0)), vt_filter=vt, ee_filter=ee,
    )  # fmt: skip
    return orc.Model(m), sc


@pytest.mark.parametrize("name", SCENES)
def test_detection_matches_reference_kernels(golden_dir, name):
    g = _load(golden_dir, name)
    model, sc = _scene(g)
    for s in range(int(g["substeps"])):
        got = orc.collide(model, sc, g[f"s{s}_q_in"], 64)
        for k in ("vt", "vt_count", "ee", "ee_count", "resize_flags"):
            np.testing.assert_array_equal(got[k], g[f"s{s}_cd0_{k}"], err_msg=f"{name} substep {s} {k}")
        assert np.abs(got["vt_min"] - g[f"s{s}_cd0_vt_min"]).max() <= 1e-12
        assert np.abs(got["ee_min"] - g[f"s{s}_cd0_ee_min"]).max() <= 1e-12
        assert got["vt_count"].sum() > 0 and got["ee_count"].sum() > 0


@pytest.mark.parametrize("name", SCENES)
def test_selfcontact_step_fp64(golden_dir, name):
    g = _load(golden_dir, name)
    model, sc = _scene(g)
    for s in range(int(g["substeps"])):
        q_after, q_out, qd_out = orc.step(
            model, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], None, float(g["dt"]), int(g["iterations"]), 64,
            self_contact=sc,
        )  # fmt: skip
        assert np.abs(q_out - g[f"s{s}_q_out"]).max() <= 1e-10, (name, s)
        assert np.abs(q_after - g[f"s{s}_q_in_after"]).max() <= 1e-10
        assert np.abs(qd_out - g[f"s{s}_qd_out"]).max() <= 1e-10 / float(g["dt"])


@pytest.mark.parametrize("name", SCENES)
def test_selfcontact_step_fp32(golden_dir, name):
    g = _load(golden_dir, name)
    model, sc = _scene(g)
    for s in range(int(g["substeps"])):
        _, q_out, _ = orc.step(
            model, g[f"s{s}_q_in"], g[f"s{s}_qd_in"], g[f"s{s}_f_ext"], None, float(g["dt"]), int(g["iterations"]), 32,
            self_contact=sc,
        )  # fmt: skip
        assert np.abs(q_out - g[f"s{s}_q_out"]).max() <= 1e-4, (name, s)


def test_box_grid_detection_equals_brute_force(golden_dir):
    """The oracle's box-grid candidate search gives exactly the brute-force buffers, overflow included."""
    g = _load(golden_dir, "step_selfcontact_fold.npz")
    model, _ = _scene(g)
    rng = np.random.default_rng(1)
    q = g["s0_q_in"] + rng.normal(scale=4e-3, size=g["s0_q_in"].shape)  # denser contacts
    for vb, eb in ((32, 64), (2, 3)):
        kw = dict(radius=0.012, margin=0.03, vertex_buffer=vb, edge_buffer=eb, rest_exclusion=0.02,
                  vt_filter=(g["sc_vt_filter"], g["sc_vt_filter_offsets"]),
                  ee_filter=(g["sc_ee_filter"], g["sc_ee_filter_offsets"]))  # fmt: skip
        a = orc.collide(model, orc.SelfContact(g["model_particle_q"], **kw), q, 64)
        b = orc.collide(model, orc.SelfContact(g["model_particle_q"], brute_force=True, **kw), q, 64)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        assert a["vt_count"].sum() > 0 and a["ee_count"].sum() > 0
        assert (a["resize_flags"][0] == 1) == (vb == 2)
