"""Particle-shape contact generation against analytic shapes: the oracle restatement against goldens computed by
the reference's own SDF functions (``sdf_box``, ``sdf_capsule``, ``sdf_cylinder``, ``sdf_ellipsoid``, ``sdf_sphere``,
``sdf_plane`` and their gradients, run through ``tests/golden/warp_shim.py``) with the frame handling of
``create_soft_contacts``; and the builder's shape table in the reference's GeoType, transform and scale layout."""

import numpy as np

from newton_chysx_b200 import sim
from oracle import vbd_oracle as orc
from tests.helpers import load_golden


def test_oracle_shape_contacts_match_reference_sdfs():
    g = load_golden("soft_contact_shapes.npz")
    cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(g["q"], g["radius"], g["flags"], g["shape_type"],
                                                     g["shape_transform"], g["shape_scale"], float(g["margin"]))  # fmt: skip
    assert cnt == len(g["particle"]) and cnt > 1000
    np.testing.assert_array_equal(p[:cnt], g["particle"])
    np.testing.assert_array_equal(s[:cnt], g["shape"])
    assert np.abs(bp[:cnt] - g["body_pos"]).max() <= 1e-12
    assert np.abs(nn[:cnt] - g["normal"]).max() <= 1e-12
    assert np.abs(bv[:cnt]).max() == 0.0
    # every analytic type contributes contacts
    assert set(np.unique(g["shape"])) == set(range(len(g["shape_type"])))


def test_builder_shape_table():
    b = sim.ModelBuilder(up_axis="Z")
    b.add_ground_plane()
    b.add_shape_sphere(xform=((0.5, 0.0, 0.3), sim.quat_identity()), radius=0.25)
    q = sim.quat_from_axis_angle((0.0, 1.0, 0.0), 0.5)
    b.add_shape_box(xform=((-0.4, -0.4, 0.3), q), hx=0.3, hy=0.2, hz=0.1)
    b.add_shape_capsule(xform=(0.2, 0.6, 0.35) + tuple(q), radius=0.1, half_height=0.2)
    b.add_shape_cylinder(radius=0.15, half_height=0.1)
    b.add_shape_ellipsoid(rx=0.3, ry=0.2, rz=0.15)
    b.add_shape_plane(plane=(0.0, 1.0, 0.0, -0.5), width=2.0, length=1.0)
    b.add_particle((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 1.0)
    m = b.finalize("cpu")
    assert list(m.shape_type) == [1, 3, 7, 4, 6, 5, 1]
    np.testing.assert_allclose(m.shape_transform[0], [0, 0, 0, 0, 0, 0, 1])
    np.testing.assert_allclose(m.shape_scale[2], [0.3, 0.2, 0.1])
    np.testing.assert_allclose(m.shape_transform[3, 3:], q, rtol=1e-6)
    # the plane y = 0.5 with normal +Y: its local +Z maps to +Y, its origin to (0, 0.5, 0)
    np.testing.assert_allclose(m.shape_transform[6, :3], [0.0, 0.5, 0.0], atol=1e-7)
    np.testing.assert_allclose(sim.quat_to_matrix(m.shape_transform[6, 3:]) @ [0, 0, 1], [0, 1, 0], atol=1e-6)
    np.testing.assert_allclose(m.shape_scale[6], [2.0, 1.0, 0.0])
    yb = sim.ModelBuilder(up_axis="Y")
    yb.add_ground_plane(height=0.1)
    yb.add_particle((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 1.0)
    ym = yb.finalize("cpu")
    np.testing.assert_allclose(sim.quat_to_matrix(ym.shape_transform[0, 3:]) @ [0, 0, 1], [0, 1, 0], atol=1e-6)
    np.testing.assert_allclose(ym.shape_transform[0, :3], [0.0, 0.1, 0.0], atol=1e-7)
