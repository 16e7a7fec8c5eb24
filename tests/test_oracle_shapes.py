"""Particle-shape contact generation against analytic shapes: the oracle restatement against goldens computed by
the reference's own SDF functions (``sdf_box``, ``sdf_capsule``, ``sdf_cylinder``, ``sdf_ellipsoid``, ``sdf_sphere``,
``sdf_plane`` and their gradients, run through ``tests/golden/warp_shim.py``) with the frame handling of
``create_soft_contacts``; and the builder's shape table in the reference's GeoType, transform and scale layout."""

import numpy as np
import pytest

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


def test_oracle_cone_and_heightfield_contacts_match_reference():
    """Cones (``sdf_cone``/``sdf_cone_grad``) and heightfields (``sample_sdf_grad_heightfield``, one of them
    scaled with a negative Y scale, one a single row that gives no contacts) against goldens from the reference's
    own functions."""
    g = load_golden("soft_contact_cone_hfield.npz")
    cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(
        g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"], g["shape_scale"], float(g["margin"]),
        heightfield_index=g["shape_heightfield_index"], heightfields=g["heightfields"], elevations=g["elevations"])
    assert cnt == len(g["particle"]) and cnt > 1000
    np.testing.assert_array_equal(p[:cnt], g["particle"])
    np.testing.assert_array_equal(s[:cnt], g["shape"])
    assert np.abs(bp[:cnt] - g["body_pos"]).max() <= 1e-12
    assert np.abs(nn[:cnt] - g["normal"]).max() <= 1e-12
    assert np.abs(bv[:cnt]).max() == 0.0
    assert set(np.unique(g["shape"])) == {0, 1, 2, 3, 4}


def test_builder_cone_and_heightfield_table():
    """Cones store (radius, half height, 0); heightfields are packed as the reference's finalize packs them: extents
    times |scale| in X and Y, min_z and max_z times the Z scale, normalized elevations concatenated."""
    b = sim.ModelBuilder(up_axis="Z")
    b.add_shape_cone(xform=((0.1, 0.2, 0.3), sim.quat_identity()), radius=0.4, half_height=0.25)
    raw = np.arange(12, dtype=np.float32).reshape(3, 4) ** 2
    hf = sim.Heightfield(raw, 3, 4, hx=0.5, hy=0.25)
    assert hf.min_z == 0.0 and hf.max_z == 121.0 and hf.data.max() == 1.0 and hf.data.min() == 0.0
    b.add_shape_heightfield(heightfield=hf, scale=(2.0, -1.0, 0.5))
    b.add_shape_heightfield(heightfield=sim.Heightfield(np.ones((2, 2)), 2, 2, min_z=-1.0, max_z=1.0))
    b.add_particle((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 1.0)
    m = b.finalize("cpu")
    assert list(m.shape_type) == [9, 2, 2]
    np.testing.assert_allclose(m.shape_scale[0], [0.4, 0.25, 0.0])
    assert list(m.shape_heightfield_index) == [-1, 0, 1]
    np.testing.assert_allclose(m.heightfield_data[0], [0, 3, 4, 1.0, 0.25, 0.0, 60.5])
    np.testing.assert_allclose(m.heightfield_data[1], [12, 2, 2, 1.0, 1.0, -1.0, 1.0])
    np.testing.assert_allclose(m.heightfield_elevations.numpy()[:12], raw.reshape(-1) / 121.0, rtol=1e-6)
    assert m.heightfield_elevations.numel() == 16 and float(m.heightfield_elevations[12:].abs().sum()) == 0.0
    with pytest.raises(ValueError):
        sim.Heightfield(np.zeros((1, 3)), 1, 3)


def test_oracle_box_mesh_matches_reference_box_sdf():
    """A closed box mesh through the mesh query (closest point + pseudo-normal sign) gives the reference's own
    ``sdf_box``/``sdf_box_grad`` contacts: outside, the closest point of a box is the clamped point; inside, the
    nearest face. The mesh carries half the box's extents at scale 2, so the scaled path is exercised. A mesh
    query only searches margin + radius / min|scale| around the surface (in the mesh's unscaled frame), so particles
    deeper inside than that have no mesh contact, as in the reference; the comparison covers the rest."""
    from tests.helpers import box_mesh

    g = load_golden("soft_contact_shapes.npz")
    s = int(np.flatnonzero(g["shape_type"] == 7)[0])
    v, tris = box_mesh(*(0.5 * g["shape_scale"][s]))
    cnt, p, _, bp, bv, nn = orc.soft_contacts_shapes(
        g["q"], g["radius"], g["flags"], np.array([8]), g["shape_transform"][s:s + 1], np.array([[2.0, 2.0, 2.0]]),
        float(g["margin"]), mesh_index=[0], meshes=[(v, tris)])  # fmt: skip
    reach = 2.0 * (float(g["margin"]) + g["radius"][g["particle"]] / 2.0)
    sel = (g["shape"] == s) & (g["distance"] > -reach)
    assert cnt == sel.sum() and cnt > 100 and ((g["shape"] == s) & ~sel).sum() > 0
    np.testing.assert_array_equal(p[:cnt], g["particle"][sel])
    assert np.abs(bp[:cnt] - g["body_pos"][sel]).max() <= 1e-12
    assert np.abs(nn[:cnt] - g["normal"][sel]).max() <= 1e-12
    assert np.abs(bv[:cnt]).max() == 0.0


def test_oracle_mesh_sign_and_distance():
    """Icosphere: distances within the tessellation error of the sphere's, inside negative. Torus (non-convex):
    points in the tube are inside, points in the hole and outside are outside."""
    from tests.helpers import icosphere, torus_mesh

    rng = np.random.default_rng(2)
    v, f = icosphere(0.5, 3)
    q = rng.normal(size=(400, 3))
    q *= (rng.uniform(0.3, 0.7, 400) / np.linalg.norm(q, axis=1))[:, None]
    ident = np.array([[0, 0, 0, 0, 0, 0, 1.0]])
    cnt, p, _, bp, _, nn = orc.soft_contacts_shapes(q, np.zeros(400), np.ones(400, np.int32), np.array([8]), ident,
                                                    np.ones((1, 3)), 1.0, mesh_index=[0], meshes=[(v, f)])  # fmt: skip
    assert cnt == 400
    d = np.einsum("ij,ij->i", q[p[:cnt]] - bp[:cnt], nn[:cnt])
    exact = np.linalg.norm(q[p[:cnt]], axis=1) - 0.5
    far = np.abs(exact) > 0.003  # the facets lie up to ~2.3 mm inside the sphere at this tessellation
    assert np.abs(d - exact).max() < 0.003 and ((d < 0) == (exact < 0))[far].all() and far.sum() > 300
    v, f = torus_mesh(0.3, 0.1)
    pts = np.array([[0.3, 0.0, 0.0], [0.0, -0.32, 0.02], [0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [0.3, 0.0, 0.15]])
    cnt, p, _, bp, _, nn = orc.soft_contacts_shapes(pts, np.zeros(5), np.ones(5, np.int32), np.array([8]), ident,
                                                    np.ones((1, 3)), 1.0, mesh_index=[0], meshes=[(v, f)])  # fmt: skip
    assert cnt == 5
    d = np.einsum("ij,ij->i", pts[p[:cnt]] - bp[:cnt], nn[:cnt])
    assert (d[:2] < 0).all() and (d[2:] > 0).all()
    np.testing.assert_allclose(d[[0, 2, 3, 4]], [-0.1, 0.2, 0.1, 0.05], atol=0.01)


def _world_scene(device):
    """Three worlds with a sphere each at the same place (the third's sphere does not collide with particles) and a
    global ground plane; particles of every world spread over the spheres."""
    rng = np.random.default_rng(9)
    top = sim.ModelBuilder(up_axis="Z")
    for w in range(3):
        b = sim.ModelBuilder(up_axis="Z")
        pts = np.stack([rng.uniform(-0.4, 0.4, 3000), rng.uniform(-0.4, 0.4, 3000), rng.uniform(-0.02, 0.5, 3000)], 1)
        b.add_particles(pts, (0.0, 0.0, 0.0), 1.0, radius=0.01)
        cfg = sim.ShapeConfig(has_particle_collision=(w != 2))
        b.add_shape_sphere(xform=((0.0, 0.0, 0.2), sim.quat_identity()), radius=0.2, cfg=cfg)
        top.add_world(b)
    top.add_ground_plane()
    return top.finalize(device)


def test_shape_worlds_and_particle_collision_flag():
    """create_soft_contacts' filters (geometry/kernels.py:1031-1043): a shape without COLLIDE_PARTICLES gets no
    contacts; a particle and a shape of different worlds do not collide unless either is global."""
    m = _world_scene("cpu")
    assert list(m.shape_world) == [0, 1, 2, -1] and list(m.shape_flags) == [4, 4, 0, 4]
    pw = m.particle_world.numpy()
    assert list(np.unique(pw)) == [0, 1, 2]
    args = (m.particle_q.double().numpy(), m.particle_radius.double().numpy(), m.particle_flags.numpy(), m.shape_type,
            m.shape_transform.astype(np.float64), m.shape_scale.astype(np.float64), 0.01)  # fmt: skip
    cnt, p, s, _, _, _ = orc.soft_contacts_shapes(*args, shape_flags=m.shape_flags, shape_world=m.shape_world,
                                                  particle_world=pw)  # fmt: skip
    p, s = p[:cnt], s[:cnt]
    assert set(s.tolist()) == {0, 1, 3}
    sph = s < 3
    assert (pw[p[sph]] == s[sph]).all()  # every sphere contact is within the particle's own world
    assert set(pw[p[s == 3]].tolist()) == {0, 1, 2}  # the global plane touches every world
    # without the filters the same particles also touch the other worlds' spheres
    cnt_all, _, s_all, _, _, _ = orc.soft_contacts_shapes(*args)
    assert cnt_all > cnt and set(s_all[:cnt_all].tolist()) == {0, 1, 2, 3}


def test_oracle_matches_reference_create_soft_contacts_kernel():
    """The reference's ``create_soft_contacts`` kernel itself, run serially through the Warp stand-in: three worlds
    with their own shapes, global shapes, a shape without COLLIDE_PARTICLES, inactive and global particles, and a
    heightfield. A serial launch lists contacts in thread order (particle-major), the oracle's loop order, so the
    lists must agree entry by entry."""
    g = load_golden("create_soft_contacts.npz")
    cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(
        g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"], g["shape_scale"], float(g["margin"]),
        heightfield_index=g["shape_heightfield_index"], heightfields=g["heightfields"], elevations=g["elevations"],
        shape_flags=g["shape_flags"], shape_world=g["shape_world"], particle_world=g["particle_world"])  # fmt: skip
    assert cnt == len(g["particle"]) and cnt > 500
    np.testing.assert_array_equal(p[:cnt], g["particle"])
    np.testing.assert_array_equal(s[:cnt], g["shape"])
    assert np.abs(bp[:cnt] - g["body_pos"]).max() <= 1e-12
    assert np.abs(nn[:cnt] - g["normal"]).max() <= 1e-12
    assert np.abs(bv[:cnt]).max() == 0.0
    # every filter is exercised: the non-colliding shape has no contact, cross-world pairs are absent, global
    # particles touch world shapes
    pw, sw = g["particle_world"][g["particle"]], g["shape_world"][g["shape"]]
    assert 5 not in set(g["shape"].tolist())
    assert ((pw == -1) | (sw == -1) | (pw == sw)).all() and ((pw == -1) & (sw >= 0)).any()


def test_oracle_matches_reference_create_soft_contacts_on_bodies():
    """``create_soft_contacts`` with shapes on two rotated, displaced bodies (geometry/kernels.py:1045-1056,
    1128-1140), run as-is: the oracle composes body_q[body] with the shape's own transform, writes contact points in
    the body's frame and normals in world, entry by entry in thread order."""
    g = load_golden("create_soft_contacts_bodies.npz")
    cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(
        g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"], g["shape_scale"], float(g["margin"]),
        shape_body=g["shape_body"], body_q=g["body_q"])  # fmt: skip
    assert cnt == len(g["particle"]) and cnt > 300
    np.testing.assert_array_equal(p[:cnt], g["particle"])
    np.testing.assert_array_equal(s[:cnt], g["shape"])
    assert np.abs(bp[:cnt] - g["body_pos"]).max() <= 1e-12
    assert np.abs(nn[:cnt] - g["normal"]).max() <= 1e-12
    # every body shape is touched, and its contact points are in the body frame, not in world
    assert set(g["shape"].tolist()) == set(range(len(g["shape_type"])))
    on_body = g["shape_body"][g["shape"]] >= 0
    static = orc.soft_contacts_shapes(g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"],
                                      g["shape_scale"], float(g["margin"]))  # fmt: skip
    assert on_body.any() and static[0] != cnt
