"""The cloth builder against the reference builder's own output (golden model arrays)."""

import numpy as np
import pytest
import torch

from newton_chysx_b200 import sim
from tests.helpers import load_golden


def lame(E, nu, h):
    return E * h / (2.0 * (1.0 + nu)), E * h * nu / (1.0 - nu * nu)


def _compare(b: sim.ModelBuilder, g):
    np.testing.assert_allclose(b.particle_q, g["model_particle_q"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(b.particle_mass, g["model_particle_mass"], rtol=1e-12, atol=0)
    np.testing.assert_array_equal(b.particle_flags, g["model_particle_flags"])
    np.testing.assert_array_equal(b.tri_indices, g["model_tri_indices"])
    np.testing.assert_allclose(b._cat(b._tri_pose, (-1, 2, 2), np.float64), g["model_tri_poses"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(b._cat(b._tri_area, (-1,), np.float64), g["model_tri_areas"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(b.tri_materials, g["model_tri_materials"], rtol=0, atol=0)
    np.testing.assert_array_equal(b.edge_indices, g["model_edge_indices"])
    np.testing.assert_allclose(b._cat(b._edge_angle, (-1,), np.float64), g["model_edge_rest_angle"], atol=1e-12)
    np.testing.assert_allclose(b._cat(b._edge_len, (-1,), np.float64), g["model_edge_rest_length"], rtol=1e-12)
    np.testing.assert_allclose(b.edge_bending_properties, g["model_edge_bending_properties"], rtol=0, atol=0)


def test_cloth_grid_matches_reference_builder():
    g = load_golden("step_grid_ground.npz")
    mu, lam = lame(1.0e4, 0.3, 1.0e-3)
    dim = 7
    b = sim.ModelBuilder()
    b.add_cloth_grid(pos=(0.0, 0.0, 0.004), rot=sim.quat_from_axis_angle((1.0, 0.0, 0.0), np.pi * 0.5),
                     vel=(0.3, 0.0, -0.5), dim_x=dim, dim_y=dim, cell_x=1.0 / dim, cell_y=1.0 / dim,
                     mass=0.2 / (dim + 1) ** 2, tri_ke=mu, tri_ka=lam, tri_kd=1e-2, edge_ke=5e-3, edge_kd=1e-3,
                     particle_radius=5e-3)  # fmt: skip
    flags = b.particle_flags
    for p in [(dim + 1) * dim, (dim + 1) * (dim + 1) - 1]:
        flags[p] &= ~int(sim.ParticleFlags.ACTIVE)
    b.set_particle_flags(flags)
    _compare(b, g)


def test_flat_grid_matches_reference_builder():
    g = load_golden("step_grid_sphere.npz")
    mu, lam = lame(1.0e4, 0.3, 1.0e-3)
    b = sim.ModelBuilder()
    b.add_cloth_grid(pos=(-0.3, -0.3, 0.205), rot=sim.quat_identity(), vel=(0.0, 0.0, -1.0), dim_x=6, dim_y=6,
                     cell_x=0.1, cell_y=0.1, mass=1e-3, tri_ke=mu, tri_ka=lam, tri_kd=0.0, edge_ke=1e-4, edge_kd=0.0,
                     particle_radius=5e-3)  # fmt: skip
    _compare(b, g)


def test_cloth_mesh_matches_reference_builder():
    g = load_golden("step_complex_rest_angle.npz")
    vs = g["model_particle_q"] - np.array([0.0, 2.0, 0.0])
    fs = g["model_tri_indices"].reshape(-1)
    b = sim.ModelBuilder()
    b.add_cloth_mesh(pos=(0.0, 2.0, 0.0), rot=sim.quat_identity(), scale=1.0, vel=(0.0, 0.0, 0.0), vertices=vs,
                     indices=fs, density=0.02, tri_ke=1e3, tri_ka=1e3, tri_kd=1e-2, edge_ke=1e3, edge_kd=1e-3)  # fmt: skip
    flags = b.particle_flags
    flags[1] = 0
    b.set_particle_flags(flags)
    # vertex positions round-trip through the golden (x + 2 - 2), so compare them loosely
    np.testing.assert_allclose(b.particle_q, g["model_particle_q"], atol=1e-12)
    g = dict(g)
    g["model_particle_q"] = b.particle_q
    _compare(b, g)


def test_mesh_hinges_boundary_and_order():
    tri = np.array([[0, 1, 2], [2, 1, 3]])
    h = sim.mesh_hinges(tri)
    # first triangle creates (0,1), (1,2), (2,0); second adds (1,3), (3,2) and closes (1,2)
    np.testing.assert_array_equal(h, [[2, -1, 0, 1], [0, 3, 1, 2], [1, -1, 2, 0], [2, -1, 1, 3], [1, -1, 3, 2]])


def test_degenerate_triangles_are_dropped():
    b = sim.ModelBuilder()
    b.add_particles([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 1, 0]], (0, 0, 0), [1, 1, 1, 1])
    areas = b.add_triangles([0, 0], [1, 1], [2, 3])
    assert areas[0] == 0.0 and areas[1] == pytest.approx(0.5)
    assert b.tri_count == 1


def test_bodies_carry_shapes_through_worlds():
    """add_body (builder.py:3814-3878) and shapes on bodies: a shape's body index moves with its world's bodies
    when builders are merged, a shape on a missing body is refused, and states carry the bodies' transforms and
    velocities."""
    from newton_chysx_b200 import sim

    b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    b.add_particles(np.zeros((2, 3)), (0.0, 0.0, 0.0), 1.0, np.full(2, 0.01), np.ones(2, np.int32))
    body = b.add_body(xform=((0.1, 0.2, 0.3), sim.quat_from_axis_angle((0.0, 0.0, 1.0), 0.5)), mass=2.0,
                      com=(0.0, 0.0, 0.05))  # fmt: skip
    b.add_shape_sphere(body=body, radius=0.1)
    b.add_shape_box(hx=0.1, hy=0.1, hz=0.1)
    with pytest.raises(ValueError, match="body 3"):
        b.add_shape_sphere(body=3, radius=0.1)
    top = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    top.add_world(b)
    top.add_world(b)
    assert top.body_count == 2 and [s["body"] for s in top.shapes] == [0, -1, 1, -1]
    assert [bd["world"] for bd in top.bodies] == [0, 1]
    m = top.finalize("cpu")
    assert m.body_count == 2 and m._shape_body_host.tolist() == [0, -1, 1, -1]
    assert m.shape_body.tolist() == [0, -1, 1, -1]
    np.testing.assert_allclose(m.body_q[1, :3].numpy(), [0.1, 0.2, 0.3], atol=1e-7)
    np.testing.assert_allclose(m.body_com[0].numpy(), [0.0, 0.0, 0.05], atol=1e-7)
    st = m.state()
    assert tuple(st.body_q.shape) == (2, 7) and tuple(st.body_qd.shape) == (2, 6)
    st2 = m.state()
    st2.body_q += 1.0
    st.assign(st2)
    assert torch.equal(st.body_q, st2.body_q)
    static = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    static.add_particles(np.zeros((1, 3)), (0.0, 0.0, 0.0), 1.0, np.full(1, 0.01), np.ones(1, np.int32))
    static.add_ground_plane()
    ms = static.finalize("cpu")
    assert ms.body_count == 0 and ms.body_q is None and ms.state().body_q is None
