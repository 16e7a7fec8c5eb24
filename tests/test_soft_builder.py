"""Host side of springs and tetrahedra: the builder reproduces the reference's ``add_soft_grid`` /
``add_tetrahedron`` / ``add_spring`` arrays (the golden soft block was built by the reference's own builder
code), and the coloring keeps every tetrahedron's vertices apart while leaving springs out of the graph, as
``construct_particle_graph`` does."""

import ctypes as C

import numpy as np

from newton_chysx_b200 import _lib, sim
from tests.helpers import load_golden


def soft_block_builder():
    """The golden soft block: a 3 x 2 x 2-cell grid hung from an anchor particle by three springs, with one
    diagonal spring."""
    b = sim.ModelBuilder()
    b.add_soft_grid(pos=(0.0, 0.0, 0.004), rot=sim.quat_identity(), vel=(0.2, 0.0, -0.8), dim_x=3, dim_y=2, dim_z=2,
                    cell_x=0.05, cell_y=0.05, cell_z=0.05, density=500.0, k_mu=2.0e4, k_lambda=3.0e4, k_damp=1.0e-3,
                    particle_radius=5e-3)  # fmt: skip
    nv = b.particle_count
    anchor = b.add_particle((0.075, 0.05, 0.4), (0.0, 0.0, 0.0), 0.0, 5e-3)
    for corner in (nv - 1, nv - 4, nv - 12):
        b.add_spring(anchor, corner, 2.0e2, 1.0e-2, 0.0)
    b.add_spring(0, nv - 1, 5.0e2, 0.0, 0.0)
    return b


def test_soft_grid_matches_reference_builder():
    g = load_golden("step_soft_block.npz")
    b = soft_block_builder()
    assert b.particle_count == len(g["model_particle_mass"])
    np.testing.assert_allclose(b.particle_q, g["model_particle_q"], atol=1e-7)
    np.testing.assert_allclose(b.particle_mass, g["model_particle_mass"], rtol=1e-12)
    np.testing.assert_array_equal(b.particle_flags, g["model_particle_flags"])
    np.testing.assert_array_equal(b.tet_indices, g["model_tet_indices"])
    np.testing.assert_allclose(b.tet_poses, g["model_tet_poses"], rtol=1e-5, atol=1e-4)
    np.testing.assert_allclose(b.tet_materials, g["model_tet_materials"], rtol=1e-12)
    np.testing.assert_array_equal(b.tri_indices, g["model_tri_indices"])
    np.testing.assert_allclose(b.tri_materials, g["model_tri_materials"], rtol=1e-12)
    np.testing.assert_array_equal(b.edge_indices, g["model_edge_indices"])
    np.testing.assert_allclose(b.edge_bending_properties, g["model_edge_bending_properties"], rtol=1e-12)
    np.testing.assert_array_equal(b.spring_indices.reshape(-1, 2), g["model_spring_indices"])
    np.testing.assert_allclose(b._cat(b._spr_rest, (-1,), np.float64), g["model_spring_rest_length"], rtol=1e-6)
    np.testing.assert_allclose(b._cat(b._spr_ke, (-1,), np.float64), g["model_spring_stiffness"])
    np.testing.assert_allclose(b._cat(b._spr_kd, (-1,), np.float64), g["model_spring_damping"])


def test_inverted_tetrahedron_is_not_added():
    b = sim.ModelBuilder()
    b.add_particles([(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)], (0, 0, 0), 1.0)
    assert b.add_tetrahedron(0, 2, 1, 3) < 0.0  # negative orientation
    assert b.tet_count == 0
    v = b.add_tetrahedron(0, 1, 2, 3, 5.0, 7.0, 0.1)
    assert abs(v - 1.0 / 6.0) < 1e-12 and b.tet_count == 1
    np.testing.assert_allclose(b.tet_poses[0], np.eye(3))
    np.testing.assert_allclose(b.tet_materials[0], [5.0, 7.0, 0.1])


def test_coloring_separates_tet_vertices_and_ignores_springs():
    b = soft_block_builder()
    b.color()
    groups = b.particle_color_groups
    colors = np.full(b.particle_count, -1)
    for c, grp in enumerate(groups):
        colors[grp] = c
    assert (colors >= 0).all()
    for t in b.tet_indices:
        assert len(set(colors[t])) == 4
    # springs are not graph edges: without balancing the anchor has no neighbours and takes the first color
    b.color(balance_colors=False)
    assert b.particle_count - 1 in set(b.particle_color_groups[0].tolist())


def test_world_copies_offset_springs_and_tets():
    inner = soft_block_builder()
    b = sim.ModelBuilder()
    b.add_world(inner)
    b.add_world(inner)
    n = inner.particle_count
    assert b.tet_count == 2 * inner.tet_count and b.spring_count == 2 * inner.spring_count
    np.testing.assert_array_equal(b.tet_indices[inner.tet_count:], inner.tet_indices + n)
    np.testing.assert_array_equal(b.spring_indices[2 * inner.spring_count:], inner.spring_indices + n)


def test_color_graph_entry_point():
    lib = _lib.load()
    ip = C.POINTER(C.c_int32)
    pairs = np.array([[0, 1], [1, 2], [2, 0], [2, 3], [3, 3]], dtype=np.int32)
    colors = np.zeros(4, np.int32)
    n = lib.vbd_color_graph(4, len(pairs), pairs.ctypes.data_as(ip), 0, 0.0, colors.ctypes.data_as(ip))
    assert n == 3
    for a, c in pairs:
        assert a == c or colors[a] != colors[c]
    bad = np.array([[0, 9]], dtype=np.int32)
    assert lib.vbd_color_graph(4, 1, bad.ctypes.data_as(ip), 0, 0.0, colors.ctypes.data_as(ip)) == _lib.VBD_ERR_INVALID_ARGUMENT
