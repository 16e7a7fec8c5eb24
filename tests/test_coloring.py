"""Particle coloring: validity on the particle graph of ModelBuilder.color (the check of
``validate_graph_coloring``, graph_coloring.py:26-31, and test_coloring.py's intent), balance, and the
world-merge rule ``combine_independent_particle_coloring``."""

import numpy as np
import pytest

from newton_chysx_b200 import sim
from tests.helpers import cloth_grid_builder


def graph_edges(b: sim.ModelBuilder, include_bending: bool):
    pairs = set()
    for t in b.tri_indices:
        for i in range(3):
            for j in range(i + 1, 3):
                pairs.add((min(t[i], t[j]), max(t[i], t[j])))
    if include_bending:
        for e, p in zip(b.edge_indices, b.edge_bending_properties, strict=True):
            if p[0] == 0.0 and p[1] == 0.0:
                continue
            v = [x for x in e if x >= 0]
            for i in range(len(v)):
                for j in range(i + 1, len(v)):
                    pairs.add((min(v[i], v[j]), max(v[i], v[j])))
    return pairs


@pytest.mark.parametrize("n", [2, 5, 16, 33])
@pytest.mark.parametrize("include_bending", [False, True])
@pytest.mark.parametrize("algorithm", [sim.ColoringAlgorithm.MCS, sim.ColoringAlgorithm.GREEDY])
def test_coloring_is_valid_and_complete(n, include_bending, algorithm):
    b = cloth_grid_builder(n=n)
    b.color(include_bending=include_bending, coloring_algorithm=algorithm)
    groups = b.particle_color_groups
    colors = -np.ones(b.particle_count, dtype=int)
    for c, g in enumerate(groups):
        assert np.all(colors[g] == -1)
        colors[g] = c
        assert np.all(np.diff(g) > 0)  # particles of a group in index order
    assert np.all(colors >= 0)
    for a, c in graph_edges(b, include_bending):
        assert colors[a] != colors[c]


def test_grid_coloring_is_small_and_balanced():
    b = cloth_grid_builder(n=64)
    b.color(include_bending=True, target_max_min_color_ratio=1.1)
    sizes = [len(g) for g in b.particle_color_groups]
    assert len(sizes) <= 6
    assert max(sizes) / min(sizes) <= 1.1 + 1e-9


def test_combine_independent_coloring():
    g1 = [np.array([0, 1, 2]), np.array([3])]
    g2 = [np.array([10]), np.array([11, 12]), np.array([13, 14, 15])]
    out = sim.combine_independent_particle_coloring(g1, g2)
    # the longer list (g2) sorted by ascending size, the shorter (g1) by descending size, then zipped
    assert [x.tolist() for x in out] == [[10, 0, 1, 2], [11, 12, 3], [13, 14, 15]]


def test_world_merge_keeps_each_world_valid():
    top = sim.ModelBuilder()
    for k in range(3):
        b = cloth_grid_builder(n=4 + k)
        top.add_world(b)
    colors = -np.ones(top.particle_count, dtype=int)
    for c, g in enumerate(top.particle_color_groups):
        colors[g] = c
    assert np.all(colors >= 0)
    for a, c in graph_edges(top, True):
        assert colors[a] != colors[c]
    assert top.world_particle_start == [0, 16, 41]


def test_mcs_is_optimal_on_a_chordal_graph():
    """Maximum cardinality search colors chordal graphs optimally (clique number); a fan of triangles around a
    hub plus a chain of triangles is chordal with clique number 3."""
    b = sim.ModelBuilder()
    k = 9
    pts = [(0.0, 0.0, 0.0)] + [(np.cos(a), np.sin(a), 0.0) for a in np.linspace(0.0, 1.5 * np.pi, k)]
    b.add_particles(pts, (0.0, 0.0, 0.0), 1.0)
    hub = np.zeros(k - 1, dtype=int)
    b.add_triangles(hub, np.arange(1, k), np.arange(2, k + 1), tri_ke=1.0, tri_ka=1.0)
    b.color(coloring_algorithm=sim.ColoringAlgorithm.MCS, balance_colors=False)
    assert len(b.particle_color_groups) == 3
