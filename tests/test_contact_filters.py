"""Topological self-contact filters (C++) against the reference's own n-ring filter builders.

The goldens hold the filter lists that ``build_vertex_n_ring_tris_collision_filter`` and
``build_edge_n_ring_edge_collision_filter`` (particle_vbd_kernels.py:2164-2255) produced for the
self-contact scenes (2-ring and 3-ring). No GPU needed: ``vbd_build_contact_filters`` is host code.
"""

import os

import numpy as np
import pytest

from newton_chysx_b200.collision import build_contact_filters, topological_filters


@pytest.mark.parametrize("name", ["step_selfcontact_layers.npz", "step_selfcontact_fold.npz"])
def test_filters_match_reference(golden_dir, name):
    g = dict(np.load(os.path.join(golden_dir, name)))
    ring = int(g["sc_ring"])
    (vf, vo), (ef, eo) = topological_filters(len(g["model_particle_mass"]), g["model_tri_indices"],
                                             g["model_edge_indices"], ring)  # fmt: skip
    np.testing.assert_array_equal(vo, g["sc_vt_filter_offsets"])
    np.testing.assert_array_equal(vf, g["sc_vt_filter"])
    np.testing.assert_array_equal(eo, g["sc_ee_filter_offsets"])
    np.testing.assert_array_equal(ef, g["sc_ee_filter"])
    assert len(vf) > 0 and len(ef) > 0


def test_external_maps_are_merged(golden_dir):
    g = dict(np.load(os.path.join(golden_dir, "step_selfcontact_layers.npz")))
    V = len(g["model_particle_mass"])
    vt, ee = build_contact_filters(V, g["model_tri_indices"], g["model_edge_indices"], 2,
                                   external_vertex_map={0: {100, 5}}, external_edge_map={3: {7}})  # fmt: skip
    base_vt, base_ee = topological_filters(V, g["model_tri_indices"], g["model_edge_indices"], 2)
    row0 = vt[0][vt[1][0] : vt[1][1]]
    assert {100, 5} <= set(row0.tolist()) and list(row0) == sorted(row0)
    assert set(row0.tolist()) == set(base_vt[0][base_vt[1][0] : base_vt[1][1]].tolist()) | {100, 5}
    assert 7 in ee[0][ee[1][3] : ee[1][4]]
    # threshold below 2: only the external maps
    vt1, ee1 = build_contact_filters(V, g["model_tri_indices"], g["model_edge_indices"], 1,
                                     external_vertex_map={2: {9}})  # fmt: skip
    assert ee1 is None and vt1[1][-1] == 1 and vt1[0][0] == 9
