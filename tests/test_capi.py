"""The C-ABI library loads without a GPU and exports every function include/vbd_b200.h declares;
host-side entry points (adjacency, coloring) run on the CPU."""

import ctypes as C
import os
import re

import numpy as np

from newton_chysx_b200 import _lib
from oracle import vbd_oracle as orc
from tests.helpers import cloth_grid_builder, load_golden

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "vbd_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(vbd_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures must cover the header exactly"


def test_adjacency_matches_reference_fill_order():
    g = load_golden("step_grid_ground.npz")
    lib = _lib.load()
    n = len(g["model_particle_mass"])
    tri = np.ascontiguousarray(g["model_tri_indices"], dtype=np.int32)
    edges = np.ascontiguousarray(g["model_edge_indices"], dtype=np.int32)
    fo = np.zeros(n + 1, np.int32)
    eo = np.zeros(n + 1, np.int32)
    fa = np.zeros(6 * len(tri), np.int32)
    ea = np.zeros(8 * len(edges), np.int32)
    ip = C.POINTER(C.c_int32)
    rc = lib.vbd_build_adjacency(n, len(tri), tri.ctypes.data_as(ip), len(edges), edges.ctypes.data_as(ip),
                                 fo.ctypes.data_as(ip), fa.ctypes.data_as(ip), eo.ctypes.data_as(ip),
                                 ea.ctypes.data_as(ip))  # fmt: skip
    assert rc == 0
    np.testing.assert_array_equal(fo, g["adj_face_offsets"])
    np.testing.assert_array_equal(fa[: fo[-1]], g["adj_faces"])
    np.testing.assert_array_equal(eo, g["adj_edge_offsets"])
    np.testing.assert_array_equal(ea[: eo[-1]], g["adj_edges"])
    ofo, ofa, oeo, oea = orc.build_adjacency(n, tri, edges)
    np.testing.assert_array_equal(fa[: fo[-1]], ofa)


def test_host_entry_points_reject_bad_input():
    lib = _lib.load()
    ip = C.POINTER(C.c_int32)
    tri = np.array([[0, 1, 7]], dtype=np.int32)  # index out of range
    fo = np.zeros(4, np.int32)
    fa = np.zeros(6, np.int32)
    rc = lib.vbd_build_adjacency(3, 1, tri.ctypes.data_as(ip), 0, None, fo.ctypes.data_as(ip), fa.ctypes.data_as(ip),
                                 fo.ctypes.data_as(ip), fa.ctypes.data_as(ip))  # fmt: skip
    assert rc == _lib.VBD_ERR_INVALID_ARGUMENT
    assert lib.vbd_create(None, None, None) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert lib.vbd_destroy(None) == _lib.VBD_ERR_INVALID_ARGUMENT


def test_coloring_entry_point_on_large_grid():
    b = cloth_grid_builder(n=256)
    b.color(include_bending=True)
    assert sum(len(g) for g in b.particle_color_groups) == 256 * 256
