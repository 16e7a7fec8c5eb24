"""Particle self-contact: collision filters and the stand-alone triangle-mesh collision detector.

``build_contact_filters`` mirrors ``SolverVBD._compute_particle_contact_filtering_list``
(``newton/_src/solvers/vbd/solver_vbd.py:1339-1404``): the n-ring topological filters are computed by
``vbd_build_contact_filters`` (C++) and the caller's external filtering maps are merged in.

``TriMeshCollisionDetector`` has the interface of the reference class of the same name
(``newton/_src/solvers/vbd/tri_mesh_collision.py:91-413``) and the same buffers (vertex -> colliding
triangles, edge -> colliding edges, counts, minimum distances, ``resize_flags``), computed by the
library's grid-based detector (``vbd_collider_*``). Within a buffer the pairs are kept in increasing
primitive id; the reference keeps them in its BVH's traversal order. With
``record_triangle_contacting_vertices`` the vertex-triangle detection also fills the triangle -> colliding
vertices buffers (``triangle_colliding_vertices``, ``_count``, ``_offsets``, ``_buffer_sizes``, ``_min_dist``;
``tri_mesh_collision.py:170-200``, ``geometry/kernels.py:1373-1384``), each triangle's vertices in increasing
id where the reference has them in the order its threads arrived.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _np(t, dtype):
    if isinstance(t, torch.Tensor):
        t = t.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(t), dtype=dtype)


def topological_filters(particle_count: int, tri_indices, edge_indices, ring: int):
    """n-ring filters (ring >= 2): ((vt_flat, vt_offsets), (ee_flat, ee_offsets)), rows sorted."""
    tri = _np(tri_indices, np.int32).reshape(-1, 3)
    edg = _np(edge_indices, np.int32).reshape(-1, 4)
    V, T, E = int(particle_count), len(tri), len(edg)
    lib = _lib.load()
    vo = np.zeros(V + 1, dtype=np.int32)
    eo = np.zeros(E + 1, dtype=np.int32)
    _lib.check(lib.vbd_build_contact_filters(V, T, _ip(tri), E, _ip(edg), int(ring), _ip(vo), None, _ip(eo), None),
               "vbd_build_contact_filters")  # fmt: skip
    vl = np.zeros(max(int(vo[-1]), 1), dtype=np.int32)
    el = np.zeros(max(int(eo[-1]), 1), dtype=np.int32)
    _lib.check(lib.vbd_build_contact_filters(V, T, _ip(tri), E, _ip(edg), int(ring), _ip(vo), _ip(vl), _ip(eo), _ip(el)),
               "vbd_build_contact_filters")  # fmt: skip
    return (vl[: vo[-1]].copy(), vo), (el[: eo[-1]].copy(), eo)


def _merge(csr, rows: int, extra: dict | None):
    if extra is None:
        return csr
    sets = [set() for _ in range(rows)]
    if csr is not None:
        flat, off = csr
        for i in range(rows):
            sets[i].update(int(x) for x in flat[off[i] : off[i + 1]])
    for k, v in extra.items():
        sets[int(k)].update(int(x) for x in v)
    off = np.zeros(rows + 1, dtype=np.int32)
    np.cumsum([len(s) for s in sets], out=off[1:])
    flat = np.fromiter((x for s in sets for x in sorted(s)), dtype=np.int32, count=int(off[-1]))
    return flat, off


def build_contact_filters(particle_count: int, tri_indices, edge_indices, threshold: int = 2,
                          external_vertex_map: dict | None = None, external_edge_map: dict | None = None):  # fmt: skip
    """(vertex -> filtered triangles, edge -> filtered edges) CSR pairs, each None when empty, as
    ``_compute_particle_contact_filtering_list`` builds them."""
    E = len(_np(edge_indices, np.int32).reshape(-1, 4))
    vt = ee = None
    if threshold >= 2:
        vt, ee = topological_filters(particle_count, tri_indices, edge_indices, threshold)
    vt = _merge(vt, int(particle_count), external_vertex_map)
    ee = _merge(ee, E, external_edge_map)
    return vt, ee


class TriMeshCollisionDetector:
    """Vertex-triangle and edge-edge proximity detection over a model's triangles and edges."""

    def __init__(self, model, record_triangle_contacting_vertices=False, vertex_positions=None,
                 vertex_collision_buffer_pre_alloc=8, vertex_collision_buffer_max_alloc=256,
                 vertex_triangle_filtering_list=None, vertex_triangle_filtering_list_offsets=None,
                 triangle_collision_buffer_pre_alloc=16, triangle_collision_buffer_max_alloc=256,
                 edge_collision_buffer_pre_alloc=8, edge_collision_buffer_max_alloc=256, edge_filtering_list=None,
                 edge_filtering_list_offsets=None, triangle_triangle_collision_buffer_pre_alloc=8,
                 triangle_triangle_collision_buffer_max_alloc=256, edge_edge_parallel_epsilon=1e-5,
                 collision_detection_block_size=16):  # fmt: skip
        self.model = model
        self.device = model.device
        self.vertex_positions = model.particle_q if vertex_positions is None else vertex_positions
        self.vertex_collision_buffer_pre_alloc = int(vertex_collision_buffer_pre_alloc)
        self.edge_collision_buffer_pre_alloc = int(edge_collision_buffer_pre_alloc)
        self.edge_edge_parallel_epsilon = float(edge_edge_parallel_epsilon)
        self.record_triangle_contacting_vertices = bool(record_triangle_contacting_vertices)
        self.triangle_collision_buffer_pre_alloc = int(triangle_collision_buffer_pre_alloc)
        V, E = model.particle_count, model.edge_count
        vb, eb = self.vertex_collision_buffer_pre_alloc, self.edge_collision_buffer_pre_alloc
        dev = self.device
        i32 = torch.int32
        self.vertex_colliding_triangles = torch.full((2 * V * vb,), -1, dtype=i32, device=dev)
        self.vertex_colliding_triangles_count = torch.zeros(V, dtype=i32, device=dev)
        self.vertex_colliding_triangles_min_dist = torch.zeros(V, dtype=torch.float32, device=dev)
        self.vertex_colliding_triangles_buffer_sizes = torch.full((V,), vb, dtype=i32, device=dev)
        self.vertex_colliding_triangles_offsets = torch.arange(0, (V + 1) * vb, vb, dtype=i32, device=dev)
        self.edge_colliding_edges = torch.full((2 * E * eb,), -1, dtype=i32, device=dev)
        self.edge_colliding_edges_count = torch.zeros(E, dtype=i32, device=dev)
        self.edge_colliding_edges_min_dist = torch.zeros(E, dtype=torch.float32, device=dev)
        self.edge_colliding_edges_buffer_sizes = torch.full((E,), eb, dtype=i32, device=dev)
        self.edge_colliding_edges_offsets = torch.arange(0, (E + 1) * eb, eb, dtype=i32, device=dev)
        self.triangle_colliding_vertices_min_dist = torch.zeros(model.tri_count, dtype=torch.float32, device=dev)
        T, tb = model.tri_count, self.triangle_collision_buffer_pre_alloc
        if self.record_triangle_contacting_vertices:
            self.triangle_colliding_vertices = torch.full((T * tb,), -1, dtype=i32, device=dev)
            self.triangle_colliding_vertices_count = torch.zeros(T, dtype=i32, device=dev)
            self.triangle_colliding_vertices_buffer_sizes = torch.full((T,), tb, dtype=i32, device=dev)
            self.triangle_colliding_vertices_offsets = torch.arange(0, (T + 1) * tb, tb, dtype=i32, device=dev)
        else:
            self.triangle_colliding_vertices = None
            self.triangle_colliding_vertices_count = None
            self.triangle_colliding_vertices_buffer_sizes = None
            self.triangle_colliding_vertices_offsets = None
        self.resize_flags = torch.zeros(4, dtype=i32, device=dev)
        self._h = None
        self.set_collision_filter_list(vertex_triangle_filtering_list, vertex_triangle_filtering_list_offsets,
                                       edge_filtering_list, edge_filtering_list_offsets)  # fmt: skip

    def set_collision_filter_list(self, vertex_triangle_filtering_list, vertex_triangle_filtering_list_offsets,
                                  edge_filtering_list, edge_filtering_list_offsets):  # fmt: skip
        """CSR filter lists (as ``set_to_csr`` builds them): triangles skipped per vertex, edges per edge."""
        self._destroy()
        m = self.model
        keep = []

        def csr(flat, off):
            if flat is None or off is None:
                return None, None
            f, o = _np(flat, np.int32), _np(off, np.int32)
            keep.extend([f, o])
            return _ip(f), _ip(o)

        vf, vo = csr(vertex_triangle_filtering_list, vertex_triangle_filtering_list_offsets)
        ef, eo = csr(edge_filtering_list, edge_filtering_list_offsets)
        h = C.c_void_p()
        lib = _lib.load()
        with torch.cuda.device(self.device):
            _lib.check(lib.vbd_collider_create(
                m.particle_count, m.tri_count, C.c_void_p(m.tri_indices.data_ptr()) if m.tri_count else None,
                m.edge_count, C.c_void_p(m.edge_indices.data_ptr()) if m.edge_count else None,
                self.vertex_collision_buffer_pre_alloc, self.edge_collision_buffer_pre_alloc,
                self.edge_edge_parallel_epsilon, vo, vf, eo, ef, C.byref(h)), "vbd_collider_create")  # fmt: skip
        self._h = h
        if self.record_triangle_contacting_vertices:
            _lib.check(lib.vbd_collider_set_triangle_buffers(
                h, self.triangle_collision_buffer_pre_alloc, C.c_void_p(self.triangle_colliding_vertices.data_ptr()),
                C.c_void_p(self.triangle_colliding_vertices_count.data_ptr()),
                C.c_void_p(self.triangle_colliding_vertices_min_dist.data_ptr())),
                "vbd_collider_set_triangle_buffers")  # fmt: skip

    def refit(self, new_pos=None):
        """The grid is rebuilt by every detection; this only records the positions to use."""
        if new_pos is not None:
            self.vertex_positions = new_pos

    def rebuild(self, new_pos=None):
        self.refit(new_pos)

    def _detect(self, what, max_query_radius, min_query_radius, ref_pos):
        q = self.vertex_positions
        if q.dtype != torch.float32 or not q.is_contiguous():
            raise TypeError("vertex positions must be a contiguous float32 tensor")
        if min_query_radius > 0.0 and ref_pos is None:
            ref_pos = q
        stream = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

        def p(t):
            return C.c_void_p(t.data_ptr())

        _lib.check(_lib.load().vbd_collider_detect(
            self._h, what, p(q), float(max_query_radius), float(min_query_radius),
            None if ref_pos is None else p(ref_pos), p(self.vertex_colliding_triangles),
            p(self.vertex_colliding_triangles_count), p(self.vertex_colliding_triangles_min_dist),
            p(self.edge_colliding_edges), p(self.edge_colliding_edges_count), p(self.edge_colliding_edges_min_dist),
            p(self.resize_flags), stream), "vbd_collider_detect")  # fmt: skip

    def vertex_triangle_collision_detection(self, max_query_radius, min_query_radius=0.0,
                                            min_distance_filtering_ref_pos=None):  # fmt: skip
        if not self.record_triangle_contacting_vertices:  # recorded: the detection initialises and fills it
            self.triangle_colliding_vertices_min_dist.fill_(float(max_query_radius))
        self._detect(1, max_query_radius, min_query_radius, min_distance_filtering_ref_pos)

    def edge_edge_collision_detection(self, max_query_radius, min_query_radius=0.0,
                                      min_distance_filtering_ref_pos=None):  # fmt: skip
        self._detect(2, max_query_radius, min_query_radius, min_distance_filtering_ref_pos)

    def _destroy(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().vbd_collider_destroy(h)
            except Exception:
                pass
        self._h = None

    def __del__(self):
        self._destroy()
