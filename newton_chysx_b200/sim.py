"""Cloth-side mirror of the reference's simulation data model (``newton/_src/sim``).

The solver boundary is ``SolverVBD.step(state_in, state_out, control, contacts, dt)``; this module
provides the objects that call carries, with the reference's field names and array layouts
(``Model``, ``State``, ``Control``, ``Contacts``), plus the part of ``ModelBuilder`` that builds
cloth (``add_cloth_grid``, ``add_cloth_mesh``, ``add_triangles``, ``add_edges``, ``color``,
``add_world``, ground plane and sphere shapes) and a ``CollisionPipeline`` for particle-shape soft
contacts. Arrays are torch tensors: float32 ``(N, 3)`` for vec3, ``(T, 2, 2)`` for mat22, int32
indices — the memory layout of the reference's Warp arrays.

Builder math follows ``newton/_src/sim/builder.py`` (``add_triangles :7716-7826``,
``add_edges :7966-8061``, ``add_cloth_grid :8063-8186``, ``add_cloth_mesh :8188-8341``,
``color :9304-9396``, world merge ``:3185-3193``), ``newton/_src/utils/mesh.py`` (``MeshAdjacency
:183-262``) and ``newton/_src/sim/graph_coloring.py`` (``combine_independent_particle_coloring
:382-426``), vectorised with numpy.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import math

import numpy as np
import torch

from . import _lib, interop


class ParticleFlags(enum.IntEnum):
    """``newton/_src/geometry/flags.py:8-14``."""

    ACTIVE = 1 << 0


class GeoType(enum.IntEnum):
    """``newton/_src/geometry/types.py:68-110`` (the same values)."""

    NONE = 0
    PLANE = 1
    HFIELD = 2
    SPHERE = 3
    CAPSULE = 4
    ELLIPSOID = 5
    CYLINDER = 6
    BOX = 7
    MESH = 8
    CONE = 9
    CONVEX_MESH = 10


@dataclasses.dataclass
class ShapeConfig:
    """Material of a collision shape (the reference's ``ModelBuilder.ShapeConfig`` defaults)."""

    ke: float = 2.5e3
    kd: float = 100.0
    mu: float = 1.0
    has_particle_collision: bool = True


# ----------------------------------------------------------------------------- quaternions (x, y, z, w)
def quat_identity():
    return (0.0, 0.0, 0.0, 1.0)


def quat_from_axis_angle(axis, angle):
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    s = math.sin(angle * 0.5)
    return (float(a[0] * s), float(a[1] * s), float(a[2] * s), math.cos(angle * 0.5))


def quat_between_vectors(a, b):
    """The rotation taking direction a to direction b (x, y, z, w)."""
    a = np.asarray(a, dtype=np.float64) / np.linalg.norm(a)
    b = np.asarray(b, dtype=np.float64) / np.linalg.norm(b)
    c = float(np.dot(a, b))
    if c < -1.0 + 1e-9:  # opposite: half a turn about any axis perpendicular to a
        axis = np.cross(a, (1.0, 0.0, 0.0))
        if np.linalg.norm(axis) < 1e-6:
            axis = np.cross(a, (0.0, 1.0, 0.0))
        return quat_from_axis_angle(axis, math.pi)
    v = np.cross(a, b)
    q = np.array([v[0], v[1], v[2], 1.0 + c])
    q /= np.linalg.norm(q)
    return tuple(float(x) for x in q)


def _xform(xform):
    """(position, quaternion xyzw) from None, a (p, q) pair or a 7-vector."""
    if xform is None:
        return (0.0, 0.0, 0.0), quat_identity()
    if len(xform) == 2:
        return tuple(float(v) for v in xform[0]), tuple(float(v) for v in xform[1])
    x = [float(v) for v in xform]
    return tuple(x[:3]), tuple(x[3:7]) if len(x) >= 7 else quat_identity()


def quat_to_matrix(q):
    x, y, z, w = (float(v) for v in q)
    u = np.array([x, y, z])
    e = np.eye(3)
    cols = [e[i] * (2.0 * w * w - 1.0) + np.cross(u, e[i]) * 2.0 * w + u * 2.0 * np.dot(u, e[i]) for i in range(3)]
    return np.stack(cols, axis=1)


# ----------------------------------------------------------------------------- mesh adjacency
def mesh_hinges(tri: np.ndarray) -> np.ndarray:
    """Hinges ``(o0, o1, v0, v1)`` of a triangle mesh, in the order ``MeshAdjacency`` creates them.

    For every triangle (in order) and its edges (0,1), (1,2), (2,0): the first triangle that has an
    undirected edge fixes ``v0, v1`` (its winding) and ``o0``; the second sets ``o1``; edges with a
    single triangle keep ``o1 = -1``; further triangles on a non-manifold edge are ignored.
    """
    tri = np.asarray(tri, dtype=np.int64).reshape(-1, 3)
    if len(tri) == 0:
        return np.zeros((0, 4), dtype=np.int32)
    i0 = np.stack([tri[:, 0], tri[:, 1], tri[:, 2]], axis=1).reshape(-1)
    i1 = np.stack([tri[:, 1], tri[:, 2], tri[:, 0]], axis=1).reshape(-1)
    op = np.stack([tri[:, 2], tri[:, 0], tri[:, 1]], axis=1).reshape(-1)
    lo, hi = np.minimum(i0, i1), np.maximum(i0, i1)
    key = lo * (int(hi.max()) + 1) + hi
    order = np.argsort(key, kind="stable")
    ks = key[order]
    start = np.ones(len(ks), dtype=bool)
    start[1:] = ks[1:] != ks[:-1]
    group_start = np.nonzero(start)[0]
    first = order[group_start]
    has_second = np.zeros(len(group_start), dtype=bool)
    second = np.full(len(group_start), -1, dtype=np.int64)
    nxt = group_start + 1
    ok = nxt < len(ks)
    ok[ok] &= ~start[nxt[ok]]
    has_second[ok] = True
    second[ok] = order[nxt[ok]]
    creation = np.argsort(first, kind="stable")
    first, second, has_second = first[creation], second[creation], has_second[creation]
    out = np.empty((len(first), 4), dtype=np.int64)
    out[:, 0] = op[first]
    out[:, 1] = np.where(has_second, op[np.maximum(second, 0)], -1)
    out[:, 2] = i0[first]
    out[:, 3] = i1[first]
    return out.astype(np.int32)


def combine_independent_particle_coloring(groups_1, groups_2):
    """Merge the colorings of two disconnected graphs (graph_coloring.py:382-426): the longer list is
    sorted by ascending group size, the shorter by descending size, and groups of equal rank join."""
    if len(groups_1) == 0:
        return groups_2
    if len(groups_2) == 0:
        return groups_1
    n = max(len(groups_1), len(groups_2))
    if len(groups_1) < len(groups_2):
        groups_1, groups_2 = groups_2, groups_1
    g1 = sorted(groups_1, key=len)
    g2 = sorted(groups_2, key=lambda g: -len(g))
    out = []
    for i in range(n):
        a = g1[i] if i < len(g1) else None
        b = g2[i] if i < len(g2) else None
        if a is not None and b is not None:
            out.append(np.concatenate([a, b]))
        elif a is not None:
            out.append(a)
        else:
            out.append(b)
    return out


class _ChunkedGroup:
    """A color group kept as a list of arrays so that merging many worlds stays linear."""

    __slots__ = ("chunks", "size")

    def __init__(self, chunks, size):
        self.chunks = chunks
        self.size = size

    def __len__(self):
        return self.size

    def array(self):
        if len(self.chunks) == 1:
            return self.chunks[0]
        return np.concatenate(self.chunks).astype(np.int32)


def _merge_chunked(groups_1, groups_2):
    """``combine_independent_particle_coloring`` on chunked groups (same ordering rule)."""
    if len(groups_1) == 0:
        return groups_2
    if len(groups_2) == 0:
        return groups_1
    n = max(len(groups_1), len(groups_2))
    if len(groups_1) < len(groups_2):
        groups_1, groups_2 = groups_2, groups_1
    g1 = sorted(groups_1, key=len)
    g2 = sorted(groups_2, key=lambda g: -len(g))
    out = []
    for i in range(n):
        a = g1[i] if i < len(g1) else None
        b = g2[i] if i < len(g2) else None
        if a is not None and b is not None:
            out.append(_ChunkedGroup(a.chunks + b.chunks, a.size + b.size))
        else:
            out.append(a if a is not None else b)
    return out


def particle_graph_pairs(tri_indices, tri_materials, edge_indices, edge_props, include_bending, tet_indices,
                         tet_materials):  # fmt: skip
    """Vertex pairs of the coloring graph of ``construct_particle_graph`` (graph_coloring.py:200-240):
    the three edges of every triangle with mu * lambda != 0, with ``include_bending`` the six vertex pairs
    of every hinge with ke or kd != 0 (pairs with a -1 left out), and the six vertex pairs of every
    tetrahedron with mu * lambda != 0. Springs are not part of the graph, as in the reference."""
    parts = []
    tri = np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
    tm = np.asarray(tri_materials, dtype=np.float32).reshape(-1, 5)
    if len(tri):
        tri = tri[(tm[:, 0] * tm[:, 1]) != 0]
        parts += [tri[:, [0, 1]], tri[:, [0, 2]], tri[:, [1, 2]]]
    ed = np.asarray(edge_indices, dtype=np.int32).reshape(-1, 4)
    ep = np.asarray(edge_props, dtype=np.float32).reshape(-1, 2)
    if include_bending and len(ed):
        ed = ed[(ep[:, 0] != 0) | (ep[:, 1] != 0)]
        for a in range(4):
            for b in range(a + 1, 4):
                pr = ed[:, [a, b]]
                parts.append(pr[(pr >= 0).all(axis=1)])
    tt = np.asarray(tet_indices, dtype=np.int32).reshape(-1, 4)
    tmat = np.asarray(tet_materials, dtype=np.float32).reshape(-1, 3)
    if len(tt):
        tt = tt[(tmat[:, 0] * tmat[:, 1]) != 0]
        for a in range(4):
            for b in range(a + 1, 4):
                parts.append(tt[:, [a, b]])
    if not parts:
        return np.zeros((0, 2), dtype=np.int32)
    return np.ascontiguousarray(np.concatenate(parts).astype(np.int32))


class ColoringAlgorithm(enum.Enum):
    """``newton/_src/sim/graph_coloring.py:12-14``."""

    MCS = 0
    GREEDY = 1


def color_particles(n, tri_indices, tri_materials, edge_indices, edge_props, include_bending=False,
                    balance_colors=True, target_max_min_color_ratio=1.1, tet_indices=None, tet_materials=None,
                    coloring_algorithm=ColoringAlgorithm.MCS):  # fmt: skip
    """Color groups (list of int32 arrays, particles in index order) for VBD's Gauss-Seidel sweep."""
    if n == 0:
        return []
    lib = _lib.load()
    pairs = particle_graph_pairs(tri_indices, tri_materials, edge_indices, edge_props, include_bending,
                                 np.zeros((0, 4)) if tet_indices is None else tet_indices,
                                 np.zeros((0, 3)) if tet_materials is None else tet_materials)  # fmt: skip
    if len(pairs) == 0:
        return [np.arange(n, dtype=np.int32)]
    colors = np.zeros(n, dtype=np.int32)
    ip = C.POINTER(C.c_int32)
    ratio = float(target_max_min_color_ratio if balance_colors else 0.0)
    ncol = lib.vbd_color_graph(n, len(pairs), pairs.ctypes.data_as(ip), ColoringAlgorithm(coloring_algorithm).value,
                               ratio, colors.ctypes.data_as(ip))  # fmt: skip
    if ncol < 0:
        _lib.check(ncol, "vbd_color_graph")
    order = np.argsort(colors, kind="stable")
    bounds = np.searchsorted(colors[order], np.arange(ncol + 1))
    return [order[bounds[c]:bounds[c + 1]].astype(np.int32) for c in range(ncol)]


# ----------------------------------------------------------------------------- builder
class ModelBuilder:
    """The particle subset of the reference ``ModelBuilder``: particles, cloth triangles and hinges,
    springs, tetrahedra, collision shapes (static or on bodies), worlds and coloring."""

    ShapeConfig = ShapeConfig

    def __init__(self, up_axis="Z", gravity: float = -9.81):
        self.up_axis = {"X": 0, "Y": 1, "Z": 2}[up_axis.upper()] if isinstance(up_axis, str) else int(up_axis)
        self.gravity = gravity
        self.default_particle_radius = 0.1
        self.default_tri_ke = 100.0
        self.default_tri_ka = 100.0
        self.default_tri_kd = 10.0
        self.default_tri_drag = 0.0
        self.default_tri_lift = 0.0
        self.default_edge_ke = 100.0
        self.default_edge_kd = 0.0
        self.default_shape_cfg = ShapeConfig()
        self._q, self._qd, self._mass, self._radius, self._flags, self._world = [], [], [], [], [], []
        self._tri, self._tri_pose, self._tri_mat, self._tri_area = [], [], [], []
        self._edge, self._edge_angle, self._edge_len, self._edge_prop = [], [], [], []
        self._spr, self._spr_rest, self._spr_ke, self._spr_kd, self._spr_ctl = [], [], [], [], []
        self._tet, self._tet_pose, self._tet_mat = [], [], []
        self._n = 0
        self._t = 0
        self._e = 0
        self._s = 0
        self._tt = 0
        self.shapes = []  # dicts: type, pos, normal, radius, ke, kd, mu, body
        self.bodies = []  # dicts: q (p, quat xyzw), com, mass, inertia, label, kinematic, world
        self._color_groups: list[_ChunkedGroup] = []
        self.world_count = 0
        self.current_world = -1
        self.world_particle_start: list[int] = []

    # -- counts
    @property
    def particle_count(self):
        return self._n

    @property
    def tri_count(self):
        return self._t

    @property
    def edge_count(self):
        return self._e

    @property
    def shape_count(self):
        return len(self.shapes)

    @property
    def body_count(self):
        return len(self.bodies)

    @property
    def spring_count(self):
        return self._s

    @property
    def tet_count(self):
        return self._tt

    @property
    def up_vector(self):
        v = [0.0, 0.0, 0.0]
        v[self.up_axis] = 1.0
        return tuple(v)

    def _cat(self, lst, shape, dtype):
        if not lst:
            return np.zeros(tuple(0 if d == -1 else d for d in shape), dtype=dtype)
        return np.concatenate([np.asarray(a, dtype=dtype).reshape(shape) for a in lst])

    @property
    def particle_q(self):
        return self._cat(self._q, (-1, 3), np.float64)

    @property
    def particle_mass(self):
        return self._cat(self._mass, (-1,), np.float64)

    @property
    def particle_flags(self):
        return self._cat(self._flags, (-1,), np.int32)

    @property
    def tri_indices(self):
        return self._cat(self._tri, (-1, 3), np.int32)

    @property
    def tri_materials(self):
        return self._cat(self._tri_mat, (-1, 5), np.float64)

    @property
    def edge_indices(self):
        return self._cat(self._edge, (-1, 4), np.int32)

    @property
    def edge_bending_properties(self):
        return self._cat(self._edge_prop, (-1, 2), np.float64)

    @property
    def spring_indices(self):
        """Flat ``[2 * spring_count]`` (end 0, end 1 per spring), the reference's layout."""
        return self._cat(self._spr, (-1,), np.int32)

    @property
    def tet_indices(self):
        return self._cat(self._tet, (-1, 4), np.int32)

    @property
    def tet_poses(self):
        return self._cat(self._tet_pose, (-1, 3, 3), np.float64)

    @property
    def tet_materials(self):
        return self._cat(self._tet_mat, (-1, 3), np.float64)

    def _set_particle_column(self, lst_name, values):
        arr = self._cat(getattr(self, lst_name), (-1,), np.float64 if lst_name != "_flags" else np.int32)
        arr[:] = values
        setattr(self, lst_name, [arr])

    def set_particle_flags(self, flags):
        self._set_particle_column("_flags", np.asarray(flags, dtype=np.int32))

    def set_particle_mass(self, mass):
        self._set_particle_column("_mass", np.asarray(mass, dtype=np.float64))

    # -- particles
    def add_particles(self, pos, vel, mass, radius=None, flags=None):
        pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        self._q.append(pos)
        self._qd.append(np.broadcast_to(np.asarray(vel, dtype=np.float64), (n, 3)).copy())
        self._mass.append(np.broadcast_to(np.asarray(mass, dtype=np.float64), (n,)).copy())
        r = self.default_particle_radius if radius is None else radius
        self._radius.append(np.broadcast_to(np.asarray(r, dtype=np.float64), (n,)).copy())
        f = int(ParticleFlags.ACTIVE) if flags is None else flags
        self._flags.append(np.broadcast_to(np.asarray(f, dtype=np.int32), (n,)).copy())
        self._world.append(np.full(n, self.current_world, dtype=np.int32))
        start = self._n
        self._n += n
        return start

    def add_particle(self, pos, vel, mass, radius=None, flags=None):
        return self.add_particles([pos], [vel], [mass], radius, flags)

    # -- triangles (builder.py:7716-7826)
    def add_triangles(self, i, j, k, tri_ke=None, tri_ka=None, tri_kd=None, tri_drag=None, tri_lift=None):
        i = np.asarray(i, dtype=np.int64)
        j = np.asarray(j, dtype=np.int64)
        k = np.asarray(k, dtype=np.int64)
        q = self.particle_q
        p, qq, r = q[i], q[j], q[k]
        qp, rp = qq - p, r - p

        def normalized(a):
            ln = np.linalg.norm(a, axis=-1, keepdims=True)
            ln[ln == 0] = 1.0
            return a / ln

        nrm = normalized(np.cross(qp, rp))
        e1 = normalized(qp)
        e2 = normalized(np.cross(nrm, e1))
        R = np.concatenate((e1[..., None], e2[..., None]), axis=-1)
        M = np.concatenate((qp[..., None], rp[..., None]), axis=-1)
        D = np.matmul(R.transpose(0, 2, 1), M)
        areas = np.linalg.det(D) / 2.0
        areas[areas < 0.0] = 0.0
        valid = areas > 0.0
        D[~valid] = np.eye(2)
        inv_D = np.linalg.inv(D)
        n = len(i)

        def col(v, d):
            return np.broadcast_to(np.asarray(d if v is None else v, dtype=np.float64), (n,))

        mats = np.stack([col(tri_ke, self.default_tri_ke), col(tri_ka, self.default_tri_ka),
                         col(tri_kd, self.default_tri_kd), col(tri_drag, self.default_tri_drag),
                         col(tri_lift, self.default_tri_lift)], axis=1)  # fmt: skip
        self._tri.append(np.stack([i, j, k], axis=1)[valid].astype(np.int32))
        self._tri_pose.append(inv_D[valid])
        self._tri_mat.append(mats[valid])
        self._tri_area.append(areas[valid])
        self._t += int(valid.sum())
        return areas

    # -- springs (builder.py:7584-7633)
    def add_springs(self, i, j, ke, kd, control=0.0):
        """Springs between particles i[k] and j[k]; the rest length is their current distance, computed in
        float32 as the reference does."""
        i = np.atleast_1d(np.asarray(i, dtype=np.int64))
        j = np.atleast_1d(np.asarray(j, dtype=np.int64))
        n = len(i)
        q = self.particle_q.astype(np.float32)
        d = q[i] - q[j]
        rest = np.sqrt((d * d).sum(axis=1, dtype=np.float32)).astype(np.float64)

        def col(v):
            return np.broadcast_to(np.asarray(v, dtype=np.float64), (n,)).copy()

        self._spr.append(np.stack([i, j], axis=1).reshape(-1).astype(np.int32))
        self._spr_rest.append(rest)
        self._spr_ke.append(col(ke))
        self._spr_kd.append(col(kd))
        self._spr_ctl.append(col(control))
        self._s += n

    def add_spring(self, i, j, ke, kd, control=0.0):
        self.add_springs([i], [j], ke, kd, control)

    # -- tetrahedra (builder.py:7827-7892)
    def add_tetrahedra(self, i, j, k, l, k_mu=1.0e3, k_lambda=1.0e3, k_damp=0.0):  # noqa: E741
        """Volumetric Neo-Hookean tetrahedra (i, j, k, l) with the rest pose of the current positions. As in
        the reference, tetrahedra whose rest volume is not positive are not added. Returns the volumes."""
        idx = [np.atleast_1d(np.asarray(a, dtype=np.int64)) for a in (i, j, k, l)]
        n = len(idx[0])
        q = self.particle_q
        p = q[idx[0]]
        Dm = np.stack([q[idx[1]] - p, q[idx[2]] - p, q[idx[3]] - p], axis=2)  # columns
        vol = np.linalg.det(Dm) / 6.0 if n else np.zeros(0)
        valid = vol > 0.0
        inv = np.linalg.inv(Dm[valid]) if valid.any() else np.zeros((0, 3, 3))

        def col(v):
            return np.broadcast_to(np.asarray(v, dtype=np.float64), (n,))

        mats = np.stack([col(k_mu), col(k_lambda), col(k_damp)], axis=1)[valid]
        self._tet.append(np.stack(idx, axis=1)[valid].astype(np.int32))
        self._tet_pose.append(inv)
        self._tet_mat.append(mats)
        self._tt += int(valid.sum())
        return vol

    def add_tetrahedron(self, i, j, k, l, k_mu=1.0e3, k_lambda=1.0e3, k_damp=0.0):  # noqa: E741
        return float(self.add_tetrahedra([i], [j], [k], [l], k_mu, k_lambda, k_damp)[0])

    # -- bending hinges (builder.py:7966-8061)
    def add_edges(self, i, j, k, l, rest=None, edge_ke=None, edge_kd=None):  # noqa: E741
        i_, j_, k_, l_ = (np.asarray(a, dtype=np.int64) for a in (i, j, k, l))
        q = self.particle_q
        x3, x4 = q[k_], q[l_]
        n = len(i_)
        if rest is None:
            rest = np.zeros(n, dtype=np.float64)
            valid = (i_ != -1) & (j_ != -1)
            x1, x2 = q[i_[valid]], q[j_[valid]]
            x3v, x4v = x3[valid], x4[valid]

            def normalized(a):
                ln = np.linalg.norm(a, axis=-1, keepdims=True)
                ln[ln == 0] = 1.0
                return a / ln

            n1 = normalized(np.cross(x3v - x1, x4v - x1))
            n2 = normalized(np.cross(x4v - x2, x3v - x2))
            e = normalized(x4v - x3v)
            cos_t = np.clip((n1 * n2).sum(-1), -1.0, 1.0)
            sin_t = (np.cross(n1, n2) * e).sum(-1)
            rest[valid] = np.arctan2(sin_t, cos_t)
        ke = np.broadcast_to(np.asarray(self.default_edge_ke if edge_ke is None else edge_ke, dtype=np.float64), (n,))
        kd = np.broadcast_to(np.asarray(self.default_edge_kd if edge_kd is None else edge_kd, dtype=np.float64), (n,))
        self._edge.append(np.stack([i_, j_, k_, l_], axis=1).astype(np.int32))
        self._edge_angle.append(np.asarray(rest, dtype=np.float64))
        self._edge_len.append(np.linalg.norm(x4 - x3, axis=1))
        self._edge_prop.append(np.stack([ke, kd], axis=1))
        self._e += n

    # -- cloth (builder.py:8063-8341)
    def add_cloth_mesh(self, pos, rot, scale, vel, vertices, indices, density, tri_ke=None, tri_ka=None, tri_kd=None,
                       tri_drag=None, tri_lift=None, edge_ke=None, edge_kd=None, particle_radius=None):  # fmt: skip
        tri_ke = self.default_tri_ke if tri_ke is None else tri_ke
        tri_ka = self.default_tri_ka if tri_ka is None else tri_ka
        tri_kd = self.default_tri_kd if tri_kd is None else tri_kd
        tri_drag = self.default_tri_drag if tri_drag is None else tri_drag
        tri_lift = self.default_tri_lift if tri_lift is None else tri_lift
        edge_ke = self.default_edge_ke if edge_ke is None else edge_ke
        edge_kd = self.default_edge_kd if edge_kd is None else edge_kd
        radius = self.default_particle_radius if particle_radius is None else particle_radius
        verts = np.asarray(vertices, dtype=np.float64).reshape(-1, 3) * scale
        rot_m = quat_to_matrix(rot).astype(np.float32).astype(np.float64)
        verts3 = verts @ rot_m.T + np.asarray(pos, dtype=np.float64)
        nv = len(verts3)
        start = self.add_particles(verts3, vel, np.zeros(nv), radius=radius)
        inds = (start + np.asarray(indices, dtype=np.int64)).reshape(-1, 3)
        t0 = self._t
        areas = self.add_triangles(inds[:, 0], inds[:, 1], inds[:, 2], tri_ke, tri_ka, tri_kd, tri_drag, tri_lift)
        mass = self.particle_mass
        add = density * areas / 3.0
        for c in range(3):
            np.add.at(mass, inds[:, c], add)
        self._mass = [mass]
        tris = self.tri_indices[t0:self._t]
        hinges = mesh_hinges(tris)
        self.add_edges(hinges[:, 0], hinges[:, 1], hinges[:, 2], hinges[:, 3], edge_ke=edge_ke, edge_kd=edge_kd)

    def add_cloth_grid(self, pos, rot, vel, dim_x, dim_y, cell_x, cell_y, mass, reverse_winding=False,
                       fix_left=False, fix_right=False, fix_top=False, fix_bottom=False, tri_ke=None, tri_ka=None,
                       tri_kd=None, tri_drag=None, tri_lift=None, edge_ke=None, edge_kd=None, particle_radius=None):  # fmt: skip
        xs, ys = np.meshgrid(np.arange(dim_x + 1), np.arange(dim_y + 1))
        vertices = np.stack([xs.ravel() * cell_x, ys.ravel() * cell_y, np.zeros(xs.size)], axis=1)
        cx, cy = np.meshgrid(np.arange(1, dim_x + 1), np.arange(1, dim_y + 1))
        cx, cy = cx.ravel(), cy.ravel()
        w = dim_x + 1
        v0 = (cy - 1) * w + (cx - 1)
        v1 = (cy - 1) * w + cx
        v2 = cy * w + cx
        v3 = cy * w + (cx - 1)
        if reverse_winding:
            idx = np.stack([v0, v1, v2, v0, v2, v3], axis=1)
        else:
            idx = np.stack([v0, v1, v3, v1, v2, v3], axis=1)
        start = self._n
        total_mass = mass * (dim_x + 1) * (dim_x + 1)
        total_area = cell_x * cell_y * dim_x * dim_y
        density = total_mass / total_area
        self.add_cloth_mesh(pos, rot, 1.0, vel, vertices, idx.reshape(-1), density, tri_ke, tri_ka, tri_kd, tri_drag,
                            tri_lift, edge_ke, edge_kd, particle_radius)  # fmt: skip
        gx, gy = xs.ravel(), ys.ravel()
        fixed = (
            ((gx == 0) & fix_left) | ((gx == dim_x) & fix_right) | ((gy == 0) & fix_bottom) | ((gy == dim_y) & fix_top)
        )
        flags = self.particle_flags
        m = self.particle_mass
        sl = slice(start, start + len(gx))
        flags[sl] = np.where(fixed, flags[sl] & ~int(ParticleFlags.ACTIVE), int(ParticleFlags.ACTIVE))
        m[sl] = np.where(fixed, 0.0, mass)
        self._flags = [flags]
        self._mass = [m]

    # -- volumetric grid (builder.py:8445-8611)
    def add_soft_grid(self, pos, rot, vel, dim_x, dim_y, dim_z, cell_x, cell_y, cell_z, density, k_mu, k_lambda,
                      k_damp, fix_left=False, fix_right=False, fix_top=False, fix_bottom=False, tri_ke=0.0, tri_ka=0.0,
                      tri_kd=0.0, tri_drag=0.0, tri_lift=0.0, add_surface_mesh_edges=True, edge_ke=0.0, edge_kd=0.0,
                      particle_radius=None, label=None):  # fmt: skip
        """A box of dim_x x dim_y x dim_z cells, five tetrahedra per cell in the alternating pattern of the
        reference, its boundary faces as triangles (for contact; zero stiffness by default) and, with
        add_surface_mesh_edges, the hinges of that surface. Every particle gets the mass of one cell;
        fix_* set the mass of a side's particles to 0."""
        del label
        nx, ny, nz = dim_x + 1, dim_y + 1, dim_z + 1
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        xx, yy, zz = xx.ravel(), yy.ravel(), zz.ravel()
        local = np.stack([xx * cell_x, yy * cell_y, zz * cell_z], axis=1)
        rot_m = quat_to_matrix(rot).astype(np.float32).astype(np.float64)
        verts = local @ rot_m.T + np.asarray(pos, dtype=np.float64)
        m = np.full(len(xx), cell_x * cell_y * cell_z * density, dtype=np.float64)
        fixed = ((xx == 0) & fix_left) | ((xx == dim_x) & fix_right) | ((yy == dim_y) & fix_top) | ((yy == 0) & fix_bottom)
        m[fixed] = 0.0
        radius = self.default_particle_radius if particle_radius is None else particle_radius
        start = self.add_particles(verts, vel, m, radius=radius)

        def gi(x, y, z):
            return start + nx * ny * z + nx * y + x

        cz, cy, cx = np.meshgrid(np.arange(dim_z), np.arange(dim_y), np.arange(dim_x), indexing="ij")
        cx, cy, cz = cx.ravel(), cy.ravel(), cz.ravel()
        v = [gi(cx, cy, cz), gi(cx + 1, cy, cz), gi(cx + 1, cy, cz + 1), gi(cx, cy, cz + 1), gi(cx, cy + 1, cz),
             gi(cx + 1, cy + 1, cz), gi(cx + 1, cy + 1, cz + 1), gi(cx, cy + 1, cz + 1)]  # fmt: skip
        odd = ((cx & 1) ^ (cy & 1) ^ (cz & 1)).astype(bool)
        pat_odd = [(0, 1, 4, 3), (2, 3, 6, 1), (5, 4, 1, 6), (7, 6, 3, 4), (4, 1, 6, 3)]
        pat_even = [(1, 2, 5, 0), (3, 0, 7, 2), (4, 7, 0, 5), (6, 5, 2, 7), (5, 2, 7, 0)]
        tets = np.empty((len(cx), 5, 4), dtype=np.int64)
        for t in range(5):
            for c in range(4):
                tets[:, t, c] = np.where(odd, v[pat_odd[t][c]], v[pat_even[t][c]])
        tets = tets.reshape(-1, 4)
        self.add_tetrahedra(tets[:, 0], tets[:, 1], tets[:, 2], tets[:, 3], k_mu, k_lambda, k_damp)
        # boundary faces: the faces (i,k,j), (j,k,l), (i,j,l), (i,l,k) of every tet that no other tet shares,
        # in the order of their first appearance
        f = np.stack([tets[:, [0, 2, 1]], tets[:, [1, 2, 3]], tets[:, [0, 1, 3]], tets[:, [0, 3, 2]]], axis=1).reshape(-1, 3)
        if len(f):
            key = np.sort(f, axis=1)
            _, first, counts = np.unique(key, axis=0, return_index=True, return_counts=True)
            keep = np.sort(first[counts == 1])
            faces = f[keep]
            t0 = self._t
            self.add_triangles(faces[:, 0], faces[:, 1], faces[:, 2], tri_ke, tri_ka, tri_kd, tri_drag, tri_lift)
            if add_surface_mesh_edges and self._t > t0:
                h = mesh_hinges(self.tri_indices[t0:self._t])
                self.add_edges(h[:, 0], h[:, 1], h[:, 2], h[:, 3], edge_ke=edge_ke, edge_kd=edge_kd)

    # -- bodies (builder.py:3814-3878): rigid bodies that carry collision shapes
    def add_body(self, xform=None, armature=None, com=None, inertia=None, mass=0.0, label=None, lock_inertia=False,
                 is_kinematic=False, custom_attributes=None) -> int:  # fmt: skip
        """A rigid body at `xform` (world frame) that shapes can be attached to (``body=`` of the add_shape_*
        methods, their xform then in the body's frame). Its motion comes from another solver: the cloth step
        (``SolverVBD(..., integrate_with_external_rigid_solver=True)``) reads the bodies' transforms from
        ``state_in.body_q`` and ``state_out.body_q`` and moves particle contacts with them. The mass properties are
        kept as given; shapes added to the body do not change them (the reference adds their mass at the shape
        density unless ``lock_inertia``), since the cloth step reads none of them."""
        p, q = _xform(xform)
        self.bodies.append(dict(q=tuple(p) + tuple(q), com=tuple(float(v) for v in (com or (0.0, 0.0, 0.0))),
                                mass=float(mass),
                                inertia=np.zeros((3, 3)) if inertia is None else np.asarray(inertia, float).reshape(3, 3),
                                label=label, kinematic=bool(is_kinematic), world=self.current_world))  # fmt: skip
        return len(self.bodies) - 1

    # -- shapes (builder.py:5900-6470): collision shapes for particle contacts, static (body -1) or on a body
    def _add_shape(self, body, type_, xform, scale, cfg, src=None):
        body = int(body)
        if body < -1 or body >= len(self.bodies):
            raise ValueError(f"body {body} does not exist (add_body first, or -1 for a static shape)")
        cfg = cfg or self.default_shape_cfg
        p, q = _xform(xform)
        self.shapes.append(dict(type=GeoType(type_), pos=p, rot=q, scale=tuple(float(v) for v in scale), ke=cfg.ke,
                                kd=cfg.kd, mu=cfg.mu, body=body, src=src, world=self.current_world,
                                flags=4 if cfg.has_particle_collision else 0))  # fmt: skip
        return len(self.shapes) - 1

    def add_shape_plane(self, plane=(0.0, 0.0, 1.0, 0.0), xform=None, width=10.0, length=10.0, body=-1,
                        cfg: ShapeConfig | None = None):  # fmt: skip
        """A plane with normal along the local Z of xform, or from the equation a x + b y + c z + d = 0; width
        and length 0 make it infinite."""
        if xform is None:
            nrm = np.asarray(plane[:3], dtype=np.float64)
            ln = np.linalg.norm(nrm)
            nrm = nrm / ln
            pos = -(plane[3] / ln) * nrm
            xform = (tuple(pos), quat_between_vectors((0.0, 0.0, 1.0), nrm))
        return self._add_shape(body, GeoType.PLANE, xform, (width, length, 0.0), cfg)

    def add_ground_plane(self, height=0.0, cfg: ShapeConfig | None = None):
        return self.add_shape_plane(plane=(*self.up_vector, -height), width=0.0, length=0.0, cfg=cfg)

    def add_shape_sphere(self, body=-1, xform=None, radius=1.0, cfg: ShapeConfig | None = None):
        return self._add_shape(body, GeoType.SPHERE, xform, (radius, 0.0, 0.0), cfg)

    def add_shape_box(self, body=-1, xform=None, hx=0.5, hy=0.5, hz=0.5, cfg: ShapeConfig | None = None):
        return self._add_shape(body, GeoType.BOX, xform, (hx, hy, hz), cfg)

    def add_shape_capsule(self, body=-1, xform=None, radius=1.0, half_height=0.5, cfg: ShapeConfig | None = None):
        """Capsule along the local Z axis of xform."""
        return self._add_shape(body, GeoType.CAPSULE, xform, (radius, half_height, 0.0), cfg)

    def add_shape_cylinder(self, body=-1, xform=None, radius=1.0, half_height=0.5, cfg: ShapeConfig | None = None):
        """Cylinder along the local Z axis of xform."""
        return self._add_shape(body, GeoType.CYLINDER, xform, (radius, half_height, 0.0), cfg)

    def add_shape_ellipsoid(self, body=-1, xform=None, rx=1.0, ry=0.75, rz=0.5, cfg: ShapeConfig | None = None):
        return self._add_shape(body, GeoType.ELLIPSOID, xform, (rx, ry, rz), cfg)

    def add_shape_cone(self, body=-1, xform=None, radius=1.0, half_height=0.5, cfg: ShapeConfig | None = None):
        """Cone along the local Z axis of xform: base of the given radius at z = -half_height, apex at
        +half_height (``builder.py:6287-6340``)."""
        return self._add_shape(body, GeoType.CONE, xform, (radius, half_height, 0.0), cfg)

    def add_shape_mesh(self, body=-1, xform=None, mesh: Mesh | None = None, scale=None,
                       cfg: ShapeConfig | None = None):  # fmt: skip
        """A static triangle mesh (``builder.py:6341-6380``); scale defaults to (1, 1, 1)."""
        if mesh is None:
            raise ValueError("add_shape_mesh() requires a Mesh instance.")
        scale = (1.0, 1.0, 1.0) if scale is None else tuple(scale)
        return self._add_shape(body, GeoType.MESH, xform, scale, cfg, src=mesh)

    def add_shape_convex_hull(self, body=-1, xform=None, mesh: Mesh | None = None, scale=None,
                              cfg: ShapeConfig | None = None):  # fmt: skip
        """A static convex mesh (``builder.py:6382-6421``): the mesh given is taken as the hull."""
        if mesh is None:
            raise ValueError("add_shape_convex_hull() requires a Mesh instance.")
        scale = (1.0, 1.0, 1.0) if scale is None else tuple(scale)
        return self._add_shape(body, GeoType.CONVEX_MESH, xform, scale, cfg, src=mesh)

    def add_shape_heightfield(self, xform=None, heightfield: Heightfield | None = None, scale=None,
                              cfg: ShapeConfig | None = None):  # fmt: skip
        """A static heightfield (``builder.py:6423-6467``); scale (default (1, 1, 1)) multiplies hx, hy and
        min_z/max_z as the reference's finalize does."""
        if heightfield is None:
            raise ValueError("add_shape_heightfield() requires a Heightfield instance.")
        scale = (1.0, 1.0, 1.0) if scale is None else tuple(scale)
        return self._add_shape(-1, GeoType.HFIELD, xform, scale, cfg, src=heightfield)

    # -- coloring (builder.py:9304-9396)
    @property
    def particle_color_groups(self) -> list[np.ndarray]:
        return [g.array() for g in self._color_groups]

    @particle_color_groups.setter
    def particle_color_groups(self, groups):
        self._color_groups = [_ChunkedGroup([np.asarray(g, dtype=np.int32)], len(g)) for g in groups]

    def color(self, include_bending=False, balance_colors=True, target_max_min_color_ratio=1.1,
              coloring_algorithm=ColoringAlgorithm.MCS):  # fmt: skip
        self.particle_color_groups = color_particles(
            self._n, self.tri_indices, self.tri_materials, self.edge_indices, self.edge_bending_properties,
            include_bending, balance_colors, target_max_min_color_ratio, self.tet_indices, self.tet_materials,
            coloring_algorithm,
        )  # fmt: skip

    def set_coloring(self, groups):
        self.particle_color_groups = groups

    # -- worlds (builder.py:3038-3193)
    def add_world(self, builder: ModelBuilder):
        start = self._n
        self.world_particle_start.append(start)
        w = self.world_count
        self.world_count += 1
        n = builder._n
        if n:
            self._q.append(builder.particle_q)
            self._qd.append(builder._cat(builder._qd, (-1, 3), np.float64))
            self._mass.append(builder.particle_mass)
            self._radius.append(builder._cat(builder._radius, (-1,), np.float64))
            self._flags.append(builder.particle_flags)
            self._world.append(np.full(n, w, dtype=np.int32))
            self._n += n
        if builder._t:
            self._tri.append(builder.tri_indices + start)
            self._tri_pose.append(builder._cat(builder._tri_pose, (-1, 2, 2), np.float64))
            self._tri_mat.append(builder.tri_materials)
            self._tri_area.append(builder._cat(builder._tri_area, (-1,), np.float64))
            self._t += builder._t
        if builder._e:
            e = builder.edge_indices.copy()
            e[e >= 0] += start
            self._edge.append(e)
            self._edge_angle.append(builder._cat(builder._edge_angle, (-1,), np.float64))
            self._edge_len.append(builder._cat(builder._edge_len, (-1,), np.float64))
            self._edge_prop.append(builder.edge_bending_properties)
            self._e += builder._e
        if builder._s:
            self._spr.append(builder.spring_indices + start)
            self._spr_rest.append(builder._cat(builder._spr_rest, (-1,), np.float64))
            self._spr_ke.append(builder._cat(builder._spr_ke, (-1,), np.float64))
            self._spr_kd.append(builder._cat(builder._spr_kd, (-1,), np.float64))
            self._spr_ctl.append(builder._cat(builder._spr_ctl, (-1,), np.float64))
            self._s += builder._s
        if builder._tt:
            self._tet.append(builder.tet_indices + start)
            self._tet_pose.append(builder.tet_poses)
            self._tet_mat.append(builder.tet_materials)
            self._tt += builder._tt
        b0 = len(self.bodies)
        self.bodies.extend(dict(bd, world=w) for bd in builder.bodies)
        self.shapes.extend(dict(s, world=w, body=s["body"] + b0 if s["body"] >= 0 else -1) for s in builder.shapes)
        translated = [_ChunkedGroup([c + start for c in g.chunks], g.size) for g in builder._color_groups]
        self._color_groups = _merge_chunked(self._color_groups, translated)

    def finalize(self, device="cuda") -> Model:
        return Model._from_builder(self, device)


class Heightfield:
    """A 2D elevation grid (``newton/_src/geometry/types.py:2095-2142``): the data are normalized to [0, 1];
    heights are ``min_z + data (max_z - min_z)``, with min_z and max_z taken from the data unless both are given;
    the grid spans [-hx, hx] x [-hy, hy]."""

    def __init__(self, data, nrow: int, ncol: int, hx: float = 1.0, hy: float = 1.0, min_z: float | None = None,
                 max_z: float | None = None):  # fmt: skip
        if nrow < 2 or ncol < 2:
            raise ValueError(f"Heightfield requires nrow >= 2 and ncol >= 2, got nrow={nrow}, ncol={ncol}")
        if (min_z is None) != (max_z is None):
            raise ValueError("min_z and max_z must both be provided or both omitted")
        raw = np.array(data, dtype=np.float32).reshape(nrow, ncol)
        lo, hi = float(raw.min()), float(raw.max())
        self._data = (raw - lo) / (hi - lo) if hi > lo else np.zeros_like(raw)
        self.nrow, self.ncol = nrow, ncol
        self.hx, self.hy = hx, hy
        self.min_z = lo if min_z is None else float(min_z)
        self.max_z = hi if max_z is None else float(max_z)

    @property
    def data(self):
        """The normalized [0, 1] elevations, shape (nrow, ncol)."""
        return self._data


class Mesh:
    """A triangle mesh for collision (``newton/_src/geometry/types.py:131-190``, the collision part): vertices
    [V, 3] and triangle indices [T, 3] (or flat), counter-clockwise seen from outside."""

    def __init__(self, vertices, indices, normals=None, uvs=None, compute_inertia=True, is_solid=True, **_render):
        del normals, uvs, compute_inertia, _render
        self.vertices = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
        self.indices = np.asarray(indices, dtype=np.int32).reshape(-1)
        if len(self.indices) % 3 or (len(self.indices) and (self.indices.min() < 0 or
                                                            self.indices.max() >= len(self.vertices))):
            raise ValueError("Mesh indices must be triangles of vertex ids")
        self.is_solid = is_solid


class _DeviceMesh:
    """A mesh's hierarchy and pseudo-normals on the GPU (``vbd_mesh_create``), freed with the model."""

    def __init__(self, mesh: Mesh):
        self._lib = _lib.load()
        h = C.c_void_p()
        pts = np.ascontiguousarray(mesh.vertices, dtype=np.float32)
        idx = np.ascontiguousarray(mesh.indices, dtype=np.int32)
        rc = self._lib.vbd_mesh_create(pts.ctypes.data_as(C.POINTER(C.c_float)), len(pts),
                                       idx.ctypes.data_as(C.POINTER(C.c_int32)), len(idx) // 3, C.byref(h))  # fmt: skip
        _lib.check(rc, "vbd_mesh_create")
        self.handle = h.value

    def __del__(self):
        if getattr(self, "handle", None):
            self._lib.vbd_mesh_destroy(self.handle)
            self.handle = None


# ----------------------------------------------------------------------------- model, state, contacts
class Model:
    """Arrays of a finalized cloth model (the reference ``Model`` fields the VBD path reads)."""

    def __init__(self):
        self.device = None
        self.particle_count = self.tri_count = self.edge_count = self.shape_count = 0
        self.body_count = 0
        self.world_count = 1
        self.spring_count = 0
        self.tet_count = 0
        self.soft_contact_ke = 1.0e3
        self.soft_contact_kd = 10.0
        self.soft_contact_mu = 0.5
        self.soft_contact_margin = 0.01

    @staticmethod
    def _from_builder(b: ModelBuilder, device) -> Model:
        m = Model()
        dev = torch.device(device)
        m.device = dev

        def t(a, dtype):
            return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)

        f32, i32 = torch.float32, torch.int32
        m.particle_count, m.tri_count, m.edge_count = b._n, b._t, b._e
        mass = b.particle_mass
        m.particle_q = t(b.particle_q, f32).reshape(-1, 3)
        m.particle_qd = t(b._cat(b._qd, (-1, 3), np.float64), f32).reshape(-1, 3)
        m.particle_mass = t(mass, f32)
        m.particle_inv_mass = t(np.where(mass > 0.0, 1.0 / np.where(mass > 0.0, mass, 1.0), 0.0), f32)
        m.particle_radius = t(b._cat(b._radius, (-1,), np.float64), f32)
        m.particle_flags = t(b.particle_flags, i32)
        m.particle_world = t(b._cat(b._world, (-1,), np.int32), i32)
        m.tri_indices = t(b.tri_indices, i32).reshape(-1, 3)
        m.tri_poses = t(b._cat(b._tri_pose, (-1, 2, 2), np.float64), f32).reshape(-1, 2, 2)
        m.tri_materials = t(b.tri_materials, f32).reshape(-1, 5)
        m.tri_areas = t(b._cat(b._tri_area, (-1,), np.float64), f32)
        m.edge_indices = t(b.edge_indices, i32).reshape(-1, 4)
        m.edge_rest_angle = t(b._cat(b._edge_angle, (-1,), np.float64), f32)
        m.edge_rest_length = t(b._cat(b._edge_len, (-1,), np.float64), f32)
        m.edge_bending_properties = t(b.edge_bending_properties, f32).reshape(-1, 2)
        m.spring_count, m.tet_count = b._s, b._tt
        m.spring_indices = t(b.spring_indices, i32).reshape(-1)
        m.spring_rest_length = t(b._cat(b._spr_rest, (-1,), np.float64), f32)
        m.spring_stiffness = t(b._cat(b._spr_ke, (-1,), np.float64), f32)
        m.spring_damping = t(b._cat(b._spr_kd, (-1,), np.float64), f32)
        m.spring_control = t(b._cat(b._spr_ctl, (-1,), np.float64), f32)
        m.tet_indices = t(b.tet_indices, i32).reshape(-1, 4)
        m.tet_poses = t(b.tet_poses, f32).reshape(-1, 3, 3)
        m.tet_materials = t(b.tet_materials, f32).reshape(-1, 3)
        m.particle_color_groups = [t(g, i32) for g in b.particle_color_groups]
        colors = np.full(b._n, -1, dtype=np.int32)
        for c, g in enumerate(b.particle_color_groups):
            colors[np.asarray(g)] = c
        m.particle_colors = t(colors, i32)
        nw = max(b.world_count, 1)
        g = np.zeros((nw, 3))
        g[:, b.up_axis] = b.gravity
        m.gravity = t(g, f32)
        m.up_axis = b.up_axis
        m.world_count = nw
        m.world_particle_start = None
        if b.world_count > 1:
            m.world_particle_start = np.array(b.world_particle_start + [b._n], dtype=np.int32)
        m.shape_count = len(b.shapes)
        S = m.shape_count
        # host copies (the contact generator takes the shape table by value): GeoType, (p, q xyzw), scale
        m.shape_type = np.array([int(s["type"]) for s in b.shapes], dtype=np.int32)
        m.shape_transform = np.array([list(s["pos"]) + list(s["rot"]) for s in b.shapes], dtype=np.float32).reshape(S, 7)
        m.shape_scale = np.array([s["scale"] for s in b.shapes], dtype=np.float32).reshape(S, 3)
        m.shape_material_ke = t(np.array([s["ke"] for s in b.shapes]).reshape(S), f32)
        m.shape_material_kd = t(np.array([s["kd"] for s in b.shapes]).reshape(S), f32)
        m.shape_material_mu = t(np.array([s["mu"] for s in b.shapes]).reshape(S), f32)
        m.shape_body = t(np.array([s["body"] for s in b.shapes], dtype=np.int32).reshape(S), i32)
        # ShapeFlags COLLIDE_PARTICLES (1 << 2) and world indices (-1 = global), builder.py:417, 3288, 5866
        m.shape_flags = np.array([s.get("flags", 4) for s in b.shapes], dtype=np.int32).reshape(S)
        m.shape_world = np.array([s.get("world", -1) for s in b.shapes], dtype=np.int32).reshape(S)
        # heightfields as the reference's finalize packs them (builder.py:10690-10735): one row (data_offset, nrow,
        # ncol, |hx sx|, |hy sy|, min_z sz, max_z sz) per heightfield shape, elevations concatenated
        m.shape_heightfield_index = np.full(S, -1, dtype=np.int32)
        rows, chunks, off = [], [], 0
        for i, sh in enumerate(b.shapes):
            if sh["type"] == GeoType.HFIELD and sh.get("src") is not None:
                hf, (sx, sy, sz) = sh["src"], sh["scale"]
                m.shape_heightfield_index[i] = len(rows)
                rows.append((off, hf.nrow, hf.ncol, abs(hf.hx * sx), abs(hf.hy * sy), hf.min_z * sz, hf.max_z * sz))
                chunks.append(np.asarray(hf.data, dtype=np.float32).reshape(-1))
                off += hf.nrow * hf.ncol
        m.heightfield_data = np.array(rows, dtype=np.float64).reshape(-1, 7)
        m.heightfield_elevations = t(np.concatenate(chunks) if chunks else np.zeros(1, np.float32), f32)
        # triangle meshes: one device hierarchy per distinct Mesh (the reference's Mesh.finalize, one wp.Mesh each)
        m.shape_mesh_index = np.full(S, -1, dtype=np.int32)
        m.meshes, m._device_meshes, seen = [], [], {}
        for i, sh in enumerate(b.shapes):
            if sh["type"] in (GeoType.MESH, GeoType.CONVEX_MESH) and sh.get("src") is not None:
                key = id(sh["src"])
                if key not in seen:
                    seen[key] = len(m.meshes)
                    m.meshes.append(sh["src"])
                    if dev.type == "cuda":
                        m._device_meshes.append(_DeviceMesh(sh["src"]))
                m.shape_mesh_index[i] = seen[key]
        # bodies (model.py body_q / body_qd / body_com ...): transforms (p, q xyzw) and spatial velocities (v, w)
        B = len(b.bodies)
        m.body_count = B
        m._shape_body_host = np.array([s["body"] for s in b.shapes], dtype=np.int32).reshape(S)
        if B:
            m.body_q = t(np.array([bd["q"] for bd in b.bodies], dtype=np.float64).reshape(B, 7), f32)
            m.body_qd = torch.zeros((B, 6), dtype=torch.float32, device=dev)
            m.body_com = t(np.array([bd["com"] for bd in b.bodies], dtype=np.float64).reshape(B, 3), f32)
            m.body_mass = t(np.array([bd["mass"] for bd in b.bodies]).reshape(B), f32)
            m.body_inertia = t(np.stack([bd["inertia"] for bd in b.bodies]).reshape(B, 3, 3), f32)
            m.body_world = t(np.array([bd["world"] for bd in b.bodies], dtype=np.int32).reshape(B), i32)
            m.body_label = [bd["label"] for bd in b.bodies]
        else:
            m.body_q = m.body_qd = m.body_com = None
        m._shape_set = _ShapeSet(m) if dev.type == "cuda" and S > 0 else None
        return m

    def refresh_shapes(self):
        """Rebuild the GPU shape set from the host shape arrays (shape_transform, shape_scale, shape_type,
        shape_flags, shape_world, heightfields) now. Contact generation also does so by itself at its next call
        when those arrays changed; a CUDA graph keeps the shapes of its capture."""
        if self.device.type == "cuda" and self.shape_count > 0:
            if self._shape_set is not None:
                self._shape_set.fingerprint = None
            _current_shape_set(self)

    def set_gravity(self, gravity, world=None):
        g = torch.as_tensor(gravity, dtype=torch.float32, device=self.device).reshape(-1, 3)
        if world is None:
            self.gravity[:] = g
        else:
            self.gravity[world] = g[0]

    def state(self, requires_grad=None) -> State:
        s = State()
        s.particle_q = self.particle_q.clone()
        s.particle_qd = self.particle_qd.clone()
        s.particle_f = torch.zeros_like(self.particle_q)
        if self.body_count:
            s.body_q = self.body_q.clone()
            s.body_qd = self.body_qd.clone()
            s.body_f = torch.zeros_like(self.body_qd)
        return s

    def control(self, requires_grad=None, clone_variables=True) -> Control:
        return Control()

    def contacts(self, soft_contact_max=None) -> Contacts:
        return Contacts(self.particle_count * max(self.shape_count, 1) if soft_contact_max is None else soft_contact_max,
                        self.device)

    def collide(self, state: State, contacts: Contacts | None = None, soft_contact_margin=None):
        contacts = contacts or self.contacts()
        margin = self.soft_contact_margin if soft_contact_margin is None else soft_contact_margin
        soft_contacts(self, state, contacts, margin)
        return contacts


class State:
    """``newton/_src/sim/state.py:47`` (particle part)."""

    def __init__(self):
        self.particle_q = None
        self.particle_qd = None
        self.particle_f = None
        self.body_q = None
        self.body_qd = None
        self.body_f = None

    @property
    def particle_count(self):
        return 0 if self.particle_q is None else self.particle_q.shape[0]

    def clear_forces(self):
        if self.particle_f is not None:
            self.particle_f.zero_()

    def assign(self, other: State):
        for k in ("particle_q", "particle_qd", "particle_f", "body_q", "body_qd", "body_f"):
            a, b = getattr(self, k), getattr(other, k)
            if a is not None and b is not None:
                a.copy_(b)


class Control:
    pass


class Contacts:
    """Particle-shape soft contacts (``newton/_src/sim/contacts.py:268-295``)."""

    def __init__(self, soft_contact_max: int, device):
        n = int(soft_contact_max)
        dev = torch.device(device)
        self.soft_contact_max = n
        self.soft_contact_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.soft_contact_particle = torch.full((n,), -1, dtype=torch.int32, device=dev)
        self.soft_contact_shape = torch.full((n,), -1, dtype=torch.int32, device=dev)
        self.soft_contact_body_pos = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.soft_contact_body_vel = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.soft_contact_normal = torch.zeros((n, 3), dtype=torch.float32, device=dev)

    def clear(self):
        self.soft_contact_count.zero_()


def _shape_table(model: Model):
    """The model's shapes as a ``VbdShapeTable`` (the reference Model's layout), with the host arrays it points to."""
    S = model.shape_count
    ip, fp = C.POINTER(C.c_int32), C.POINTER(C.c_float)
    keep = dict(
        st=np.ascontiguousarray(model.shape_type, dtype=np.int32),
        sx=np.ascontiguousarray(model.shape_transform, dtype=np.float32),
        ss=np.ascontiguousarray(model.shape_scale, dtype=np.float32),
        hidx=np.ascontiguousarray(getattr(model, "shape_heightfield_index", np.full(S, -1)), dtype=np.int32),
        sfl=np.ascontiguousarray(getattr(model, "shape_flags", np.full(S, 4)), dtype=np.int32),
        swl=np.ascontiguousarray(getattr(model, "shape_world", np.full(S, -1)), dtype=np.int32),
        sbd=np.ascontiguousarray(getattr(model, "_shape_body_host", np.full(S, -1)), dtype=np.int32),
    )  # fmt: skip
    rows = getattr(model, "heightfield_data", np.zeros((0, 7)))
    keep["hfs"] = hfs = (_lib.VbdHeightfield * max(len(rows), 1))()
    for k, r in enumerate(rows):
        hfs[k] = _lib.VbdHeightfield(int(r[0]), int(r[1]), int(r[2]), *(float(v) for v in r[3:]))
    elev = getattr(model, "heightfield_elevations", None)
    midx = getattr(model, "shape_mesh_index", np.full(S, -1))
    dmeshes = getattr(model, "_device_meshes", [])
    keep["handles"] = handles = (C.c_void_p * max(S, 1))(*[dmeshes[k].handle if k >= 0 else None for k in midx])
    tb = _lib.VbdShapeTable(
        S, keep["st"].ctypes.data_as(ip), keep["sx"].ctypes.data_as(fp), keep["ss"].ctypes.data_as(fp),
        keep["hidx"].ctypes.data_as(ip), len(rows), hfs, None if elev is None else elev.data_ptr(),
        0 if elev is None else elev.numel(), C.cast(handles, C.POINTER(C.c_void_p)), keep["sfl"].ctypes.data_as(ip),
        keep["swl"].ctypes.data_as(ip), None, keep["sbd"].ctypes.data_as(ip), int(getattr(model, "body_count", 0)),
        None,
    )  # fmt: skip
    return tb, keep


_SHAPE_FIELDS = ("shape_type", "shape_transform", "shape_scale", "shape_flags", "shape_world", "shape_heightfield_index",
                 "heightfield_data", "shape_mesh_index", "_shape_body_host")  # fmt: skip


def _shape_fingerprint(model: Model):
    """A cheap digest of the host shape arrays a shape set is built from, and of the elevation array's address
    (its contents are read on the device at every launch, so in-place edits need no rebuild)."""
    parts = []
    for k in _SHAPE_FIELDS:
        a = getattr(model, k, None)
        parts.append(None if a is None else (np.asarray(a).dtype.str, np.asarray(a).shape,
                                             np.ascontiguousarray(a).tobytes()))  # fmt: skip
    elev = getattr(model, "heightfield_elevations", None)
    return hash(tuple(parts)), None if elev is None else elev.data_ptr()


class _ShapeSet:
    """The model's shapes on the GPU (``vbd_shape_set_create``), built at finalize and rebuilt when the host shape
    arrays change; freed with the model."""

    def __init__(self, model: Model):
        self._lib = _lib.load()
        self.fingerprint = _shape_fingerprint(model)
        tb, keep = _shape_table(model)
        h = C.c_void_p()
        with torch.cuda.device(model.device):
            _lib.check(self._lib.vbd_shape_set_create(C.byref(tb), C.byref(h)), "vbd_shape_set_create")
        self.handle = h.value
        self.device = model.device
        del keep

    def use_parameter_table(self, enable: bool):
        """Sets of up to 16 shapes launch with their records as a kernel parameter (default); False sends every
        size through the global-memory kernel. Both give the same contacts."""
        _lib.check(self._lib.vbd_shape_set_use_parameter_table(self.handle, int(bool(enable))),
                   "vbd_shape_set_use_parameter_table")  # fmt: skip

    def __del__(self):
        if getattr(self, "handle", None):
            try:
                with torch.cuda.device(self.device):
                    self._lib.vbd_shape_set_destroy(self.handle)
            except Exception:
                pass
            self.handle = None


def _current_shape_set(model: Model) -> _ShapeSet:
    """The model's shape set, rebuilt first when the host shape arrays (shape_transform, shape_scale, shape_type,
    shape_flags, shape_world, heightfields) changed since it was built, as the reference reads the model's arrays
    at every create_soft_contacts launch. A replaced set is kept until the model is freed: a CUDA graph captured
    before the change may still read it (the graph keeps the shapes of its capture; capture again after an edit)."""
    ss = getattr(model, "_shape_set", None)
    if ss is None or ss.fingerprint != _shape_fingerprint(model):
        if ss is not None:
            model._retired_shape_sets = getattr(model, "_retired_shape_sets", []) + [ss]
        model._shape_set = ss = _ShapeSet(model)
    return ss


def soft_contacts(model: Model, state: State, contacts: Contacts, margin: float):
    """Particle contacts against the model's shapes on the GPU (``vbd_soft_contacts_set``): any number of shapes;
    a particle of world w meets the global shapes and world w's; shapes on bodies move with ``state.body_q``. Edits
    of the host shape arrays after finalize take effect at the next call."""
    lib = _lib.load()
    if model.shape_count == 0:
        contacts.soft_contact_count.zero_()
        return
    ss = _current_shape_set(model)
    pw = getattr(model, "particle_world", None)
    bq = None
    if getattr(model, "body_count", 0) and bool(np.any(getattr(model, "_shape_body_host", np.zeros(0)) >= 0)):
        if getattr(state, "body_q", None) is None:
            raise ValueError("the model has shapes on bodies: state.body_q must hold the body transforms")
        bq = interop.pointer(state.body_q, "state.body_q", interop.F32, 7 * model.body_count)
    stream = torch.cuda.current_stream(model.device).cuda_stream
    with torch.cuda.device(model.device):
        rc = lib.vbd_soft_contacts_set(
            ss.handle, model.particle_count, state.particle_q.data_ptr(), model.particle_radius.data_ptr(),
            model.particle_flags.data_ptr(), None if pw is None else pw.data_ptr(), bq, float(margin),
            contacts.soft_contact_max, contacts.soft_contact_count.data_ptr(), contacts.soft_contact_particle.data_ptr(),
            contacts.soft_contact_shape.data_ptr(), contacts.soft_contact_body_pos.data_ptr(),
            contacts.soft_contact_body_vel.data_ptr(), contacts.soft_contact_normal.data_ptr(), C.c_void_p(stream),
        )  # fmt: skip
    _lib.check(rc, "vbd_soft_contacts_set")


class CollisionPipeline:
    """Particle-shape part of ``newton/_src/sim/collide.py:485`` (static planes, heightfields, spheres, boxes,
    capsules, cylinders, cones, ellipsoids and triangle meshes)."""

    def __init__(self, model: Model, soft_contact_max=None, soft_contact_margin=0.01, **_ignored):
        self.model = model
        self.soft_contact_margin = soft_contact_margin
        self.soft_contact_max = (model.particle_count * max(model.shape_count, 1) if soft_contact_max is None
                                 else soft_contact_max)  # fmt: skip

    def contacts(self) -> Contacts:
        return Contacts(self.soft_contact_max, self.model.device)

    def collide(self, state: State, contacts: Contacts):
        soft_contacts(self.model, state, contacts, self.soft_contact_margin)
