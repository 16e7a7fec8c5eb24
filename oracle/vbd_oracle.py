"""ctypes wrapper of the CPU oracle (``oracle/vbd_oracle.cpp``). TEST INFRASTRUCTURE ONLY.

Imported by ``tests/``, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
``bench.py``; never by the product package. Arrays are numpy; the model is a dict with the
reference ``Model`` field names (``particle_mass``, ``tri_poses`` …) plus the solver-side
adjacency (``adj_*``) and coloring (``color_offsets``, ``color_particles``, ``particle_colors``).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libvbd_oracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OracleModel(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("T", C.c_int), ("E", C.c_int), ("C", C.c_int), ("S", C.c_int),
        ("mass", _dp), ("inv_mass", _dp), ("radius", _dp), ("flags", _ip),
        ("tri_indices", _ip), ("tri_poses", _dp), ("tri_materials", _dp), ("tri_areas", _dp),
        ("edge_indices", _ip), ("edge_rest_angle", _dp), ("edge_rest_length", _dp), ("edge_bending_properties", _dp),
        ("adj_face_offsets", _ip), ("adj_faces", _ip), ("adj_edge_offsets", _ip), ("adj_edges", _ip),
        ("color_offsets", _ip), ("color_particles", _ip), ("particle_colors", _ip),
        ("gravity", _dp), ("soft_ke", C.c_double), ("soft_kd", C.c_double), ("soft_mu", C.c_double),
        ("shape_ke", _dp), ("shape_kd", _dp), ("shape_mu", _dp),
        ("friction_epsilon", C.c_double), ("beta", C.c_double),
    ]  # fmt: skip


class OracleContacts(C.Structure):
    _fields_ = [
        ("count", C.c_int), ("max", C.c_int), ("particle", _ip), ("shape", _ip),
        ("body_pos", _dp), ("body_vel", _dp), ("normal", _dp),
    ]  # fmt: skip


def build() -> str:
    """Compile the oracle library with ``make`` (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.oracle_vbd_step.argtypes = [
            C.POINTER(OracleModel), _dp, _dp, _dp, C.POINTER(OracleContacts), C.c_double, C.c_int, _dp, _dp, C.c_int,
            C.c_int,
        ]  # fmt: skip
        _lib.oracle_membrane.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp] + [C.c_double] * 5 + [_dp]
        _lib.oracle_bending.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int] + [C.c_double] * 5 + [_dp]
        _lib.oracle_contact.argtypes = [C.c_int, C.c_double, _dp, _dp] + [C.c_double] * 5 + [_dp]
        _lib.oracle_build_adjacency.argtypes = [C.c_int, C.c_int, _ip, C.c_int, _ip, _ip, _ip, _ip, _ip]
        _lib.oracle_soft_contacts.argtypes = [
            C.c_int, _dp, _dp, _ip, C.c_int, _ip, _dp, _dp, C.c_double, C.c_int, _ip, _ip, _dp, _dp, _dp,
        ]  # fmt: skip
        _lib.oracle_max_threads.restype = C.c_int
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def build_adjacency(n, tri_indices, edge_indices):
    """Vertex→(element, order) CSR in the reference's fill order; offsets count 2 ints per entry."""
    tri, tp = _i(np.asarray(tri_indices).reshape(-1, 3))
    edg, ep = _i(np.asarray(edge_indices).reshape(-1, 4))
    fo, fop = _i(np.zeros(n + 1))
    fa, fap = _i(np.zeros(max(6 * len(tri), 1)))
    eo, eop = _i(np.zeros(n + 1))
    ea, eap = _i(np.zeros(max(8 * len(edg), 1)))
    lib().oracle_build_adjacency(n, len(tri), tp, len(edg), ep, fop, fap, eop, eap)
    return fo, fa[: fo[-1]].copy(), eo, ea[: eo[-1]].copy()


class Model:
    """Keeps the numpy arrays alive and exposes them as an ``OracleModel`` struct."""

    def __init__(self, m: dict):
        self._keep = []

        def d(k, shape=None):
            a, p = _d(m[k] if shape is None else np.asarray(m[k]).reshape(shape))
            self._keep.append(a)
            return p

        def i(k, shape=None):
            a, p = _i(m[k] if shape is None else np.asarray(m[k]).reshape(shape))
            self._keep.append(a)
            return p

        shapes = np.asarray(m.get("shapes", np.zeros((0, 3))), dtype=np.float64).reshape(-1, 3)
        if len(shapes) == 0:
            shapes = np.zeros((1, 3))
        sk, skp = _d(shapes[:, 0])
        skd, skdp = _d(shapes[:, 1])
        smu, smup = _d(shapes[:, 2])
        self._keep += [sk, skd, smu]
        soft = np.asarray(m.get("soft", (1.0e3, 10.0, 0.5)), dtype=np.float64)
        self.n = len(np.asarray(m["particle_mass"]))
        self.s = OracleModel(
            n=self.n, T=len(np.asarray(m["tri_indices"]).reshape(-1, 3)),
            E=len(np.asarray(m["edge_indices"]).reshape(-1, 4)), C=len(m["color_offsets"]) - 1, S=len(shapes),
            mass=d("particle_mass"), inv_mass=d("particle_inv_mass"), radius=d("particle_radius"),
            flags=i("particle_flags"), tri_indices=i("tri_indices", (-1,)), tri_poses=d("tri_poses", (-1,)),
            tri_materials=d("tri_materials", (-1,)), tri_areas=d("tri_areas"), edge_indices=i("edge_indices", (-1,)),
            edge_rest_angle=d("edge_rest_angle"), edge_rest_length=d("edge_rest_length"),
            edge_bending_properties=d("edge_bending_properties", (-1,)), adj_face_offsets=i("adj_face_offsets"),
            adj_faces=i("adj_faces"), adj_edge_offsets=i("adj_edge_offsets"), adj_edges=i("adj_edges"),
            color_offsets=i("color_offsets"), color_particles=i("color_particles"),
            particle_colors=i("particle_colors"), gravity=d("gravity", (-1,)), soft_ke=soft[0], soft_kd=soft[1],
            soft_mu=soft[2], shape_ke=skp, shape_kd=skdp, shape_mu=smup,
            friction_epsilon=float(m.get("friction_epsilon", 1e-2)), beta=float(m.get("beta", 0.0)),
        )  # fmt: skip


def make_contacts(count, particle, shape, body_pos, body_vel, normal):
    keep = []
    p, pp = _i(particle)
    s, sp = _i(shape)
    bp, bpp = _d(np.asarray(body_pos).reshape(-1))
    bv, bvp = _d(np.asarray(body_vel).reshape(-1))
    nn, nnp = _d(np.asarray(normal).reshape(-1))
    keep += [p, s, bp, bv, nn]
    c = OracleContacts(count=int(count), max=len(p), particle=pp, shape=sp, body_pos=bpp, body_vel=bvp, normal=nnp)
    return c, keep


def step(model: Model, q_in, qd_in, f_ext, contacts=None, dt=1.0 / 600.0, iterations=10, precision=64, nthreads=1):
    """One VBD step. Returns (q_in_after, q_out, qd_out), mirroring the reference's state side effects."""
    n = model.n
    q, qp = _d(np.array(q_in, dtype=np.float64).reshape(-1))
    qd, qdp = _d(np.asarray(qd_in).reshape(-1))
    f, fp = _d(np.zeros(3 * n) if f_ext is None else np.asarray(f_ext).reshape(-1))
    qo, qop = _d(np.zeros(3 * n))
    vo, vop = _d(np.zeros(3 * n))
    if contacts is None:
        contacts = make_contacts(0, np.zeros(1), np.zeros(1), np.zeros(3), np.zeros(3), np.zeros(3))
    c, _keep = contacts
    rc = lib().oracle_vbd_step(C.byref(model.s), qp, qdp, fp, C.byref(c), dt, iterations, qop, vop, precision, nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle_vbd_step failed: {rc}")
    return q.reshape(-1, 3), qo.reshape(-1, 3), vo.reshape(-1, 3)


def soft_contacts(q, radius, flags, shape_type, shape_pos, shape_radius, margin, max_contacts=None):
    """Particle-shape contacts for static planes (type 0) and spheres (type 1), in (particle, shape) order."""
    n = len(radius)
    S = len(shape_type)
    max_contacts = max_contacts or n * max(S, 1)
    qq, qp = _d(np.asarray(q).reshape(-1))
    r, rp = _d(radius)
    fl, flp = _i(flags)
    st, stp = _i(shape_type)
    sp_, spp = _d(np.asarray(shape_pos).reshape(-1))
    sr, srp = _d(shape_radius)
    part, pp = _i(-np.ones(max_contacts))
    shp, shpp = _i(-np.ones(max_contacts))
    bp, bpp = _d(np.zeros(3 * max_contacts))
    bv, bvp = _d(np.zeros(3 * max_contacts))
    nn, nnp = _d(np.zeros(3 * max_contacts))
    cnt = lib().oracle_soft_contacts(n, qp, rp, flp, S, stp, spp, srp, margin, max_contacts, pp, shpp, bpp, bvp, nnp)
    return cnt, part, shp, bp.reshape(-1, 3), bv.reshape(-1, 3), nn.reshape(-1, 3)


def element(kind, precision, *args):
    out, op = _d(np.zeros(12))
    if kind == "membrane":
        order, x, xp, pose, area, mu, lmbd, damping, dt = args
        x_, xp_p = _d(x)
        xp_, xpp = _d(xp)
        po, pop = _d(pose)
        lib().oracle_membrane(precision, int(order), xp_p, xpp, pop, area, mu, lmbd, damping, dt, op)
    elif kind == "bending":
        order, x, xp, boundary, rest_angle, rest_len, ke, kd, dt = args
        x_, xp_p = _d(x)
        xp_, xpp = _d(xp)
        lib().oracle_bending(precision, int(order), xp_p, xpp, int(boundary), rest_angle, rest_len, ke, kd, dt, op)
    elif kind == "contact":
        pen, n, rel, ke, kd, mu, eps, dt = args
        n_, npp = _d(n)
        r_, rp = _d(rel)
        lib().oracle_contact(precision, pen, npp, rp, ke, kd, mu, eps, dt, op)
    else:
        raise ValueError(kind)
    return out[:3].copy(), out[3:].reshape(3, 3).copy()
