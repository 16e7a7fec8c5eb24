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
        ("spring_count", C.c_int), ("spring_indices", _ip), ("spring_rest_length", _dp), ("spring_stiffness", _dp),
        ("spring_damping", _dp), ("tet_count", C.c_int), ("tet_indices", _ip), ("tet_poses", _dp),
        ("tet_materials", _dp), ("adj_tet_offsets", _ip), ("adj_tets", _ip),
    ]  # fmt: skip


class OracleContacts(C.Structure):
    _fields_ = [
        ("count", C.c_int), ("max", C.c_int), ("particle", _ip), ("shape", _ip),
        ("body_pos", _dp), ("body_vel", _dp), ("normal", _dp), ("shape_body", _ip), ("body_q", _dp),
        ("body_q_prev", _dp), ("body_qd", _dp), ("body_com", _dp),
    ]  # fmt: skip


class OracleSelfContact(C.Structure):
    _fields_ = [
        ("radius", C.c_double), ("margin", C.c_double), ("relaxation", C.c_double),
        ("edge_parallel_epsilon", C.c_double), ("rest_exclusion", C.c_double), ("vertex_buffer", C.c_int),
        ("edge_buffer", C.c_int), ("interval", C.c_int), ("rest_q", _dp), ("vt_filter_offsets", _ip),
        ("vt_filter", _ip), ("ee_filter_offsets", _ip), ("ee_filter", _ip), ("brute_force", C.c_int),
    ]  # fmt: skip


class SelfContact:
    """Self-contact settings with the ``SolverVBD`` keyword meanings (``solver_vbd.py:204-216``).
    ``vt_filter`` / ``ee_filter`` are (flat, offsets) CSR lists of filtered triangles per vertex and
    filtered edges per edge, each row sorted, or None. ``brute_force`` tests every primitive pair in
    the detection instead of the candidates of a box grid (the same pairs, slower)."""

    def __init__(self, rest_q, *, radius, margin, relaxation=0.85, vertex_buffer=32, edge_buffer=64, interval=0,
                 edge_parallel_epsilon=1e-5, rest_exclusion=0.0, vt_filter=None, ee_filter=None,
                 brute_force=False):  # fmt: skip
        self._keep = []

        def ints(a):
            if a is None:
                return None
            arr, ptr = _i(a)
            self._keep.append(arr)
            return ptr

        rq, rqp = _d(np.asarray(rest_q).reshape(-1))
        self._keep.append(rq)
        vf, vfo = vt_filter if vt_filter is not None else (None, None)
        ef, efo = ee_filter if ee_filter is not None else (None, None)
        self.vertex_buffer, self.edge_buffer = int(vertex_buffer), int(edge_buffer)
        self.s = OracleSelfContact(
            radius=radius, margin=margin, relaxation=relaxation, edge_parallel_epsilon=edge_parallel_epsilon,
            rest_exclusion=rest_exclusion, vertex_buffer=self.vertex_buffer, edge_buffer=self.edge_buffer,
            interval=int(interval), rest_q=rqp, vt_filter_offsets=ints(vfo), vt_filter=ints(vf),
            ee_filter_offsets=ints(efo), ee_filter=ints(ef), brute_force=int(bool(brute_force)),
        )  # fmt: skip


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
        ]
        _lib.oracle_soft_contacts_shapes.argtypes = [
            C.c_int, _dp, _dp, _ip, C.c_int, _ip, _dp, _dp, _ip, _ip, _dp, _dp, _ip, _ip, _ip, _dp, _ip, _ip, _ip, _ip,
            C.c_double, C.c_int, _ip, _ip, _dp, _dp, _dp, _ip, _dp,
        ]  # fmt: skip
        _lib.oracle_max_threads.restype = C.c_int
        _lib.oracle_vbd_step_sc.argtypes = [
            C.POINTER(OracleModel), _dp, _dp, _dp, C.POINTER(OracleContacts), C.POINTER(OracleSelfContact), C.c_double,
            C.c_int, _dp, _dp, C.c_int, C.c_int,
        ]  # fmt: skip
        _lib.oracle_collide.argtypes = [
            C.POINTER(OracleModel), C.POINTER(OracleSelfContact), _dp, C.c_int, _ip, _ip, _dp, _ip, _ip, _dp, _ip, C.c_int,
        ]  # fmt: skip
        _lib.oracle_sc_vt.argtypes = [C.c_int, _dp, _dp] + [C.c_double] * 6 + [_dp]
        _lib.oracle_sc_ee.argtypes = [C.c_int, _dp, _dp] + [C.c_double] * 7 + [_dp]
        _lib.oracle_sc_plane.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double, _dp]
        _lib.oracle_tri_closest.argtypes = [_dp, _dp]
        _lib.oracle_edge_closest.argtypes = [_dp, C.c_double, _dp]
        _lib.oracle_sc_norm.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        _lib.oracle_tet.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp] + [C.c_double] * 4 + [_dp]
        _lib.oracle_spring.argtypes = [C.c_int, _dp, _dp] + [C.c_double] * 4 + [_dp]
        _lib.oracle_build_tet_adjacency.argtypes = [C.c_int, C.c_int, _ip, _ip, _ip]
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def build_tet_adjacency(n, tet_indices):
    """Vertex→(tet, order) CSR in the reference's fill order; offsets count 2 ints per entry."""
    tet, tp = _i(np.asarray(tet_indices).reshape(-1, 4))
    to, top = _i(np.zeros(n + 1))
    ta, tap = _i(np.zeros(max(8 * len(tet), 1)))
    lib().oracle_build_tet_adjacency(n, len(tet), tp, top, tap)
    return to, ta[: to[-1]].copy()


def tet_element(precision, order, x, xp, Dinv, mu, lmbd, damping, dt):
    x_, xp_p = _d(np.asarray(x).reshape(-1))
    p_, pp = _d(np.asarray(xp).reshape(-1))
    D_, dp = _d(np.asarray(Dinv).reshape(-1))
    out, op = _d(np.zeros(12))
    lib().oracle_tet(precision, int(order), xp_p, pp, dp, mu, lmbd, damping, dt, op)
    return out[:3].copy(), out[3:].reshape(3, 3).copy()


def spring_element(precision, x, xa, rest, ke, kd, dt):
    x_, xp_ = _d(np.asarray(x).reshape(-1))
    a_, ap = _d(np.asarray(xa).reshape(-1))
    out, op = _d(np.zeros(15))
    lib().oracle_spring(precision, xp_, ap, rest, ke, kd, dt, op)
    return out[:3].copy(), out[3:6].copy(), out[6:].reshape(3, 3).copy()


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
        ns = len(np.asarray(m.get("spring_rest_length", ())))
        if ns:
            self.s.spring_count = ns
            self.s.spring_indices = i("spring_indices", (-1,))
            self.s.spring_rest_length = d("spring_rest_length")
            self.s.spring_stiffness = d("spring_stiffness")
            self.s.spring_damping = d("spring_damping")
        nt = len(np.asarray(m.get("tet_indices", np.zeros((0, 4)))).reshape(-1, 4))
        if nt:
            if "adj_tet_offsets" not in m:
                m = dict(m)
                m["adj_tet_offsets"], m["adj_tets"] = build_tet_adjacency(self.n, m["tet_indices"])
            self.s.tet_count = nt
            self.s.tet_indices = i("tet_indices", (-1,))
            self.s.tet_poses = d("tet_poses", (-1,))
            self.s.tet_materials = d("tet_materials", (-1,))
            self.s.adj_tet_offsets = i("adj_tet_offsets")
            self.s.adj_tets = i("adj_tets")


def make_contacts(count, particle, shape, body_pos, body_vel, normal, shape_body=None, body_q=None, body_q_prev=None,
                  body_qd=None, body_com=None):  # fmt: skip
    """Contacts for ``step``. With shapes on bodies: ``shape_body`` [S] (-1 = static) and the body arrays the step
    reads (``body_q`` [B,7], ``body_q_prev`` [B,7] or None, ``body_qd`` [B,6], ``body_com`` [B,3]); contact
    points are then in the body's frame."""
    keep = []
    p, pp = _i(particle)
    s, sp = _i(shape)
    bp, bpp = _d(np.asarray(body_pos).reshape(-1))
    bv, bvp = _d(np.asarray(body_vel).reshape(-1))
    nn, nnp = _d(np.asarray(normal).reshape(-1))
    keep += [p, s, bp, bv, nn]
    extra = {}
    if shape_body is not None and body_q is not None:
        a, ap = _i(shape_body)
        keep.append(a)
        extra["shape_body"] = ap
        for name, arr in (("body_q", body_q), ("body_q_prev", body_q_prev), ("body_qd", body_qd),
                          ("body_com", body_com)):  # fmt: skip
            if arr is not None:
                a, ap = _d(np.asarray(arr).reshape(-1))
                keep.append(a)
                extra[name] = ap
    c = OracleContacts(count=int(count), max=len(p), particle=pp, shape=sp, body_pos=bpp, body_vel=bvp, normal=nnp,
                       **extra)  # fmt: skip
    return c, keep


def step(model: Model, q_in, qd_in, f_ext, contacts=None, dt=1.0 / 600.0, iterations=10, precision=64, nthreads=1,
         self_contact: SelfContact | None = None):  # fmt: skip
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
    if self_contact is None:
        rc = lib().oracle_vbd_step(C.byref(model.s), qp, qdp, fp, C.byref(c), dt, iterations, qop, vop, precision,
                                   nthreads)  # fmt: skip
    else:
        rc = lib().oracle_vbd_step_sc(C.byref(model.s), qp, qdp, fp, C.byref(c), C.byref(self_contact.s), dt,
                                      iterations, qop, vop, precision, nthreads)  # fmt: skip
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


def soft_contacts_shapes(q, radius, flags, shape_type, shape_transform, shape_scale, margin, max_contacts=None,
                         heightfield_index=None, heightfields=None, elevations=None, mesh_index=None, meshes=None,
                         shape_flags=None, shape_world=None, particle_world=None, shape_body=None, body_q=None):
    """Particle-shape contacts against static analytic shapes (GeoType values: plane 1, heightfield 2, sphere 3,
    capsule 4, ellipsoid 5, cylinder 6, box 7, cone 9) with transforms [S, 7] (position, quaternion xyzw) and
    scales [S, 3], in (particle, shape) order, skipping shapes without the COLLIDE_PARTICLES flag (1 << 2) and
    pairs of different worlds unless either is global (-1). Heightfield shape s uses grid ``heightfield_index[s]`` of
    ``heightfields`` (rows of (data_offset, nrow, ncol, hx, hy, min_z, max_z), scale applied) over the
    concatenated normalized ``elevations``. Mesh shape s (types 8, 10) uses ``meshes[mesh_index[s]]``, a
    (points [V, 3], triangles [T, 3]) pair. A shape on a body (``shape_body[s]`` >= 0) has its transform in the frame
    of ``body_q[shape_body[s]]`` (a [B, 7] array of (position, quaternion xyzw)); its contact points are returned in
    that body's frame, as create_soft_contacts writes them."""
    n = len(radius)
    S = len(shape_type)
    max_contacts = max_contacts or n * max(S, 1)
    qq, qp = _d(np.asarray(q).reshape(-1))
    r, rp = _d(radius)
    fl, flp = _i(flags)
    st, stp = _i(shape_type)
    sx, sxp = _d(np.asarray(shape_transform).reshape(-1))
    ss, ssp = _d(np.asarray(shape_scale).reshape(-1))
    part, pp = _i(-np.ones(max_contacts))
    shp, shpp = _i(-np.ones(max_contacts))
    bp, bpp = _d(np.zeros(3 * max_contacts))
    bv, bvp = _d(np.zeros(3 * max_contacts))
    nn, nnp = _d(np.zeros(3 * max_contacts))
    hfi = hfg = hfe = elv = None
    if heightfields is not None and len(heightfields):
        hf = np.asarray(heightfields, dtype=np.float64).reshape(-1, 7)
        hfi = _i(heightfield_index)
        hfg = _i(hf[:, :3].astype(np.int64))
        hfe = _d(hf[:, 3:])
        elv = _d(np.asarray(elevations).reshape(-1))
    mi = mvo = mto = mpt = mtr = None
    if meshes is not None and len(meshes):
        mi = _i(mesh_index)
        mvo = _i(np.cumsum([0] + [len(np.asarray(p).reshape(-1, 3)) for p, _ in meshes]))
        mto = _i(np.cumsum([0] + [len(np.asarray(t).reshape(-1, 3)) for _, t in meshes]))
        mpt = _d(np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1) for p, _ in meshes]))
        mtr = _i(np.concatenate([np.asarray(t).reshape(-1) for _, t in meshes]))
    sfl = None if shape_flags is None else _i(shape_flags)
    swl = None if shape_world is None else _i(shape_world)
    pwl = None if particle_world is None else _i(particle_world)
    sbd = None if shape_body is None or body_q is None else _i(shape_body)
    bq = None if shape_body is None or body_q is None else _d(np.asarray(body_q).reshape(-1))
    cnt = lib().oracle_soft_contacts_shapes(n, qp, rp, flp, S, stp, sxp, ssp, *(None if a is None else a[1] for a in
                                            (hfi, hfg, hfe, elv, mi, mvo, mto, mpt, mtr, sfl, swl, pwl)), margin,
                                            max_contacts, pp, shpp, bpp, bvp, nnp, None if sbd is None else sbd[1],
                                            None if bq is None else bq[1])  # fmt: skip
    if cnt < 0:
        raise ValueError("a shape type without an analytic SDF")
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


def collide(model: Model, sc: SelfContact, q, precision=64, nthreads=1) -> dict:
    """One self-contact detection at positions q; the buffers of ``TriMeshCollisionInfo``."""
    n, E = model.n, model.s.E
    qq, qp = _d(np.asarray(q).reshape(-1))
    vt, vtp = _i(np.zeros(2 * n * sc.vertex_buffer))
    vc, vcp = _i(np.zeros(n))
    vm, vmp = _d(np.zeros(n))
    ee, eep = _i(np.zeros(max(2 * E * sc.edge_buffer, 1)))
    ec, ecp = _i(np.zeros(max(E, 1)))
    em, emp = _d(np.zeros(max(E, 1)))
    fl, flp = _i(np.zeros(4))
    lib().oracle_collide(C.byref(model.s), C.byref(sc.s), qp, precision, vtp, vcp, vmp, eep, ecp, emp, flp, nthreads)
    return {"vt": vt, "vt_count": vc, "vt_min": vm, "ee": ee[: 2 * E * sc.edge_buffer], "ee_count": ec[:E],
            "ee_min": em[:E], "resize_flags": fl}  # fmt: skip


def sc_pair(kind, precision, x, xa, radius, ke, kd, mu, eps, dt, ee_eps=1e-5):
    """Self-contact pair term. kind "vt": x = (a, b, c, p) -> forces (4, 3), Hessians (4, 3, 3);
    kind "ee": x = (e1.v0, e1.v1, e2.v0, e2.v1) -> forces (2, 3), Hessians (2, 3, 3) of e1's vertices."""
    x_, xp = _d(np.asarray(x).reshape(-1))
    a_, ap = _d(np.asarray(xa).reshape(-1))
    if kind == "vt":
        out, op = _d(np.zeros(48))
        hit = lib().oracle_sc_vt(precision, xp, ap, radius, ke, kd, mu, eps, dt, op)
        return bool(hit), out[:12].reshape(4, 3), out[12:].reshape(4, 3, 3)
    out, op = _d(np.zeros(24))
    hit = lib().oracle_sc_ee(precision, xp, ap, radius, ke, kd, mu, eps, dt, ee_eps, op)
    return bool(hit), out[:6].reshape(2, 3), out[6:].reshape(2, 3, 3)


def sc_plane(kind, precision, x, dx, eps=1e-5, gamma=0.85):
    """Division plane of a pair: (dummy[4], n, d, t[4]); kind "vt": x = (v, t1, t2, t3), "ee": two edges."""
    x_, xp = _d(np.asarray(x).reshape(-1))
    d_, dp = _d(np.asarray(dx).reshape(-1))
    out, op = _d(np.zeros(14))
    lib().oracle_sc_plane(precision, 0 if kind == "vt" else 1, xp, dp, eps, gamma, op)
    return out[:4] != 0.0, out[4:7], out[7:10], out[10:14]


def tri_closest(a, b, c, p):
    x_, xp = _d(np.concatenate([a, b, c, p]))
    out, op = _d(np.zeros(7))
    lib().oracle_tri_closest(xp, op)
    return out[:3], out[3:6], int(out[6])


def edge_closest(p1, q1, p2, q2, eps=1e-5):
    x_, xp = _d(np.concatenate([p1, q1, p2, q2]))
    out, op = _d(np.zeros(3))
    lib().oracle_edge_closest(xp, eps, op)
    return out


def sc_norm(dis, radius, k):
    out, op = _d(np.zeros(2))
    lib().oracle_sc_norm(dis, radius, k, op)
    return out[0], out[1]
