"""GPU particle-shape contact generation (``vbd_soft_contacts_shapes``) against goldens from the reference's own SDF
functions, and the builder's shapes through ``CollisionPipeline`` against the oracle.

Contacts come from an atomic counter, so they are compared as sets keyed by (particle, shape). FP32 against the
float64 goldens: contact points and normals to 2e-5; pairs whose distance lies within 1e-5 of the contact
threshold (margin + radius) may fall on either side of it in FP32 and are not required to match."""

import ctypes as C

import numpy as np
import pytest
import torch

from newton_chysx_b200 import _lib, sim
from oracle import vbd_oracle as orc
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu


def _gpu_contacts(q, radius, flags, shape_type, shape_transform, shape_scale, margin, hf_index=None,
                  heightfields=None, elevations=None, mesh_index=None, meshes=None):
    lib = _lib.load()
    n, S = len(radius), len(shape_type)
    cmax = n * S
    dev = torch.device("cuda")
    qd = torch.as_tensor(np.asarray(q, dtype=np.float32), device=dev).contiguous()
    rd = torch.as_tensor(np.asarray(radius, dtype=np.float32), device=dev)
    fd = torch.as_tensor(np.asarray(flags, dtype=np.int32), device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    part = torch.full((cmax,), -1, dtype=torch.int32, device=dev)
    shp = torch.full((cmax,), -1, dtype=torch.int32, device=dev)
    bp = torch.zeros((cmax, 3), dtype=torch.float32, device=dev)
    bv = torch.zeros((cmax, 3), dtype=torch.float32, device=dev)
    nn = torch.zeros((cmax, 3), dtype=torch.float32, device=dev)
    st = np.ascontiguousarray(shape_type, dtype=np.int32)
    sx = np.ascontiguousarray(shape_transform, dtype=np.float32)
    ss = np.ascontiguousarray(shape_scale, dtype=np.float32)
    ip, fp = C.POINTER(C.c_int32), C.POINTER(C.c_float)
    outs = (cmax, cnt.data_ptr(), part.data_ptr(), shp.data_ptr(), bp.data_ptr(), bv.data_ptr(), nn.data_ptr(), None)
    if heightfields is None and meshes is None:
        rc = lib.vbd_soft_contacts_shapes(n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), S, st.ctypes.data_as(ip),
                                          sx.ctypes.data_as(fp), ss.ctypes.data_as(fp), float(margin), *outs)  # fmt: skip
    else:
        tb = _lib.VbdShapeTable(S, st.ctypes.data_as(ip), sx.ctypes.data_as(fp), ss.ctypes.data_as(fp))
        if heightfields is not None:
            hi = np.ascontiguousarray(hf_index, dtype=np.int32)
            hfs = (_lib.VbdHeightfield * len(heightfields))(
                *[_lib.VbdHeightfield(int(r[0]), int(r[1]), int(r[2]), *map(float, r[3:])) for r in heightfields])
            ev = torch.as_tensor(np.asarray(elevations, dtype=np.float32), device=dev)
            tb.shape_heightfield_index_host = hi.ctypes.data_as(ip)
            tb.heightfield_count, tb.heightfields_host = len(heightfields), hfs
            tb.elevations_dev, tb.elevation_count = ev.data_ptr(), ev.numel()
        if meshes is not None:
            dm = [sim._DeviceMesh(sim.Mesh(v, f)) for v, f in meshes]
            handles = (C.c_void_p * S)(*[dm[k].handle if k >= 0 else None for k in mesh_index])
            tb.shape_mesh_host = C.cast(handles, C.POINTER(C.c_void_p))
        rc = lib.vbd_soft_contacts_table(n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), C.byref(tb), float(margin),
                                         *outs)  # fmt: skip
    _lib.check(rc, "vbd_soft_contacts")
    torch.cuda.synchronize()
    k = int(cnt.item())
    return {(int(a), int(b)): (x, y, z) for a, b, x, y, z in
            zip(part[:k].cpu().numpy(), shp[:k].cpu().numpy(), bp[:k].cpu().numpy(), bv[:k].cpu().numpy(),
                nn[:k].cpu().numpy())}  # fmt: skip


def _compare(gpu, ref_pairs, ref_bp, ref_nn, near, ref_d=None):
    """Same pairs (outside `near`), contact points and normals within 2e-5, zero body velocity. With ref_d (mesh
    contacts, whose normal is normalize(x - closest point)): FP32 squared distances (relative rounding 6e-8) fix
    the closest point along the surface only to about sqrt(2 * 6e-8) |d| = 3.5e-4 |d| where two triangles meet,
    and the coordinates' rounding adds ~1e-7 / |d|; normals are held to 1e-3 + 1e-6 / |d|, and pairs with
    |d| < 1e-4 to their contact point only."""
    ref = {pr: (b, nv) for pr, b, nv in zip(ref_pairs, ref_bp, ref_nn)}
    dist = dict(zip(ref_pairs, ref_d)) if ref_d is not None else {}
    missing = [pr for pr in ref if pr not in gpu and pr not in near]
    extra = [pr for pr in gpu if pr not in ref and pr not in near]
    assert not missing and not extra, (missing[:5], extra[:5])
    common = [pr for pr in ref if pr in gpu]
    assert len(common) > 0.99 * len(ref)
    eb = max(np.abs(gpu[pr][0] - ref[pr][0]).max() for pr in common)
    assert eb <= 2e-5, eb
    for pr in common:
        d = abs(dist.get(pr, 1.0))
        if d >= 1e-4:
            tol = 2e-5 if pr not in dist else 1e-3 + 1e-6 / d
            assert np.abs(gpu[pr][2] - ref[pr][1]).max() <= tol, (pr, d)
    assert max(np.abs(gpu[pr][1]).max() for pr in common) == 0.0


def test_shape_contacts_match_reference_sdfs():
    g = load_golden("soft_contact_shapes.npz")
    gpu = _gpu_contacts(g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"], g["shape_scale"],
                        float(g["margin"]))  # fmt: skip
    # pairs within 1e-5 of the threshold, recomputed in float64 for every (particle, shape)
    near = set()
    for s in range(len(g["shape_type"])):
        one = orc.soft_contacts_shapes(g["q"], g["radius"], g["flags"], g["shape_type"][s:s + 1],
                                       g["shape_transform"][s:s + 1], g["shape_scale"][s:s + 1],
                                       float(g["margin"]) + 1e-5)  # fmt: skip
        loose = set(zip(one[1][:one[0]].tolist()))
        tight = orc.soft_contacts_shapes(g["q"], g["radius"], g["flags"], g["shape_type"][s:s + 1],
                                         g["shape_transform"][s:s + 1], g["shape_scale"][s:s + 1],
                                         float(g["margin"]) - 1e-5)  # fmt: skip
        near |= {(p[0], s) for p in loose - set(zip(tight[1][:tight[0]].tolist()))}
    pairs = list(zip(g["particle"].tolist(), g["shape"].tolist()))
    _compare(gpu, pairs, g["body_pos"], g["normal"], near)


def test_collision_pipeline_shapes_match_oracle():
    b = sim.ModelBuilder()
    rng = np.random.default_rng(3)
    pts = np.stack([rng.uniform(-1.0, 1.0, 20000), rng.uniform(-1.0, 1.0, 20000), rng.uniform(-0.05, 0.7, 20000)], 1)
    b.add_particles(pts, (0.0, 0.0, 0.0), 1.0, radius=0.01)
    b.add_ground_plane()
    q = sim.quat_from_axis_angle((0.2, 1.0, 0.3), 0.6)
    b.add_shape_box(xform=((-0.4, -0.4, 0.3), q), hx=0.3, hy=0.2, hz=0.1)
    b.add_shape_capsule(xform=((0.2, 0.6, 0.3), q), radius=0.1, half_height=0.2)
    b.add_shape_cylinder(xform=((0.6, -0.6, 0.2), q), radius=0.15, half_height=0.1)
    b.add_shape_ellipsoid(xform=((-0.1, 0.0, 0.45), q), rx=0.3, ry=0.2, rz=0.15)
    b.add_shape_sphere(xform=((0.5, 0.1, 0.3), sim.quat_identity()), radius=0.2)
    b.add_shape_plane(xform=((-0.6, 0.5, 0.25), q), width=0.6, length=0.4)
    model = b.finalize("cuda")
    pipe = sim.CollisionPipeline(model, soft_contact_max=model.particle_count * model.shape_count,
                                 soft_contact_margin=0.01)  # fmt: skip
    contacts = pipe.contacts()
    state = model.state()
    pipe.collide(state, contacts)
    torch.cuda.synchronize()
    k = int(contacts.soft_contact_count.item())
    gpu = {(int(a), int(s)): (x, y, z) for a, s, x, y, z in zip(
        contacts.soft_contact_particle[:k].cpu().numpy(), contacts.soft_contact_shape[:k].cpu().numpy(),
        contacts.soft_contact_body_pos[:k].cpu().numpy(), contacts.soft_contact_body_vel[:k].cpu().numpy(),
        contacts.soft_contact_normal[:k].cpu().numpy())}  # fmt: skip
    qf = model.particle_q.cpu().numpy().astype(np.float64)
    r = model.particle_radius.cpu().numpy().astype(np.float64)
    fl = model.particle_flags.cpu().numpy()
    args = (model.shape_type, model.shape_transform.astype(np.float64), model.shape_scale.astype(np.float64))
    cnt, p, s, bp, _, nn = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01)
    lo = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 - 1e-5)
    hi = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 + 1e-5)
    near = set(zip(hi[1][:hi[0]].tolist(), hi[2][:hi[0]].tolist()))
    near -= set(zip(lo[1][:lo[0]].tolist(), lo[2][:lo[0]].tolist()))
    assert len(set(s[:cnt].tolist())) == model.shape_count
    _compare(gpu, list(zip(p[:cnt].tolist(), s[:cnt].tolist())), bp[:cnt], nn[:cnt], near)


def test_cone_and_heightfield_contacts_match_reference():
    """Cones and heightfields (scaled, rotated, one grid of a single row) against goldens from the reference's
    ``sdf_cone``/``sdf_cone_grad`` and ``sample_sdf_grad_heightfield``."""
    g = load_golden("soft_contact_cone_hfield.npz")
    hf = dict(hf_index=g["shape_heightfield_index"], heightfields=g["heightfields"], elevations=g["elevations"])
    gpu = _gpu_contacts(g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"], g["shape_scale"],
                        float(g["margin"]), **hf)  # fmt: skip
    near = set()
    for s in range(len(g["shape_type"])):
        one = dict(heightfield_index=g["shape_heightfield_index"][s:s + 1], heightfields=g["heightfields"],
                   elevations=g["elevations"])  # fmt: skip
        args = (g["q"], g["radius"], g["flags"], g["shape_type"][s:s + 1], g["shape_transform"][s:s + 1],
                g["shape_scale"][s:s + 1])  # fmt: skip
        loose = orc.soft_contacts_shapes(*args, float(g["margin"]) + 1e-5, **one)
        tight = orc.soft_contacts_shapes(*args, float(g["margin"]) - 1e-5, **one)
        near |= {(p, s) for p in set(loose[1][:loose[0]].tolist()) - set(tight[1][:tight[0]].tolist())}
    pairs = list(zip(g["particle"].tolist(), g["shape"].tolist()))
    _compare(gpu, pairs, g["body_pos"], g["normal"], near)
    assert {s for _, s in gpu} == {0, 1, 2, 3, 4}


def test_shape_table_arguments_are_checked():
    """A heightfield without its grid table, an index out of range, a grid overrunning the elevations, a zero
    extent, a mesh shape without a handle or with a zero scale are refused before any launch; the plain entry
    point refuses heightfields and meshes."""
    from tests.helpers import box_mesh

    lib = _lib.load()
    dev = torch.device("cuda")
    q = torch.zeros((4, 3), device=dev)
    r = torch.full((4,), 0.01, device=dev)
    fl = torch.ones(4, dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    oi = torch.zeros(64, dtype=torch.int32, device=dev)
    of = torch.zeros((64, 3), device=dev)
    ev = torch.zeros(12, device=dev)
    ip, fp = C.POINTER(C.c_int32), C.POINTER(C.c_float)
    sx = np.array([0, 0, 0, 0, 0, 0, 1], dtype=np.float32)
    outs = (64, cnt.data_ptr(), oi.data_ptr(), oi.data_ptr(), of.data_ptr(), of.data_ptr(), of.data_ptr(), None)

    def call(typ, idx=0, grids=(), n_elev=12, scale=(1.0, 1.0, 1.0), mesh=None):
        st = np.array([typ], dtype=np.int32)
        ss = np.array(scale, dtype=np.float32)
        hi = np.array([idx], dtype=np.int32)
        hfs = (_lib.VbdHeightfield * max(len(grids), 1))(*grids)
        tb = _lib.VbdShapeTable(1, st.ctypes.data_as(ip), sx.ctypes.data_as(fp), ss.ctypes.data_as(fp),
                                hi.ctypes.data_as(ip), len(grids), hfs, ev.data_ptr(), n_elev)  # fmt: skip
        handles = (C.c_void_p * 1)(None if mesh is None else mesh.handle)
        tb.shape_mesh_host = C.cast(handles, C.POINTER(C.c_void_p))
        return lib.vbd_soft_contacts_table(4, q.data_ptr(), r.data_ptr(), fl.data_ptr(), C.byref(tb), 0.01, *outs)

    good = _lib.VbdHeightfield(0, 3, 4, 1.0, 1.0, 0.0, 1.0)
    assert call(2, 0, [good]) == _lib.VBD_OK
    torch.cuda.synchronize()
    assert int(cnt.item()) == 4  # all four particles lie on the flat grid (z = 0, inside the margin)
    assert call(2, 1, [good]) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert call(2, 0, [good], n_elev=11) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert call(2, 0, [_lib.VbdHeightfield(0, 3, 4, 0.0, 1.0, 0.0, 1.0)]) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert call(2, 0, []) == _lib.VBD_ERR_INVALID_ARGUMENT
    dm = sim._DeviceMesh(sim.Mesh(*box_mesh(0.1, 0.1, 0.1)))
    assert call(8, mesh=dm) == _lib.VBD_OK
    torch.cuda.synchronize()
    assert int(cnt.item()) == 0  # 0.1 deep inside: beyond the query's reach margin + radius = 0.02, as in the reference
    dm = sim._DeviceMesh(sim.Mesh(*box_mesh(0.015, 0.015, 0.015)))
    assert call(8, mesh=dm) == _lib.VBD_OK
    torch.cuda.synchronize()
    assert int(cnt.item()) == 4  # 0.015 inside: within reach
    assert call(8) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert call(10, mesh=dm, scale=(1.0, 0.0, 1.0)) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert call(11) == _lib.VBD_ERR_UNSUPPORTED
    for typ in (2, 8):
        st = np.array([typ], dtype=np.int32)
        rc = lib.vbd_soft_contacts_shapes(4, q.data_ptr(), r.data_ptr(), fl.data_ptr(), 1, st.ctypes.data_as(ip),
                                          sx.ctypes.data_as(fp), np.ones(3, np.float32).ctypes.data_as(fp), 0.01,
                                          *outs)  # fmt: skip
        assert rc == _lib.VBD_ERR_UNSUPPORTED
    torch.cuda.synchronize()


def _terrain(n=33, seed=5, noise=0.01):
    gx, gy = np.meshgrid(np.linspace(-1.0, 1.0, n), np.linspace(-1.0, 1.0, n))
    z = 0.05 * np.sin(3.0 * gx) * np.cos(2.0 * gy) + noise * np.random.default_rng(seed).uniform(size=gx.shape)
    return sim.Heightfield(z, n, n, hx=0.8, hy=0.8)


def _drop_cloth(shape_fn, steps, kd=1.0):
    """A 24 x 24 cloth of 1 m dropped from 0.35 m onto the shapes `shape_fn(builder, cfg)` adds, stepped through
    CollisionPipeline + SolverVBD. The shapes' contact damping kd is 1: the reference's damping Hessian
    (kd ke / dt) nn^T at the default kd = 100 makes this light cloth (0.35 g per particle) unstable on creased or
    tilted surfaces in the reference's own algorithm (the oracle shows the same)."""
    from newton_chysx_b200 import SolverVBD

    n, side = 24, 1.0
    mu, lam = 1.0e4 * 1e-3 / 2.6, 1.0e4 * 1e-3 * 0.3 / 0.91
    b = sim.ModelBuilder(gravity=-9.81)
    b.add_cloth_grid(pos=(-0.5, -0.5, 0.35), rot=sim.quat_identity(), vel=(0.0, 0.0, 0.0), dim_x=n - 1, dim_y=n - 1,
                     cell_x=side / (n - 1), cell_y=side / (n - 1), mass=0.2 / (n * n), tri_ke=mu, tri_ka=lam,
                     tri_kd=0.0, edge_ke=1e-4, edge_kd=0.0, particle_radius=5e-3)  # fmt: skip
    b.color(include_bending=True)
    shape_fn(b, sim.ShapeConfig(kd=kd))
    model = b.finalize("cuda")
    model.soft_contact_ke = 1.0e4
    solver = SolverVBD(model, iterations=10)
    pipe = sim.CollisionPipeline(model, soft_contact_margin=0.02)
    contacts = pipe.contacts()
    s0, s1 = model.state(), model.state()
    for _ in range(steps):
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, 1.0 / 600.0)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    assert solver.device_errors() == 0
    x = s0.particle_q.cpu().numpy().astype(np.float64)
    v = s0.particle_qd.cpu().numpy().astype(np.float64)
    assert np.isfinite(x).all() and np.isfinite(v).all()
    return model, x, v


def test_collision_pipeline_cone_heightfield_match_oracle():
    b = sim.ModelBuilder()
    rng = np.random.default_rng(4)
    pts = np.stack([rng.uniform(-1.0, 1.0, 20000), rng.uniform(-1.0, 1.0, 20000), rng.uniform(-0.1, 0.6, 20000)], 1)
    b.add_particles(pts, (0.0, 0.0, 0.0), 1.0, radius=0.01)
    q = sim.quat_from_axis_angle((0.2, 1.0, 0.3), 0.6)
    b.add_shape_heightfield(xform=((0.0, 0.0, 0.05), sim.quat_from_axis_angle((0.0, 0.0, 1.0), 0.4)),
                            heightfield=_terrain(), scale=(1.0, 0.8, 1.5))  # fmt: skip
    b.add_shape_cone(xform=((0.3, -0.2, 0.3), q), radius=0.2, half_height=0.25)
    b.add_shape_cone(xform=((-0.4, 0.4, 0.35), sim.quat_identity()), radius=0.3, half_height=0.15)
    model = b.finalize("cuda")
    pipe = sim.CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    pipe.collide(model.state(), contacts)
    torch.cuda.synchronize()
    k = int(contacts.soft_contact_count.item())
    gpu = {(int(a), int(s)): (x, y, z) for a, s, x, y, z in zip(
        contacts.soft_contact_particle[:k].cpu().numpy(), contacts.soft_contact_shape[:k].cpu().numpy(),
        contacts.soft_contact_body_pos[:k].cpu().numpy(), contacts.soft_contact_body_vel[:k].cpu().numpy(),
        contacts.soft_contact_normal[:k].cpu().numpy())}  # fmt: skip
    qf = model.particle_q.cpu().numpy().astype(np.float64)
    r = model.particle_radius.cpu().numpy().astype(np.float64)
    fl = model.particle_flags.cpu().numpy()
    args = (model.shape_type, model.shape_transform.astype(np.float64), model.shape_scale.astype(np.float64))
    hf = dict(heightfield_index=model.shape_heightfield_index, heightfields=model.heightfield_data,
              elevations=model.heightfield_elevations.cpu().numpy())  # fmt: skip
    cnt, p, s, bp, _, nn = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01, **hf)
    lo = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 - 1e-5, **hf)
    hi = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 + 1e-5, **hf)
    near = set(zip(hi[1][:hi[0]].tolist(), hi[2][:hi[0]].tolist()))
    near -= set(zip(lo[1][:lo[0]].tolist(), lo[2][:lo[0]].tolist()))
    assert len(set(s[:cnt].tolist())) == model.shape_count
    _compare(gpu, list(zip(p[:cnt].tolist(), s[:cnt].tolist())), bp[:cnt], nn[:cnt], near)


def test_cloth_settles_on_heightfield():
    """A cloth dropped on terrain lands on it: after 0.6 s every particle has its centre above the plane of the
    terrain triangle under it and within 0.2 m of it (it started 0.3 m up), and nothing has blown up (speeds stay
    below the 2.4 m/s of the fall)."""
    model, x, v = _drop_cloth(lambda b, cfg: b.add_shape_heightfield(heightfield=_terrain(noise=0.0), cfg=cfg), 360)
    # signed distance of every particle to its terrain triangle's plane, from the oracle's query with a wide margin
    cnt, p, _, bp, _, nn = orc.soft_contacts_shapes(
        x, np.zeros(len(x)), np.ones(len(x), np.int32), model.shape_type, model.shape_transform.astype(np.float64),
        model.shape_scale.astype(np.float64), 1.0, heightfield_index=model.shape_heightfield_index,
        heightfields=model.heightfield_data, elevations=model.heightfield_elevations.cpu().numpy())  # fmt: skip
    assert cnt == len(x)
    d = np.einsum("ij,ij->i", x[p[:cnt]] - bp[:cnt], nn[:cnt])
    assert d.min() >= 0.0 and d.max() <= 0.2, (d.min(), d.max())
    assert np.abs(v).max() < 2.4


def test_box_mesh_contacts_match_reference_box_sdf():
    """A closed box mesh at scale 2 against the reference's own ``sdf_box`` goldens, for every particle within the
    mesh query's reach (margin + radius / min|scale| in the unscaled frame)."""
    from tests.helpers import box_mesh

    g = load_golden("soft_contact_shapes.npz")
    s = int(np.flatnonzero(g["shape_type"] == 7)[0])
    mesh = box_mesh(*(0.5 * g["shape_scale"][s]))
    args = (g["q"], g["radius"], g["flags"], np.array([8]), g["shape_transform"][s:s + 1], np.array([[2.0, 2.0, 2.0]]))
    gpu = _gpu_contacts(*args, float(g["margin"]), mesh_index=[0], meshes=[mesh])
    gpu = {(p, 0): v for (p, _), v in gpu.items()}
    reach = 2.0 * (float(g["margin"]) + g["radius"][g["particle"]] / 2.0)
    sel = (g["shape"] == s) & (g["distance"] > -reach)
    # pairs within 1e-5 of either threshold (the contact margin, the search reach) may fall either way in FP32
    one = dict(mesh_index=[0], meshes=[mesh])
    loose = orc.soft_contacts_shapes(*args, float(g["margin"]) + 1e-5, **one)
    tight = orc.soft_contacts_shapes(*args, float(g["margin"]) - 1e-5, **one)
    near = {(p, 0) for p in set(loose[1][:loose[0]].tolist()) - set(tight[1][:tight[0]].tolist())}
    near |= {(int(p), 0) for p, dd, rr in zip(g["particle"], g["distance"], reach) if abs(dd + rr) < 1e-5}
    pairs = [(int(p), 0) for p in g["particle"][sel]]
    _compare(gpu, pairs, g["body_pos"][sel], g["normal"][sel], near, g["distance"][sel])


def test_collision_pipeline_meshes_match_oracle():
    """Box, icosphere and torus meshes (rotated; uniform, non-uniform and sub-unit scales; a convex hull shape)
    through CollisionPipeline against the oracle's brute-force query."""
    from tests.helpers import box_mesh, icosphere, torus_mesh

    b = sim.ModelBuilder()
    rng = np.random.default_rng(6)
    pts = np.stack([rng.uniform(-1.0, 1.0, 20000), rng.uniform(-1.0, 1.0, 20000), rng.uniform(-0.1, 0.7, 20000)], 1)
    b.add_particles(pts, (0.0, 0.0, 0.0), 1.0, radius=0.01)
    q = sim.quat_from_axis_angle((0.2, 1.0, 0.3), 0.6)
    box = sim.Mesh(*box_mesh(0.3, 0.2, 0.1))
    b.add_shape_mesh(xform=((-0.4, -0.4, 0.3), q), mesh=box)
    b.add_shape_convex_hull(xform=((0.5, 0.5, 0.3), sim.quat_identity()), mesh=sim.Mesh(*icosphere(0.5, 3)),
                            scale=(0.5, 0.4, 0.6))  # fmt: skip
    b.add_shape_mesh(xform=((0.4, -0.4, 0.3), q), mesh=sim.Mesh(*torus_mesh(0.3, 0.1)), scale=(1.2, 1.0, 0.8))
    b.add_shape_mesh(xform=((-0.5, 0.5, 0.2), sim.quat_identity()), mesh=box, scale=(0.7, 1.5, 2.0))
    model = b.finalize("cuda")
    assert list(model.shape_mesh_index) == [0, 1, 2, 0] and len(model._device_meshes) == 3
    pipe = sim.CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    pipe.collide(model.state(), contacts)
    torch.cuda.synchronize()
    k = int(contacts.soft_contact_count.item())
    gpu = {(int(a), int(s)): (x, y, z) for a, s, x, y, z in zip(
        contacts.soft_contact_particle[:k].cpu().numpy(), contacts.soft_contact_shape[:k].cpu().numpy(),
        contacts.soft_contact_body_pos[:k].cpu().numpy(), contacts.soft_contact_body_vel[:k].cpu().numpy(),
        contacts.soft_contact_normal[:k].cpu().numpy())}  # fmt: skip
    qf = model.particle_q.cpu().numpy().astype(np.float64)
    r = model.particle_radius.cpu().numpy().astype(np.float64)
    fl = model.particle_flags.cpu().numpy()
    args = (model.shape_type, model.shape_transform.astype(np.float64), model.shape_scale.astype(np.float64))
    ms = dict(mesh_index=model.shape_mesh_index, meshes=[(m.vertices, m.indices) for m in model.meshes])
    cnt, p, s, bp, _, nn = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01, **ms)
    # near either threshold: the margin (d against margin + r) and the search reach (scaled by min|scale|)
    lo = orc.soft_contacts_shapes(qf, r * (1 - 1e-5), fl, *args, 0.01 - 1e-5, **ms)
    hi = orc.soft_contacts_shapes(qf, r * (1 + 1e-5), fl, *args, 0.01 + 1e-5, **ms)
    near = set(zip(hi[1][:hi[0]].tolist(), hi[2][:hi[0]].tolist())) - set(zip(lo[1][:lo[0]].tolist(),
                                                                               lo[2][:lo[0]].tolist()))  # fmt: skip
    assert len(set(s[:cnt].tolist())) == model.shape_count
    d = np.einsum("ij,ij->i", qf[p[:cnt]] - bp[:cnt], nn[:cnt])
    _compare(gpu, list(zip(p[:cnt].tolist(), s[:cnt].tolist())), bp[:cnt], nn[:cnt], near, d)


def test_cloth_drapes_over_mesh_box():
    """A cloth dropped on a box mesh lying on the ground: after 0.6 s no particle centre is inside the box, none is
    below the ground, and the cloth has come down onto the box."""
    from tests.helpers import box_mesh

    def shapes(b, cfg):
        b.add_ground_plane(cfg=cfg)
        b.add_shape_mesh(xform=((0.0, 0.0, 0.1), sim.quat_from_axis_angle((0.0, 0.0, 1.0), 0.5)),
                         mesh=sim.Mesh(*box_mesh(0.2, 0.15, 0.1)), cfg=cfg)  # fmt: skip

    _, x, _ = _drop_cloth(shapes, 360)
    assert x[:, 2].min() >= 0.0
    c, sn = np.cos(-0.5), np.sin(-0.5)
    loc = (x - [0.0, 0.0, 0.1]) @ np.array([[c, -sn, 0.0], [sn, c, 0.0], [0.0, 0.0, 1.0]]).T
    inside = (np.abs(loc[:, 0]) < 0.2) & (np.abs(loc[:, 1]) < 0.15) & (np.abs(loc[:, 2]) < 0.1)
    assert not inside.any()
    assert x[:, 2].max() < 0.25


def test_collision_pipeline_worlds_match_oracle():
    """World filtering and the COLLIDE_PARTICLES flag on the GPU against the oracle (three worlds, one sphere each,
    one of them not colliding with particles, and a global ground plane)."""
    from tests.test_oracle_shapes import _world_scene

    m = _world_scene("cuda")
    pipe = sim.CollisionPipeline(m, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    pipe.collide(m.state(), contacts)
    torch.cuda.synchronize()
    k = int(contacts.soft_contact_count.item())
    gpu = {(int(a), int(s)): (x, y, z) for a, s, x, y, z in zip(
        contacts.soft_contact_particle[:k].cpu().numpy(), contacts.soft_contact_shape[:k].cpu().numpy(),
        contacts.soft_contact_body_pos[:k].cpu().numpy(), contacts.soft_contact_body_vel[:k].cpu().numpy(),
        contacts.soft_contact_normal[:k].cpu().numpy())}  # fmt: skip
    qf = m.particle_q.cpu().numpy().astype(np.float64)
    r = m.particle_radius.cpu().numpy().astype(np.float64)
    fl = m.particle_flags.cpu().numpy()
    args = (m.shape_type, m.shape_transform.astype(np.float64), m.shape_scale.astype(np.float64))
    kw = dict(shape_flags=m.shape_flags, shape_world=m.shape_world, particle_world=m.particle_world.cpu().numpy())
    cnt, p, s, bp, _, nn = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01, **kw)
    lo = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 - 1e-5, **kw)
    hi = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 + 1e-5, **kw)
    near = set(zip(hi[1][:hi[0]].tolist(), hi[2][:hi[0]].tolist()))
    near -= set(zip(lo[1][:lo[0]].tolist(), lo[2][:lo[0]].tolist()))
    assert {sh for _, sh in gpu} == {0, 1, 3}
    _compare(gpu, list(zip(p[:cnt].tolist(), s[:cnt].tolist())), bp[:cnt], nn[:cnt], near)


def test_many_worlds_and_shapes_match_oracle():
    """More shapes than one kernel parameter table holds: 40 worlds with a sphere and a rotated box each (80 world
    shapes), a global ground plane, a global capsule that does not collide with particles, and particles in every
    world plus 2,000 global particles (which meet every shape), through the model's device shape set."""
    rng = np.random.default_rng(12)
    top = sim.ModelBuilder(up_axis="Z")
    q = sim.quat_from_axis_angle((0.3, 1.0, 0.2), 0.7)
    for w in range(40):
        b = sim.ModelBuilder(up_axis="Z")
        pts = np.stack([rng.uniform(-0.5, 0.5, 500), rng.uniform(-0.5, 0.5, 500), rng.uniform(-0.02, 0.5, 500)], 1)
        b.add_particles(pts, (0.0, 0.0, 0.0), 1.0, radius=0.01)
        c = rng.uniform(-0.2, 0.2, 2)
        b.add_shape_sphere(xform=((c[0], c[1], 0.2), sim.quat_identity()), radius=0.15)
        b.add_shape_box(xform=((-c[0], -c[1], 0.25), q), hx=0.1, hy=0.15, hz=0.05)
        top.add_world(b)
    pts = np.stack([rng.uniform(-0.5, 0.5, 2000), rng.uniform(-0.5, 0.5, 2000), rng.uniform(-0.02, 0.5, 2000)], 1)
    top.add_particles(pts, (0.0, 0.0, 0.0), 1.0, radius=0.01)
    top.add_ground_plane()
    top.add_shape_capsule(xform=((0.0, 0.0, 0.2), q), radius=0.2, half_height=0.2,
                          cfg=sim.ShapeConfig(has_particle_collision=False))  # fmt: skip
    m = top.finalize("cuda")
    assert m.shape_count == 82 and (m.shape_world[:80] >= 0).all() and list(m.shape_world[80:]) == [-1, -1]
    pipe = sim.CollisionPipeline(m, soft_contact_max=200000, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    pipe.collide(m.state(), contacts)
    torch.cuda.synchronize()
    k = int(contacts.soft_contact_count.item())
    gpu = {(int(a), int(s)): (x, y, z) for a, s, x, y, z in zip(
        contacts.soft_contact_particle[:k].cpu().numpy(), contacts.soft_contact_shape[:k].cpu().numpy(),
        contacts.soft_contact_body_pos[:k].cpu().numpy(), contacts.soft_contact_body_vel[:k].cpu().numpy(),
        contacts.soft_contact_normal[:k].cpu().numpy())}  # fmt: skip
    qf = m.particle_q.cpu().numpy().astype(np.float64)
    r = m.particle_radius.cpu().numpy().astype(np.float64)
    fl = m.particle_flags.cpu().numpy()
    args = (m.shape_type, m.shape_transform.astype(np.float64), m.shape_scale.astype(np.float64))
    kw = dict(shape_flags=m.shape_flags, shape_world=m.shape_world, particle_world=m.particle_world.cpu().numpy(),
              max_contacts=200000)  # fmt: skip
    cnt, p, s, bp, _, nn = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01, **kw)
    lo = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 - 1e-5, **kw)
    hi = orc.soft_contacts_shapes(qf, r, fl, *args, 0.01 + 1e-5, **kw)
    near = set(zip(hi[1][:hi[0]].tolist(), hi[2][:hi[0]].tolist()))
    near -= set(zip(lo[1][:lo[0]].tolist(), lo[2][:lo[0]].tolist()))
    assert k == cnt or abs(k - cnt) <= len(near)
    pw = m.particle_world.cpu().numpy()
    glob = np.flatnonzero(pw == -1)
    assert {sh for pp, sh in gpu if pp in set(glob.tolist())} >= set(range(0, 80, 7))  # global particles meet worlds
    assert 81 not in {sh for _, sh in gpu}
    _compare(gpu, list(zip(p[:cnt].tolist(), s[:cnt].tolist())), bp[:cnt], nn[:cnt], near)


@pytest.mark.parametrize("path", ["table", "set", "set_global"])
def test_reference_create_soft_contacts_kernel_golden(path):
    """Every device path against the reference's ``create_soft_contacts`` kernel run as-is: worlds, the
    particle-collision flag, a heightfield and seven analytic shapes. "table" is ``vbd_soft_contacts_table``;
    "set" a shape set (9 shapes: its records launch as a kernel parameter); "set_global" the same set forced
    through the global-memory kernel with its per-world shape lists."""
    g = load_golden("create_soft_contacts.npz")
    lib = _lib.load()
    dev = torch.device("cuda")
    n, S = len(g["radius"]), len(g["shape_type"])
    cmax = n * S
    qd = torch.as_tensor(g["q"].astype(np.float32), device=dev).contiguous()
    rd = torch.as_tensor(g["radius"].astype(np.float32), device=dev)
    fd = torch.as_tensor(g["flags"], device=dev)
    pw = torch.as_tensor(g["particle_world"], device=dev)
    ev = torch.as_tensor(g["elevations"].astype(np.float32), device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    part = torch.full((cmax,), -1, dtype=torch.int32, device=dev)
    shp = torch.full((cmax,), -1, dtype=torch.int32, device=dev)
    bp, bv, nn = (torch.zeros((cmax, 3), dtype=torch.float32, device=dev) for _ in range(3))
    ip, fp = C.POINTER(C.c_int32), C.POINTER(C.c_float)
    arrs = dict(st=g["shape_type"].astype(np.int32), sx=g["shape_transform"].astype(np.float32),
                ss=g["shape_scale"].astype(np.float32), hi=g["shape_heightfield_index"].astype(np.int32),
                sf=g["shape_flags"].astype(np.int32), sw=g["shape_world"].astype(np.int32))  # fmt: skip
    hf = g["heightfields"][0]
    hfs = (_lib.VbdHeightfield * 1)(_lib.VbdHeightfield(int(hf[0]), int(hf[1]), int(hf[2]), *map(float, hf[3:])))
    tb = _lib.VbdShapeTable(S, arrs["st"].ctypes.data_as(ip), arrs["sx"].ctypes.data_as(fp),
                            arrs["ss"].ctypes.data_as(fp), arrs["hi"].ctypes.data_as(ip), 1, hfs, ev.data_ptr(),
                            ev.numel(), None, arrs["sf"].ctypes.data_as(ip), arrs["sw"].ctypes.data_as(ip),
                            pw.data_ptr())  # fmt: skip
    outs = (cmax, cnt.data_ptr(), part.data_ptr(), shp.data_ptr(), bp.data_ptr(), bv.data_ptr(), nn.data_ptr(), None)
    if path == "table":
        rc = lib.vbd_soft_contacts_table(n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), C.byref(tb), float(g["margin"]),
                                         *outs)  # fmt: skip
        _lib.check(rc, "vbd_soft_contacts_table")
        torch.cuda.synchronize()
    else:
        h = C.c_void_p()
        _lib.check(lib.vbd_shape_set_create(C.byref(tb), C.byref(h)), "vbd_shape_set_create")
        if path == "set_global":
            _lib.check(lib.vbd_shape_set_use_parameter_table(h, 0), "vbd_shape_set_use_parameter_table")
        rc = lib.vbd_soft_contacts_set(h, n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), pw.data_ptr(), None,
                                       float(g["margin"]), *outs)  # fmt: skip
        _lib.check(rc, "vbd_soft_contacts_set")
        torch.cuda.synchronize()
        lib.vbd_shape_set_destroy(h)
    k = int(cnt.item())
    gpu = {(int(a), int(b)): (x, y, z) for a, b, x, y, z in zip(
        part[:k].cpu().numpy(), shp[:k].cpu().numpy(), bp[:k].cpu().numpy(), bv[:k].cpu().numpy(),
        nn[:k].cpu().numpy())}  # fmt: skip
    kw = dict(heightfield_index=g["shape_heightfield_index"], heightfields=g["heightfields"], elevations=g["elevations"],
              shape_flags=g["shape_flags"], shape_world=g["shape_world"], particle_world=g["particle_world"])  # fmt: skip
    args = (g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"], g["shape_scale"])
    lo = orc.soft_contacts_shapes(*args, float(g["margin"]) - 1e-5, **kw)
    hi_ = orc.soft_contacts_shapes(*args, float(g["margin"]) + 1e-5, **kw)
    near = set(zip(hi_[1][:hi_[0]].tolist(), hi_[2][:hi_[0]].tolist()))
    near -= set(zip(lo[1][:lo[0]].tolist(), lo[2][:lo[0]].tolist()))
    pairs = list(zip(g["particle"].tolist(), g["shape"].tolist()))
    _compare(gpu, pairs, g["body_pos"], g["normal"], near)


@pytest.mark.parametrize("path", ["table", "set", "set_global", "pipeline"])
def test_reference_create_soft_contacts_on_bodies(path):
    """Shapes on two rotated, displaced bodies against the reference's ``create_soft_contacts`` run as-is: each
    shape's world frame is body_q[body] times its own transform, contact points come out in the body's frame and
    normals in world. "table" and "set"/"set_global" call the C ABI (the body transforms in the table, or per call
    for a set); "pipeline" builds the scene with ``ModelBuilder.add_body`` and runs ``CollisionPipeline.collide``
    on a state whose ``body_q`` holds the transforms."""
    g = load_golden("create_soft_contacts_bodies.npz")
    lib = _lib.load()
    dev = torch.device("cuda")
    n, S = len(g["radius"]), len(g["shape_type"])
    cmax = n * S
    bq = torch.as_tensor(g["body_q"].astype(np.float32), device=dev).contiguous()
    if path == "pipeline":
        b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
        b.add_particles(g["q"], (0.0, 0.0, 0.0), 1.0, g["radius"], g["flags"])
        bodies = [b.add_body() for _ in g["body_q"]]  # at the origin: the state's body_q moves them
        kinds = {1: "plane", 3: "sphere", 4: "capsule", 5: "ellipsoid", 6: "cylinder", 7: "box", 9: "cone"}
        for t, X, sc, body in zip(g["shape_type"], g["shape_transform"], g["shape_scale"], g["shape_body"]):
            xf = (tuple(X[:3]), tuple(X[3:]))
            bd = -1 if body < 0 else bodies[body]
            k = kinds[int(t)]
            if k == "plane":
                b.add_shape_plane(xform=xf, width=0.0, length=0.0, body=bd)
            elif k == "sphere":
                b.add_shape_sphere(body=bd, xform=xf, radius=float(sc[0]))
            elif k == "box":
                b.add_shape_box(body=bd, xform=xf, hx=float(sc[0]), hy=float(sc[1]), hz=float(sc[2]))
            elif k == "ellipsoid":
                b.add_shape_ellipsoid(body=bd, xform=xf, rx=float(sc[0]), ry=float(sc[1]), rz=float(sc[2]))
            else:
                getattr(b, f"add_shape_{k}")(body=bd, xform=xf, radius=float(sc[0]), half_height=float(sc[1]))
        m = b.finalize("cuda")
        assert m.body_count == 2 and np.array_equal(m._shape_body_host, g["shape_body"])
        np.testing.assert_allclose(m.shape_scale, g["shape_scale"], atol=1e-7)
        state = m.state()
        state.body_q.copy_(bq)
        pipe = sim.CollisionPipeline(m, soft_contact_margin=float(g["margin"]))
        c = pipe.contacts()
        pipe.collide(state, c)
        torch.cuda.synchronize()
        k = int(c.soft_contact_count.item())
        part, shp, bp, bv, nn = (c.soft_contact_particle, c.soft_contact_shape, c.soft_contact_body_pos,
                                 c.soft_contact_body_vel, c.soft_contact_normal)  # fmt: skip
        with pytest.raises(ValueError, match="body_q"):
            pipe.collide(_no_bodies(state), c)
    else:
        qd = torch.as_tensor(g["q"].astype(np.float32), device=dev).contiguous()
        rd = torch.as_tensor(g["radius"].astype(np.float32), device=dev)
        fd = torch.as_tensor(g["flags"], device=dev)
        cnt = torch.zeros(1, dtype=torch.int32, device=dev)
        part = torch.full((cmax,), -1, dtype=torch.int32, device=dev)
        shp = torch.full((cmax,), -1, dtype=torch.int32, device=dev)
        bp, bv, nn = (torch.zeros((cmax, 3), dtype=torch.float32, device=dev) for _ in range(3))
        ip, fp = C.POINTER(C.c_int32), C.POINTER(C.c_float)
        arrs = dict(st=g["shape_type"].astype(np.int32), sx=g["shape_transform"].astype(np.float32),
                    ss=g["shape_scale"].astype(np.float32), sb=g["shape_body"].astype(np.int32))  # fmt: skip
        tb = _lib.VbdShapeTable(S, arrs["st"].ctypes.data_as(ip), arrs["sx"].ctypes.data_as(fp),
                                arrs["ss"].ctypes.data_as(fp), None, 0, None, None, 0, None, None, None, None,
                                arrs["sb"].ctypes.data_as(ip), 2, bq.data_ptr())  # fmt: skip
        outs = (cmax, cnt.data_ptr(), part.data_ptr(), shp.data_ptr(), bp.data_ptr(), bv.data_ptr(), nn.data_ptr(),
                None)  # fmt: skip
        if path == "table":
            _lib.check(lib.vbd_soft_contacts_table(n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), C.byref(tb),
                                                   float(g["margin"]), *outs), "vbd_soft_contacts_table")  # fmt: skip
        else:
            h = C.c_void_p()
            _lib.check(lib.vbd_shape_set_create(C.byref(tb), C.byref(h)), "vbd_shape_set_create")
            if path == "set_global":
                _lib.check(lib.vbd_shape_set_use_parameter_table(h, 0), "vbd_shape_set_use_parameter_table")
            # a set with shapes on bodies needs the transforms of the call
            assert lib.vbd_soft_contacts_set(h, n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), None, None,
                                             float(g["margin"]), *outs) == _lib.VBD_ERR_INVALID_ARGUMENT  # fmt: skip
            _lib.check(lib.vbd_soft_contacts_set(h, n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), None,
                                                 bq.data_ptr(), float(g["margin"]), *outs),
                       "vbd_soft_contacts_set")  # fmt: skip
            torch.cuda.synchronize()
            lib.vbd_shape_set_destroy(h)
        torch.cuda.synchronize()
        k = int(cnt.item())
    gpu = {(int(a), int(b_)): (x, y, z) for a, b_, x, y, z in zip(
        part[:k].cpu().numpy(), shp[:k].cpu().numpy(), bp[:k].cpu().numpy(), bv[:k].cpu().numpy(),
        nn[:k].cpu().numpy())}  # fmt: skip
    kw = dict(shape_body=g["shape_body"], body_q=g["body_q"].astype(np.float32).astype(np.float64))
    args = (g["q"], g["radius"], g["flags"], g["shape_type"], g["shape_transform"], g["shape_scale"])
    lo = orc.soft_contacts_shapes(*args, float(g["margin"]) - 1e-5, **kw)
    hi_ = orc.soft_contacts_shapes(*args, float(g["margin"]) + 1e-5, **kw)
    near = set(zip(hi_[1][:hi_[0]].tolist(), hi_[2][:hi_[0]].tolist()))
    near -= set(zip(lo[1][:lo[0]].tolist(), lo[2][:lo[0]].tolist()))
    _compare(gpu, list(zip(g["particle"].tolist(), g["shape"].tolist())), g["body_pos"], g["normal"], near)


def _no_bodies(state):
    s = sim.State()
    s.particle_q = state.particle_q
    return s


@pytest.mark.parametrize("param_table", [True, False])
def test_shape_set_contact_overflow(param_table):
    """More contacts than soft_contact_max through the shape set, in both of its kernels: the count reports them
    all, as the reference's counter does, only the first soft_contact_max slots are written, and the slots past
    them stay untouched."""
    m = _world_scene_many()
    sim._current_shape_set(m).use_parameter_table(param_table)
    full = sim.CollisionPipeline(m, soft_contact_max=m.particle_count * m.shape_count, soft_contact_margin=0.01)
    cf = full.contacts()
    full.collide(m.state(), cf)
    small = sim.CollisionPipeline(m, soft_contact_max=50, soft_contact_margin=0.01)
    cs = small.contacts()
    cs.soft_contact_particle = torch.full((60,), -7, dtype=torch.int32, device="cuda")  # 10 guard slots
    small.collide(m.state(), cs)
    torch.cuda.synchronize()
    total = int(cf.soft_contact_count.item())
    assert total > 50 and int(cs.soft_contact_count.item()) == total
    written = cs.soft_contact_particle[:50].cpu().numpy()
    assert (written >= 0).all() and (written < m.particle_count).all()
    assert (cs.soft_contact_particle[50:].cpu().numpy() == -7).all()
    pairs = set(zip(cf.soft_contact_particle[:total].cpu().tolist(), cf.soft_contact_shape[:total].cpu().tolist()))
    assert set(zip(written.tolist(), cs.soft_contact_shape[:50].cpu().tolist())) <= pairs


def _world_scene_many():
    from tests.test_oracle_shapes import _world_scene

    return _world_scene("cuda")


def test_shapes_edited_after_finalize_take_effect():
    """The reference reads the model's shape arrays at every create_soft_contacts launch. Moving a sphere,
    scaling it and switching its particle-collision flag off after finalize change the next contacts without a
    refresh call; a graph captured before the edit keeps the shapes of its capture."""
    b = sim.ModelBuilder(up_axis="Z")
    pts = np.stack(np.meshgrid(np.linspace(-0.5, 0.5, 21), np.linspace(-0.5, 0.5, 21), [0.0], indexing="ij"), -1)
    b.add_particles(pts.reshape(-1, 3), (0.0, 0.0, 0.0), 1.0, radius=5e-3)
    # radius 0.02 centred 0.02 below the sheet: touches the centre particle only (the next ones, 0.05 m away, are
    # 0.034 m from its surface, beyond margin + radius = 0.015 m)
    b.add_shape_sphere(xform=((0.0, 0.0, -0.02), sim.quat_identity()), radius=0.02)
    m = b.finalize("cuda")
    pipe = sim.CollisionPipeline(m, soft_contact_margin=0.01)
    c, s = pipe.contacts(), m.state()

    def touched():
        pipe.collide(s, c)
        torch.cuda.synchronize()
        k = int(c.soft_contact_count.item())
        return set(c.soft_contact_particle[:k].cpu().tolist())

    centre = 10 * 21 + 10
    assert touched() == {centre}
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side), torch.cuda.graph(g, stream=side):
        pipe.collide(s, c)
    torch.cuda.current_stream().wait_stream(side)
    m.shape_transform[0, 0] = 0.25  # move the sphere under particle (15, 10)
    assert touched() == {15 * 21 + 10}
    m.shape_scale[0, 0] = 0.3  # radius 0.3: a disc of particles
    many = touched()
    assert len(many) > 20 and 15 * 21 + 10 in many
    g.replay()  # the captured graph still sees the sphere as it was captured
    torch.cuda.synchronize()
    k = int(c.soft_contact_count.item())
    assert set(c.soft_contact_particle[:k].cpu().tolist()) == {centre}
    m.shape_flags[0] &= ~4  # COLLIDE_PARTICLES off
    assert touched() == set()
