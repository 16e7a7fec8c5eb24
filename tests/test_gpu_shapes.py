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


def _gpu_contacts(q, radius, flags, shape_type, shape_transform, shape_scale, margin):
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
    rc = lib.vbd_soft_contacts_shapes(n, qd.data_ptr(), rd.data_ptr(), fd.data_ptr(), S, st.ctypes.data_as(ip),
                                      sx.ctypes.data_as(fp), ss.ctypes.data_as(fp), float(margin), cmax, cnt.data_ptr(),
                                      part.data_ptr(), shp.data_ptr(), bp.data_ptr(), bv.data_ptr(), nn.data_ptr(),
                                      None)  # fmt: skip
    _lib.check(rc, "vbd_soft_contacts_shapes")
    torch.cuda.synchronize()
    k = int(cnt.item())
    return {(int(a), int(b)): (x, y, z) for a, b, x, y, z in
            zip(part[:k].cpu().numpy(), shp[:k].cpu().numpy(), bp[:k].cpu().numpy(), bv[:k].cpu().numpy(),
                nn[:k].cpu().numpy())}  # fmt: skip


def _compare(gpu, ref_pairs, ref_bp, ref_nn, near):
    ref = {pr: (b, nv) for pr, b, nv in zip(ref_pairs, ref_bp, ref_nn)}
    missing = [pr for pr in ref if pr not in gpu and pr not in near]
    extra = [pr for pr in gpu if pr not in ref and pr not in near]
    assert not missing and not extra, (missing[:5], extra[:5])
    common = [pr for pr in ref if pr in gpu]
    assert len(common) > 0.99 * len(ref)
    eb = max(np.abs(gpu[pr][0] - ref[pr][0]).max() for pr in common)
    en = max(np.abs(gpu[pr][2] - ref[pr][1]).max() for pr in common)
    assert eb <= 2e-5 and en <= 2e-5, (eb, en)
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
