"""vbd_step_noalloc against the allocating entry point (vbd_step), through the C ABI.

vbd_step_noalloc serves callers that may not allocate device memory: a host application that owns
all device memory through its own pool and forbids plug-ins to call cudaMalloc, or code that steps
the cloth while capturing a larger CUDA graph. It keeps its scratch in one fixed device array shared
by every call, so the tests run calls in a row (each reuses what the one before left there) and compare
them with the allocating path, within the 1e-4 m position tolerance of the other GPU parity tests. The
fixed array holds four contact slots per particle: a particle with more contacts keeps its four of lowest
index in the contact list, the same ones on every call, and the call reports the overflow through
vbd_step_noalloc_error. The file sorts last so that a run stopping at the first failure has run every
other test before it; it also passes when run alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from newton_chysx_b200 import CollisionPipeline, SolverVBD, _lib, sim
from tests.helpers import cloth_grid_builder

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0


def _p(t):
    return C.c_void_p(t.data_ptr())


class _NoAlloc:
    """The reference-layout adjacency on the device and a caller of vbd_step_noalloc for one model."""

    def __init__(self, model, solver):
        self.lib = _lib.load()
        self.solver = solver
        n = model.particle_count
        tri = np.ascontiguousarray(model.tri_indices.cpu().numpy(), dtype=np.int32).reshape(-1, 3)
        edges = np.ascontiguousarray(model.edge_indices.cpu().numpy(), dtype=np.int32).reshape(-1, 4)
        fo, eo = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        fa, ea = np.zeros(max(6 * len(tri), 1), np.int32), np.zeros(max(8 * len(edges), 1), np.int32)
        ip = C.POINTER(C.c_int32)
        assert self.lib.vbd_build_adjacency(n, len(tri), tri.ctypes.data_as(ip), len(edges), edges.ctypes.data_as(ip),
                                            fo.ctypes.data_as(ip), fa.ctypes.data_as(ip), eo.ctypes.data_as(ip),
                                            ea.ctypes.data_as(ip)) == 0  # fmt: skip
        self._keep = [torch.as_tensor(a, device="cuda") for a in (fo, fa[: max(fo[-1], 1)], eo, ea[: max(eo[-1], 1)])]
        self.adj = _lib.VbdRefAdjacency(*(_p(t) for t in self._keep))

    def step(self, s_in, s_out, contacts, iterations=10):
        cdesc = None
        if contacts is not None:
            cdesc = _lib.VbdContactsDesc(_p(contacts.soft_contact_count), contacts.soft_contact_max,
                                         _p(contacts.soft_contact_particle), _p(contacts.soft_contact_shape),
                                         _p(contacts.soft_contact_body_pos), _p(contacts.soft_contact_body_vel),
                                         _p(contacts.soft_contact_normal))  # fmt: skip
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        return self.lib.vbd_step_noalloc(C.byref(self.solver._md), C.byref(self.adj), iterations, 1e-2,
                                         _p(s_in.particle_q), _p(s_out.particle_q), _p(s_in.particle_qd),
                                         _p(s_out.particle_qd), _p(s_in.particle_f),
                                         None if cdesc is None else C.byref(cdesc), DT, stream)  # fmt: skip

    def error_bits(self):
        bits = C.c_int32(-1)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert self.lib.vbd_step_noalloc_error(C.byref(bits), stream) == 0
        return bits.value


def _ground_scene(planes=1):
    b = cloth_grid_builder(n=24, height=0.004)  # bottom row starts inside the contact margin
    for k in range(planes):
        b.add_ground_plane(height=-1.0e-3 * k)
    model = b.finalize("cuda")
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e3, 10.0, 0.5
    return model


def test_noalloc_step_matches_allocating_step_on_two_calls():
    model = _ground_scene()
    solver = SolverVBD(model, iterations=10, schedule="per_color", lanes_per_vertex=1)
    na = _NoAlloc(model, solver)
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    ref_in, ref_out = model.state(), model.state()
    na_in, na_out = model.state(), model.state()
    # start from a state with motion and ground contacts
    for k in range(30):
        pipe.collide(ref_in, contacts)
        solver.step(ref_in, ref_out, None, contacts, DT)
        ref_in, ref_out = ref_out, ref_in
    na_in.assign(ref_in)
    for call in range(2):
        pipe.collide(ref_in, contacts)
        torch.cuda.synchronize()
        assert int(contacts.soft_contact_count.item()) > 0
        solver.step(ref_in, ref_out, None, contacts, DT)
        rc = na.step(na_in, na_out, contacts)
        assert rc == 0, f"call {call}: {rc}"
        torch.cuda.synchronize()
        assert torch.abs(na_out.particle_q - ref_out.particle_q).max().item() <= 1e-4
        assert torch.abs(na_out.particle_qd - ref_out.particle_qd).max().item() <= 1e-4 / DT
        assert torch.equal(na_in.particle_q, na_out.particle_q)  # the reference writes state_in too
        assert na.error_bits() & _lib.VBD_DEVERR_CONTACT_OVERFLOW == 0
        ref_in, ref_out = ref_out, ref_in
        na_in, na_out = na_out, na_in


def _lowest_four(contacts):
    """A copy of the contact list holding, for every particle, only its four contacts of lowest index (in the
    same relative order)."""
    n = int(contacts.soft_contact_count.item())
    part = contacts.soft_contact_particle[:n].cpu().numpy()
    keep, seen = [], {}
    for t, p in enumerate(part):
        seen[p] = seen.get(p, 0) + 1
        if seen[p] <= _lib.VBD_NOALLOC_MAX_CONTACT_SLOTS:
            keep.append(t)
    idx = torch.as_tensor(np.array(keep, dtype=np.int64), device="cuda")
    out = sim.Contacts(contacts.soft_contact_max, "cuda")
    out.soft_contact_count.fill_(len(keep))
    for name in ("soft_contact_particle", "soft_contact_shape", "soft_contact_body_pos", "soft_contact_body_vel",
                 "soft_contact_normal"):  # fmt: skip
        getattr(out, name)[: len(keep)] = getattr(contacts, name)[idx]
    return out, max(seen.values())


def test_noalloc_keeps_the_lowest_index_contacts_and_reports_overflow():
    """Six ground planes 1 mm apart give the sheet's bottom particles six contacts each, more than the four
    slots. Two calls from the same input give the same positions bit for bit (the kept contacts do not depend
    on thread timing), set the overflow bit, and equal the allocating step given only each particle's four
    lowest-index contacts."""
    model = _ground_scene(planes=6)
    solver = SolverVBD(model, iterations=10, schedule="per_color", lanes_per_vertex=1)
    na = _NoAlloc(model, solver)
    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    s_in = model.state()
    pipe.collide(s_in, contacts)
    torch.cuda.synchronize()
    kept, most = _lowest_four(contacts)
    assert most > _lib.VBD_NOALLOC_MAX_CONTACT_SLOTS
    outs = []
    for _ in range(2):
        a_in, a_out = model.state(), model.state()
        a_in.assign(s_in)
        assert na.step(a_in, a_out, contacts) == 0
        torch.cuda.synchronize()
        assert na.error_bits() & _lib.VBD_DEVERR_CONTACT_OVERFLOW
        outs.append(a_out.particle_q.clone())
    assert torch.equal(outs[0], outs[1])
    r_in, r_out = model.state(), model.state()
    r_in.assign(s_in)
    solver.step(r_in, r_out, None, kept, DT)
    torch.cuda.synchronize()
    assert torch.abs(outs[0] - r_out.particle_q).max().item() <= 1e-4
    # a call without the overflow clears the bit
    one = _ground_scene(planes=1)
    s1 = SolverVBD(one, iterations=10, schedule="per_color", lanes_per_vertex=1)
    na1, p1 = _NoAlloc(one, s1), CollisionPipeline(one, soft_contact_margin=0.01)
    c1, x_in, x_out = p1.contacts(), one.state(), one.state()
    p1.collide(x_in, c1)
    assert na1.step(x_in, x_out, c1) == 0
    assert na1.error_bits() & _lib.VBD_DEVERR_CONTACT_OVERFLOW == 0


def test_noalloc_reports_skipped_singular_blocks():
    """A free particle of negligible mass and no elements has |det H| = (m / dt^2)^3 below the 1e-8 threshold:
    the update is skipped, as the reference does, and the error word says so."""
    b = cloth_grid_builder(n=8, height=0.5)
    b.add_particle((3.0, 0.0, 1.0), (0.0, 0.0, 0.0), 1.0e-12, radius=5.0e-3)
    b.color(include_bending=True)
    model = b.finalize("cuda")
    solver = SolverVBD(model, iterations=2, schedule="per_color", lanes_per_vertex=1)
    na = _NoAlloc(model, solver)
    s_in, s_out = model.state(), model.state()
    assert na.step(s_in, s_out, None, iterations=2) == 0
    assert na.error_bits() & _lib.VBD_DEVERR_SINGULAR_SKIPPED


def test_noalloc_rejects_models_beyond_its_scratch():
    lib = _lib.load()
    md = _lib.VbdModelDesc()
    md.particle_count = _lib.VBD_NOALLOC_MAX_PARTICLES + 1
    offs = np.array([0, md.particle_count], dtype=np.int32)
    md.color_count = 1
    md.color_offsets_host = offs.ctypes.data_as(C.POINTER(C.c_int32))
    md.color_particles_dev = C.c_void_p(1)  # never dereferenced: the size check comes first
    adj = _lib.VbdRefAdjacency(C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1))
    dummy = C.c_void_p(1)
    rc = lib.vbd_step_noalloc(C.byref(md), C.byref(adj), 10, 1e-2, dummy, dummy, dummy, dummy, None, None,
                              1.0 / 600.0, None)  # fmt: skip
    assert rc == _lib.VBD_ERR_TOO_LARGE
