"""vbd_step_noalloc against the allocating entry point (vbd_step), through the C ABI.

vbd_step_noalloc serves callers that may not allocate device memory: a host application that owns
all device memory through its own pool and forbids plug-ins to call cudaMalloc, or code that steps
the cloth while capturing a larger CUDA graph. It keeps its scratch in one fixed device array shared
by every call, so this test runs two calls in a row (the second reuses what the first left there)
and compares both with the allocating path, within the 1e-4 m position tolerance of the other GPU
parity tests. The file sorts last so that a run stopping at the first failure has run every other
test before it; it also passes when run alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from newton_chysx_b200 import CollisionPipeline, SolverVBD, _lib
from tests.helpers import cloth_grid_builder

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_step_matches_allocating_step_on_two_calls():
    b = cloth_grid_builder(n=24, height=0.004)  # bottom row starts inside the contact margin
    b.add_ground_plane()
    model = b.finalize("cuda")
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e3, 10.0, 0.5
    solver = SolverVBD(model, iterations=10, schedule="per_color", lanes_per_vertex=1)
    lib = _lib.load()

    # reference-layout adjacency, built on the host and copied to the device by the caller
    n = model.particle_count
    tri = np.ascontiguousarray(model.tri_indices.cpu().numpy(), dtype=np.int32)
    edges = np.ascontiguousarray(model.edge_indices.cpu().numpy(), dtype=np.int32)
    fo, eo = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
    fa, ea = np.zeros(6 * len(tri), np.int32), np.zeros(8 * len(edges), np.int32)
    ip = C.POINTER(C.c_int32)
    assert lib.vbd_build_adjacency(n, len(tri), tri.ctypes.data_as(ip), len(edges), edges.ctypes.data_as(ip),
                                   fo.ctypes.data_as(ip), fa.ctypes.data_as(ip), eo.ctypes.data_as(ip),
                                   ea.ctypes.data_as(ip)) == 0  # fmt: skip
    d_fo, d_fa = torch.as_tensor(fo, device="cuda"), torch.as_tensor(fa[: fo[-1]], device="cuda")
    d_eo, d_ea = torch.as_tensor(eo, device="cuda"), torch.as_tensor(ea[: eo[-1]], device="cuda")
    adj = _lib.VbdRefAdjacency(_p(d_fo), _p(d_fa), _p(d_eo), _p(d_ea))

    pipe = CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    cdesc = _lib.VbdContactsDesc(_p(contacts.soft_contact_count), contacts.soft_contact_max,
                                 _p(contacts.soft_contact_particle), _p(contacts.soft_contact_shape),
                                 _p(contacts.soft_contact_body_pos), _p(contacts.soft_contact_body_vel),
                                 _p(contacts.soft_contact_normal))  # fmt: skip
    dt = 1.0 / 600.0
    ref_in, ref_out = model.state(), model.state()
    na_in, na_out = model.state(), model.state()
    # start from a state with motion and ground contacts
    for k in range(30):
        pipe.collide(ref_in, contacts)
        solver.step(ref_in, ref_out, None, contacts, dt)
        ref_in, ref_out = ref_out, ref_in
    na_in.assign(ref_in)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        pipe.collide(ref_in, contacts)
        torch.cuda.synchronize()
        assert int(contacts.soft_contact_count.item()) > 0
        solver.step(ref_in, ref_out, None, contacts, dt)
        rc = lib.vbd_step_noalloc(C.byref(solver._md), C.byref(adj), 10, 1e-2, _p(na_in.particle_q),
                                  _p(na_out.particle_q), _p(na_in.particle_qd), _p(na_out.particle_qd),
                                  _p(na_in.particle_f), C.byref(cdesc), dt, stream)  # fmt: skip
        assert rc == 0, f"call {call}: {rc}"
        torch.cuda.synchronize()
        assert torch.abs(na_out.particle_q - ref_out.particle_q).max().item() <= 1e-4
        assert torch.abs(na_out.particle_qd - ref_out.particle_qd).max().item() <= 1e-4 / dt
        assert torch.equal(na_in.particle_q, na_out.particle_q)  # the reference writes state_in too
        ref_in, ref_out = ref_out, ref_in
        na_in, na_out = na_out, na_in


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
