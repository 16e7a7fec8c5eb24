"""``SolverVBD``: drop-in for the particle (cloth) path of ``newton.solvers.SolverVBD``.

Same constructor keywords (``newton/_src/solvers/vbd/solver_vbd.py:196-242``) and the same
``step(state_in, state_out, control, contacts, dt)`` (``:1575-1622``) with the reference's side
effects: ``state_in.particle_q`` receives the solution, ``state_out.particle_q`` the same positions and
``state_out.particle_qd = (q - q_prev) / dt``. The work runs in ``libvbd_b200.so`` (hand-written
sm_100a kernels) on the current torch CUDA stream, so a substep loop can be captured in a CUDA graph.

Beyond the reference keywords:

* ``precision``: ``"fp32"`` (the reference's arithmetic), ``"mixed"`` (contact vertices add their contact
  terms and solve in FP64, other vertices solve in FP64 when their block is ill-conditioned; FP64 residual
  sums, see ``residuals()``), ``"fp64"`` (all FP64; the state arrays must be float64).
* ``schedule``: ``"per_color"`` (one launch per color and iteration), ``"persistent"`` (one launch
  per substep, a CTA per cloth instance/world), ``"auto"``.
* ``lanes_per_vertex`` / ``block_size``: launch shape (0 = default; see ``autotune``).
* ``positions_in_shared``: ``"auto"`` / ``"off"`` / ``"on"`` — the persistent kernel keeps each
  instance's positions in shared memory during the sweep (FP32 and mixed precision).
* ``layout``: ``"ell"`` / ``"ell16"`` (per-incidence stencil records in sweep order, coalesced; one
  lane per vertex; 32- or 16-bit vertex ids), ``"ring"`` (one-ring fan records: each vertex walks its
  triangle fan once and shares every face normal between membrane and bending; persistent schedule,
  manifold fans), ``"csr"`` (adjacency + element records; any lanes per vertex), ``"auto"``.
* ``min_blocks_per_sm``: 2..4 compiles the persistent stencil kernel for that many resident CTAs of
  256 threads per SM (a register budget); 0 leaves the compiler's choice.
* ``pair_vertices``: the ell16 persistent kernel (FP32) solves two vertices per thread, one in each lane
  of Blackwell's paired FP32 instructions (FFMA2 / FADD2 / FMUL2), halving the arithmetic instructions.
* ``instance_per_warp``: the persistent csr kernel gives each warp its own instance (colors separated by
  ``__syncwarp`` instead of a CTA barrier), for batches of small instances such as soft-body blocks.

Particle self-contact (``particle_enable_self_contact=True`` and the ``particle_self_contact_*``
keywords) runs with the csr layout, on the per-color schedule for one cloth and on the persistent schedule
(one CTA per world, the detections grid-wide between persistent launches) for a model of several worlds; on
the persistent schedule a world's vertices and edges only meet its own triangles and edges, and the AVBD
penalty ramp (``rigid_avbd_beta``) must be 0. See ``collision.py`` for the filters and the stand-alone
detector.

Arrays. The model, states and contacts may hold torch tensors (this package's ``sim``), the reference's Warp
arrays, or any device array with ``__cuda_array_interface__``; each is checked for its element type, size and
contiguity (``interop``). With Warp arrays the step launches on Warp's current stream of the device, as the
reference does; otherwise on torch's current stream. The reference Model's ``particle_world_start``
([world_count + 2], ``newton/_src/sim/model.py:172-187``) gives the worlds of a batched model, as this
package's ``world_particle_start`` does.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib, interop
from .interop import F32, F64, I32
from .sim import Contacts, Model, State


def _ptr(obj, what="array", typestr=None, count=None, at_least=None):
    return interop.pointer(obj, what, typestr, count, at_least)


def contacts_desc(contacts, model):
    """The ``VbdContactsDesc`` of a ``Contacts`` (its arrays checked for type and size), or None when there is
    nothing to collide with."""
    if contacts is None or contacts.soft_contact_max <= 0 or model.shape_count <= 0:
        return None
    cmax = int(contacts.soft_contact_max)
    cdesc = _lib.VbdContactsDesc()
    cdesc.soft_contact_count_dev = _ptr(contacts.soft_contact_count, "contacts.soft_contact_count", I32, at_least=1)
    cdesc.soft_contact_max = cmax
    cdesc.soft_contact_particle_dev = _ptr(contacts.soft_contact_particle, "contacts.soft_contact_particle", I32,
                                           at_least=cmax)  # fmt: skip
    cdesc.soft_contact_shape_dev = _ptr(contacts.soft_contact_shape, "contacts.soft_contact_shape", I32,
                                        at_least=cmax)  # fmt: skip
    cdesc.soft_contact_body_pos_dev = _ptr(contacts.soft_contact_body_pos, "contacts.soft_contact_body_pos", F32,
                                           at_least=3 * cmax)  # fmt: skip
    cdesc.soft_contact_body_vel_dev = _ptr(contacts.soft_contact_body_vel, "contacts.soft_contact_body_vel", F32,
                                           at_least=3 * cmax)  # fmt: skip
    cdesc.soft_contact_normal_dev = _ptr(contacts.soft_contact_normal, "contacts.soft_contact_normal", F32,
                                         at_least=3 * cmax)  # fmt: skip
    return cdesc


class SolverVBD:
    def __init__(
        self,
        model: Model,
        iterations: int = 10,
        friction_epsilon: float = 1e-2,
        integrate_with_external_rigid_solver: bool = False,
        particle_enable_self_contact: bool = False,
        particle_self_contact_radius: float = 0.2,
        particle_self_contact_margin: float = 0.2,
        particle_conservative_bound_relaxation: float = 0.85,
        particle_vertex_contact_buffer_size: int = 32,
        particle_edge_contact_buffer_size: int = 64,
        particle_collision_detection_interval: int = 0,
        particle_edge_parallel_epsilon: float = 1e-5,
        particle_enable_tile_solve: bool = True,
        particle_topological_contact_filter_threshold: int = 2,
        particle_rest_shape_contact_exclusion_radius: float = 0.0,
        particle_external_vertex_contact_filtering_map: dict | None = None,
        particle_external_edge_contact_filtering_map: dict | None = None,
        rigid_avbd_alpha: float = 0.95,
        rigid_avbd_joint_alpha: float | None = None,
        rigid_avbd_contact_alpha: float | None = None,
        rigid_avbd_beta: float = 0.0,
        rigid_avbd_linear_beta: float | None = None,
        rigid_avbd_angular_beta: float | None = None,
        rigid_avbd_gamma: float = 0.999,
        rigid_contact_hard: bool = True,
        rigid_contact_history: bool = False,
        rigid_contact_stick_motion_eps: float = 1.0e-4,
        rigid_contact_stick_freeze_translation_eps: float = 1.0e-4,
        rigid_contact_stick_freeze_angular_eps: float = 1.0e-4,
        rigid_contact_k_start: float = 1.0e2,
        rigid_body_contact_buffer_size: int = 64,
        rigid_body_particle_contact_buffer_size: int = 256,
        rigid_joint_linear_ke: float = 1.0e5,
        rigid_joint_angular_ke: float = 1.0e5,
        rigid_joint_linear_k_start: float = 1.0e2,
        rigid_joint_angular_k_start: float = 1.0e1,
        rigid_joint_linear_kd: float = 0.0,
        rigid_joint_angular_kd: float = 0.0,
        rigid_enable_dahl_friction: bool | None = None,
        *,
        precision: str = "fp32",
        schedule: str = "auto",
        lanes_per_vertex: int = 0,
        block_size: int = 0,
        fp64_solve_threshold: float = 1e-3,
        contact_slots: int = 0,
        positions_in_shared: str = "auto",
        layout: str = "auto",
        min_blocks_per_sm: int = 0,
        pair_vertices: bool = False,
        instance_per_warp: bool = False,
    ):
        if rigid_avbd_beta < 0:
            raise ValueError(f"rigid_avbd_beta must be >= 0, got {rigid_avbd_beta}")
        linear_beta = rigid_avbd_linear_beta if rigid_avbd_linear_beta is not None else rigid_avbd_beta
        self.model = model
        self.iterations = iterations
        self.friction_epsilon = friction_epsilon
        self.integrate_with_external_rigid_solver = integrate_with_external_rigid_solver
        self.particle_enable_self_contact = particle_enable_self_contact
        self.particle_self_contact_radius = particle_self_contact_radius
        self.particle_self_contact_margin = particle_self_contact_margin
        self.particle_conservative_bound_relaxation = particle_conservative_bound_relaxation
        self.particle_collision_detection_interval = particle_collision_detection_interval
        self.particle_topological_contact_filter_threshold = particle_topological_contact_filter_threshold
        self.particle_rest_shape_contact_exclusion_radius = particle_rest_shape_contact_exclusion_radius
        if particle_enable_self_contact:
            if particle_self_contact_margin < particle_self_contact_radius:
                raise ValueError(
                    "particle_self_contact_margin is smaller than particle_self_contact_radius, this will result in "
                    "missing contacts and cause instability."
                )
            if layout not in ("auto", "csr") or schedule not in ("auto", "per_color", "persistent"):
                raise ValueError("particle self-contact runs with the csr layout on the per_color or persistent schedule")
            if schedule == "auto":
                # several worlds: one CTA per world (pairs within a world); one cloth: per-color launches
                soft = int(getattr(model, "spring_count", 0) or 0) + int(getattr(model, "tet_count", 0) or 0) > 0
                worlds = interop.world_starts(model)
                schedule = "persistent" if worlds is not None and linear_beta == 0.0 and not soft else "per_color"
            layout = "csr"
            if lanes_per_vertex == 0:
                # a vertex's faces, hinges and self-contact entries are split over its lanes, each kind from
                # lane 0. One large sheet (per-color schedule) has tens of edge-edge entries per vertex: 16 lanes
                # measured fastest on a 256 x 256 sheet draped on a sphere, timed from one settled state (8.91 ms
                # per substep against 9.22 ms with 8; 21 ms with one). Batched sheets (persistent schedule) have
                # about one: 4 lanes measured fastest (2,048 sheets of 16 x 16 from one settled state: 16.5 ms
                # against 18.9 ms with 2 and 18.4 ms with 8; 256 of 32 x 32: 11.8 ms against 15.0 ms with 16)
                lanes_per_vertex = 4 if schedule == "persistent" else 16
        if model.body_count > 0 and not integrate_with_external_rigid_solver:
            raise NotImplementedError("rigid bodies (AVBD) are not part of this solver")
        if model.particle_count == 0:
            raise ValueError("model has no particles")
        if len(model.particle_color_groups) == 0:
            raise ValueError(
                "model.particle_color_groups is empty! When using the SolverVBD you must call ModelBuilder.color() "
                "or ModelBuilder.set_coloring() before calling ModelBuilder.finalize()."
            )
        if precision not in _lib.PRECISION:
            raise ValueError(f"precision must be one of {list(_lib.PRECISION)}")
        if schedule not in _lib.SCHEDULE:
            raise ValueError(f"schedule must be one of {list(_lib.SCHEDULE)}")
        device = interop.torch_device(getattr(model, "device", None))
        if device.type != "cuda":
            raise RuntimeError("SolverVBD needs a CUDA model (finalize(device='cuda'))")
        self.precision = precision
        self.device = device
        self._lib = _lib.load()
        self._warp = interop.from_warp(model.particle_mass)

        groups = [np.ascontiguousarray(interop.to_host(g), dtype=np.int32).reshape(-1)
                  for g in model.particle_color_groups]  # fmt: skip
        self._color_offsets = np.concatenate([[0], np.cumsum([g.size for g in groups])]).astype(np.int32)
        self._color_particles = torch.as_tensor(np.concatenate(groups), device=device).contiguous()
        if self._color_offsets[-1] != model.particle_count:
            raise ValueError("particle_color_groups must cover every particle exactly once")
        self._world_start = interop.world_starts(model)

        V, T, Ecount = int(model.particle_count), int(model.tri_count), int(model.edge_count)
        S = int(model.shape_count)
        md = _lib.VbdModelDesc()
        md.particle_count = V
        md.tri_count = T
        md.edge_count = Ecount
        md.shape_count = S
        md.particle_mass_dev = _ptr(model.particle_mass, "model.particle_mass", F32, V)
        md.particle_inv_mass_dev = _ptr(model.particle_inv_mass, "model.particle_inv_mass", F32, V)
        md.particle_flags_dev = _ptr(model.particle_flags, "model.particle_flags", I32, V)
        md.particle_radius_dev = _ptr(model.particle_radius, "model.particle_radius", F32, V)
        if T:
            md.tri_indices_dev = _ptr(model.tri_indices, "model.tri_indices", I32, 3 * T)
            md.tri_poses_dev = _ptr(model.tri_poses, "model.tri_poses", F32, 4 * T)
            md.tri_materials_dev = _ptr(model.tri_materials, "model.tri_materials", F32, 5 * T)
            md.tri_areas_dev = _ptr(model.tri_areas, "model.tri_areas", F32, T)
        if Ecount:
            md.edge_indices_dev = _ptr(model.edge_indices, "model.edge_indices", I32, 4 * Ecount)
            md.edge_rest_angle_dev = _ptr(model.edge_rest_angle, "model.edge_rest_angle", F32, Ecount)
            md.edge_rest_length_dev = _ptr(model.edge_rest_length, "model.edge_rest_length", F32, Ecount)
            md.edge_bending_properties_dev = _ptr(model.edge_bending_properties, "model.edge_bending_properties",
                                                  F32, 2 * Ecount)  # fmt: skip
        md.color_count = len(groups)
        md.color_offsets_host = self._color_offsets.ctypes.data_as(C.POINTER(C.c_int32))
        md.color_particles_dev = _ptr(self._color_particles, "particle_color_groups", I32, V)
        md.world_count = 0 if self._world_start is None else len(self._world_start) - 1
        md.world_particle_start_host = (
            None if self._world_start is None else self._world_start.ctypes.data_as(C.POINTER(C.c_int32))
        )
        md.gravity_dev = _ptr(model.gravity, "model.gravity", F32, at_least=3)
        md.soft_contact_ke = float(model.soft_contact_ke)
        md.soft_contact_kd = float(model.soft_contact_kd)
        md.soft_contact_mu = float(model.soft_contact_mu)
        if S:
            md.shape_material_ke_dev = _ptr(model.shape_material_ke, "model.shape_material_ke", F32, S)
            md.shape_material_kd_dev = _ptr(model.shape_material_kd, "model.shape_material_kd", F32, S)
            md.shape_material_mu_dev = _ptr(model.shape_material_mu, "model.shape_material_mu", F32, S)
            md.shape_body_dev = _ptr(model.shape_body, "model.shape_body", I32, S)
        md.body_com_dev = _ptr(getattr(model, "body_com", None), "model.body_com", F32)
        ns, nt = int(getattr(model, "spring_count", 0) or 0), int(getattr(model, "tet_count", 0) or 0)
        if ns:
            md.spring_count = ns
            md.spring_indices_dev = _ptr(model.spring_indices, "model.spring_indices", I32, 2 * ns)
            md.spring_rest_length_dev = _ptr(model.spring_rest_length, "model.spring_rest_length", F32, ns)
            md.spring_stiffness_dev = _ptr(model.spring_stiffness, "model.spring_stiffness", F32, ns)
            md.spring_damping_dev = _ptr(model.spring_damping, "model.spring_damping", F32, ns)
        if nt:
            md.tet_count = nt
            md.tet_indices_dev = _ptr(model.tet_indices, "model.tet_indices", I32, 4 * nt)
            md.tet_poses_dev = _ptr(model.tet_poses, "model.tet_poses", F32, 9 * nt)
            md.tet_materials_dev = _ptr(model.tet_materials, "model.tet_materials", F32, at_least=3 * nt)
        self._md = md

        prm = _lib.VbdSolverParams()
        prm.iterations = int(iterations)
        prm.friction_epsilon = float(friction_epsilon)
        prm.avbd_linear_beta = float(linear_beta)
        prm.contact_k_start = float(rigid_contact_k_start)
        prm.precision = _lib.PRECISION[precision]
        prm.fp64_solve_threshold = float(fp64_solve_threshold)
        prm.schedule = _lib.SCHEDULE[schedule]
        prm.lanes_per_vertex = int(lanes_per_vertex)
        prm.block_size = int(block_size)
        prm.contact_slots = int(contact_slots)
        prm.positions_in_shared = {"auto": 0, "off": 1, "on": 2}[positions_in_shared]
        prm.layout = _lib.LAYOUT[layout]
        prm.min_blocks_per_sm = int(min_blocks_per_sm)
        prm.pair_vertices = int(bool(pair_vertices))
        prm.instance_per_warp = int(bool(instance_per_warp))
        self._prm = prm

        h = C.c_void_p()
        with torch.cuda.device(self.device):
            rc = self._lib.vbd_create(C.byref(md), C.byref(prm), C.byref(h))
        if rc == _lib.VBD_ERR_EMPTY_COLORING:
            raise ValueError("model.particle_color_groups is empty")
        _lib.check(rc, "vbd_create")
        self._h = h
        s, lanes, blk, smem, lay = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        self._lib.vbd_get_config(h, C.byref(s), C.byref(lanes), C.byref(blk), C.byref(smem), C.byref(lay))
        self.layout = _lib.LAYOUT_NAME[lay.value]
        self.schedule = _lib.SCHEDULE_NAME[s.value]
        self.lanes_per_vertex = lanes.value
        self.block_size = blk.value
        self.shared_bytes = smem.value
        if particle_enable_self_contact:
            self._set_self_contact(
                particle_vertex_contact_buffer_size, particle_edge_contact_buffer_size, particle_edge_parallel_epsilon,
                particle_external_vertex_contact_filtering_map, particle_external_edge_contact_filtering_map,
            )  # fmt: skip
        n = C.c_int32()
        self._lib.vbd_launches_per_step(h, C.byref(n))
        self.launches_per_step = n.value

    def _set_self_contact(self, vertex_buffer, edge_buffer, edge_eps, external_vertex_map, external_edge_map):
        """Collision filters and detector set-up of ``_init_particle_system`` (solver_vbd.py:489-526,
        1339-1404), handed to ``vbd_set_self_contact``."""
        from .collision import build_contact_filters

        m = self.model
        vt = ee = None
        if m.tri_count:
            vt, ee = build_contact_filters(
                m.particle_count, m.tri_indices, m.edge_indices, self.particle_topological_contact_filter_threshold,
                external_vertex_map, external_edge_map,
            )  # fmt: skip
        self._filters = (vt, ee)  # kept alive while the call copies them
        d = _lib.VbdSelfContactDesc()
        d.radius = float(self.particle_self_contact_radius)
        d.margin = float(self.particle_self_contact_margin)
        d.relaxation = float(self.particle_conservative_bound_relaxation)
        d.edge_parallel_epsilon = float(edge_eps)
        d.rest_exclusion_radius = float(self.particle_rest_shape_contact_exclusion_radius)
        d.vertex_buffer_size = int(vertex_buffer)
        d.edge_buffer_size = int(edge_buffer)
        d.detection_interval = int(self.particle_collision_detection_interval)
        self._rest_q = interop.as_torch(m.particle_q, self.device).detach().to(torch.float32).contiguous()
        d.rest_q_dev = _ptr(self._rest_q, "model.particle_q", F32, 3 * m.particle_count)
        ip = C.POINTER(C.c_int32)
        if vt is not None:
            d.vt_filter_host, d.vt_filter_offsets_host = vt[0].ctypes.data_as(ip), vt[1].ctypes.data_as(ip)
        if ee is not None:
            d.ee_filter_host, d.ee_filter_offsets_host = ee[0].ctypes.data_as(ip), ee[1].ctypes.data_as(ip)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.vbd_set_self_contact(self._h, C.byref(d)), "vbd_set_self_contact")

    def self_contact_counts(self) -> tuple[int, int, int]:
        """(vertex-triangle pairs, edge-edge pairs, overflow flags) of the last detection of the last step."""
        nv, ne, fl = C.c_int32(), C.c_int32(), C.c_int32()
        stream = self._stream()
        _lib.check(self._lib.vbd_get_self_contact_counts(self._h, C.byref(nv), C.byref(ne), C.byref(fl), stream),
                   "vbd_get_self_contact_counts")  # fmt: skip
        return nv.value, ne.value, fl.value

    # ------------------------------------------------------------------ reference API
    def _stream(self):
        return C.c_void_p(interop.launch_stream(self.device, self._warp))

    def step(self, state_in: State, state_out: State, control, contacts: Contacts | None, dt: float) -> None:
        n3 = 3 * int(self.model.particle_count)
        want = F64 if self.precision == "fp64" else F32
        q_in = _ptr(state_in.particle_q, "state_in.particle_q", want, n3)
        q_out = _ptr(state_out.particle_q, "state_out.particle_q", want, n3)
        qd_in = _ptr(state_in.particle_qd, "state_in.particle_qd", want, n3)
        qd_out = _ptr(state_out.particle_qd, "state_out.particle_qd", want, n3)
        for name, p in (("state_in.particle_q", q_in), ("state_out.particle_q", q_out),
                        ("state_in.particle_qd", qd_in), ("state_out.particle_qd", qd_out)):  # fmt: skip
            if p is None:
                raise TypeError(f"{name} must be a device array of particle_count x 3 values")
        f = _ptr(getattr(state_in, "particle_f", None), "state_in.particle_f", want, n3)
        cdesc = contacts_desc(contacts, self.model)
        bodies = None
        if getattr(state_in, "body_q", None) is not None:
            bodies = _lib.VbdBodyState()
            if self.integrate_with_external_rigid_solver:
                bodies.body_q_dev = _ptr(state_out.body_q, "state_out.body_q", F32)
                bodies.body_q_prev_dev = _ptr(state_in.body_q, "state_in.body_q", F32)
                bodies.body_qd_dev = _ptr(state_out.body_qd, "state_out.body_qd", F32)
            else:
                bodies.body_q_dev = _ptr(state_in.body_q, "state_in.body_q", F32)
                bodies.body_qd_dev = _ptr(state_in.body_qd, "state_in.body_qd", F32)
        fn = self._lib.vbd_step_f64 if self.precision == "fp64" else self._lib.vbd_step
        rc = fn(self._h, q_in, q_out, qd_in, qd_out, f, None if cdesc is None else C.byref(cdesc),
                None if bodies is None else C.byref(bodies), float(dt), self._stream())  # fmt: skip
        if rc == _lib.VBD_ERR_UNSUPPORTED:
            raise RuntimeError("contact buffers must grow while a CUDA graph is being captured; step once before capturing")
        _lib.check(rc, "vbd_step")

    def notify_model_changed(self, flags: int = 0) -> None:
        stream = self._stream()
        _lib.check(self._lib.vbd_refresh_model(self._h, stream), "vbd_refresh_model")

    def rebuild_bvh(self, state: State) -> None:
        """The reference rebuilds its self-contact BVHs here. This solver's detector rebuilds its grid
        at every detection, so there is nothing to do."""

    @staticmethod
    def register_custom_attributes(builder) -> None:
        """The reference registers rigid-body Dahl-friction attributes here; cloth needs none."""

    # ------------------------------------------------------------------ diagnostics
    def device_errors(self) -> int:
        bits = C.c_int32()
        stream = self._stream()
        _lib.check(self._lib.vbd_get_error(self._h, C.byref(bits), stream), "vbd_get_error")
        return bits.value

    def residuals(self) -> np.ndarray:
        """FP64 per-iteration sums of |f|^2 of the last step (precision='mixed')."""
        out = np.zeros(max(self.iterations, 1), dtype=np.float64)
        stream = self._stream()
        _lib.check(self._lib.vbd_get_residuals(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), self.iterations,
                                               stream), "vbd_get_residuals")  # fmt: skip
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.vbd_destroy(h)
            except Exception:
                pass
            self._h = None
