"""ctypes binding of ``libvbd_b200.so`` (C ABI: ``include/vbd_b200.h``).

The library is built in-tree by ``newton_chysx_b200.build`` (``__graft_entry__.build()``). Loading
fails loudly when it is missing: there is no CPU or Python fallback for the solver.
"""

from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvbd_b200.so")

VBD_OK = 0
VBD_ERR_INVALID_ARGUMENT = -1
VBD_ERR_CUDA = -2
VBD_ERR_OUT_OF_MEMORY = -3
VBD_ERR_UNSUPPORTED = -4
VBD_ERR_EMPTY_COLORING = -5
VBD_ERR_TOO_LARGE = -6
VBD_NOALLOC_MAX_PARTICLES = 32768
VBD_NOALLOC_MAX_CONTACT_SLOTS = 4

VBD_DEVERR_NONFINITE = 1
VBD_DEVERR_CONTACT_OVERFLOW = 2
VBD_DEVERR_SINGULAR_SKIPPED = 4
VBD_DEVERR_BAD_CONTACT = 8

PRECISION = {"fp32": 0, "mixed": 1, "fp64": 2}
SCHEDULE = {"auto": 0, "per_color": 1, "persistent": 2}
SCHEDULE_NAME = {v: k for k, v in SCHEDULE.items()}
LAYOUT = {"auto": 0, "csr": 1, "ell": 2, "ell16": 3, "ring": 4}
LAYOUT_NAME = {v: k for k, v in LAYOUT.items()}

_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p


class VbdModelDesc(C.Structure):
    _fields_ = [
        ("particle_count", C.c_int32), ("tri_count", C.c_int32), ("edge_count", C.c_int32), ("shape_count", C.c_int32),
        ("particle_mass_dev", _vp), ("particle_inv_mass_dev", _vp), ("particle_flags_dev", _vp),
        ("particle_radius_dev", _vp),
        ("tri_indices_dev", _vp), ("tri_poses_dev", _vp), ("tri_materials_dev", _vp), ("tri_areas_dev", _vp),
        ("edge_indices_dev", _vp), ("edge_rest_angle_dev", _vp), ("edge_rest_length_dev", _vp),
        ("edge_bending_properties_dev", _vp),
        ("color_count", C.c_int32), ("color_offsets_host", _ip), ("color_particles_dev", _vp),
        ("world_count", C.c_int32), ("world_particle_start_host", _ip),
        ("gravity_dev", _vp),
        ("soft_contact_ke", C.c_float), ("soft_contact_kd", C.c_float), ("soft_contact_mu", C.c_float),
        ("shape_material_ke_dev", _vp), ("shape_material_kd_dev", _vp), ("shape_material_mu_dev", _vp),
        ("shape_body_dev", _vp), ("body_com_dev", _vp),
        ("spring_count", C.c_int32), ("spring_indices_dev", _vp), ("spring_rest_length_dev", _vp),
        ("spring_stiffness_dev", _vp), ("spring_damping_dev", _vp),
        ("tet_count", C.c_int32), ("tet_indices_dev", _vp), ("tet_poses_dev", _vp), ("tet_materials_dev", _vp),
    ]  # fmt: skip


class VbdSolverParams(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("friction_epsilon", C.c_float), ("avbd_linear_beta", C.c_float),
        ("contact_k_start", C.c_float), ("precision", C.c_int32), ("fp64_solve_threshold", C.c_float),
        ("schedule", C.c_int32), ("lanes_per_vertex", C.c_int32), ("block_size", C.c_int32),
        ("contact_slots", C.c_int32), ("positions_in_shared", C.c_int32), ("layout", C.c_int32),
        ("min_blocks_per_sm", C.c_int32), ("pair_vertices", C.c_int32),
        ("instance_per_warp", C.c_int32),
    ]  # fmt: skip


class VbdContactsDesc(C.Structure):
    _fields_ = [
        ("soft_contact_count_dev", _vp), ("soft_contact_max", C.c_int32), ("soft_contact_particle_dev", _vp),
        ("soft_contact_shape_dev", _vp), ("soft_contact_body_pos_dev", _vp), ("soft_contact_body_vel_dev", _vp),
        ("soft_contact_normal_dev", _vp),
    ]  # fmt: skip


class VbdBodyState(C.Structure):
    _fields_ = [("body_q_dev", _vp), ("body_q_prev_dev", _vp), ("body_qd_dev", _vp)]


class VbdHeightfield(C.Structure):
    _fields_ = [("data_offset", C.c_int32), ("nrow", C.c_int32), ("ncol", C.c_int32), ("hx", C.c_float),
                ("hy", C.c_float), ("min_z", C.c_float), ("max_z", C.c_float)]  # fmt: skip


class VbdShapeTable(C.Structure):
    _fields_ = [
        ("shape_count", C.c_int32), ("shape_type_host", _ip), ("shape_transform_host", _fp),
        ("shape_scale_host", _fp), ("shape_heightfield_index_host", _ip), ("heightfield_count", C.c_int32),
        ("heightfields_host", C.POINTER(VbdHeightfield)), ("elevations_dev", _vp), ("elevation_count", C.c_int64),
        ("shape_mesh_host", C.POINTER(_vp)), ("shape_flags_host", _ip), ("shape_world_host", _ip),
        ("particle_world_dev", _vp), ("shape_body_host", _ip), ("body_count", C.c_int32), ("body_q_dev", _vp),
    ]  # fmt: skip


class VbdRefAdjacency(C.Structure):
    _fields_ = [("face_offsets_dev", _vp), ("faces_dev", _vp), ("edge_offsets_dev", _vp), ("edges_dev", _vp)]


class VbdSelfContactDesc(C.Structure):
    _fields_ = [
        ("radius", C.c_double), ("margin", C.c_double), ("relaxation", C.c_double),
        ("edge_parallel_epsilon", C.c_double), ("rest_exclusion_radius", C.c_double),
        ("vertex_buffer_size", C.c_int32), ("edge_buffer_size", C.c_int32), ("detection_interval", C.c_int32),
        ("rest_q_dev", _vp), ("vt_filter_offsets_host", _ip), ("vt_filter_host", _ip),
        ("ee_filter_offsets_host", _ip), ("ee_filter_host", _ip),
    ]  # fmt: skip


# every symbol the header declares, with its ctypes signature
SIGNATURES = {
    "vbd_create": ([C.POINTER(VbdModelDesc), C.POINTER(VbdSolverParams), C.POINTER(_vp)], C.c_int),
    "vbd_refresh_model": ([_vp, _vp], C.c_int),
    "vbd_step": (
        [_vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(VbdContactsDesc), C.POINTER(VbdBodyState), C.c_float, _vp],
        C.c_int,
    ),
    "vbd_step_f64": (
        [_vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(VbdContactsDesc), C.POINTER(VbdBodyState), C.c_double, _vp],
        C.c_int,
    ),
    "vbd_record_step": ([_vp, _vp, _vp, _vp, _vp, C.c_double, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "vbd_adjoint_step": ([_vp, _vp, _vp, _vp, _vp, C.c_double, _vp, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "vbd_get_error": ([_vp, _ip, _vp], C.c_int),
    "vbd_get_residuals": ([_vp, _dp, C.c_int32, _vp], C.c_int),
    "vbd_launches_per_step": ([_vp, _ip], C.c_int),
    "vbd_get_config": ([_vp, _ip, _ip, _ip, _ip, _ip], C.c_int),
    "vbd_destroy": ([_vp], C.c_int),
    "vbd_color_particles": (
        [C.c_int32, C.c_int32, _ip, _fp, C.c_int32, _ip, _fp, C.c_int32, C.c_float, _ip],
        C.c_int,
    ),
    "vbd_color_graph": ([C.c_int32, C.c_int32, _ip, C.c_int32, C.c_float, _ip], C.c_int),
    "vbd_build_adjacency": ([C.c_int32, C.c_int32, _ip, C.c_int32, _ip, _ip, _ip, _ip, _ip], C.c_int),
    "vbd_step_noalloc": (
        [C.POINTER(VbdModelDesc), C.POINTER(VbdRefAdjacency), C.c_int32, C.c_float, _vp, _vp, _vp, _vp, _vp,
         C.POINTER(VbdContactsDesc), C.c_float, _vp],
        C.c_int,
    ),
    "vbd_step_noalloc_error": ([_ip, _vp], C.c_int),
    "vbd_eval_atan2": ([C.c_int32, _vp, _vp, _vp, _vp], C.c_int),
    "vbd_set_self_contact": ([_vp, C.POINTER(VbdSelfContactDesc)], C.c_int),
    "vbd_get_self_contact_counts": ([_vp, _ip, _ip, _ip, _vp], C.c_int),
    "vbd_build_contact_filters": ([C.c_int32, C.c_int32, _ip, C.c_int32, _ip, C.c_int32, _ip, _ip, _ip, _ip], C.c_int),
    "vbd_collider_create": (
        [C.c_int32, C.c_int32, _vp, C.c_int32, _vp, C.c_int32, C.c_int32, C.c_float, _ip, _ip, _ip, _ip, C.POINTER(_vp)],
        C.c_int,
    ),
    "vbd_collider_set_triangle_buffers": ([_vp, C.c_int32, _vp, _vp, _vp], C.c_int),
    "vbd_collider_detect": (
        [_vp, C.c_int32, _vp, C.c_float, C.c_float, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
        C.c_int,
    ),
    "vbd_collider_destroy": ([_vp], C.c_int),
    "vbd_soft_contacts_shapes": (
        [C.c_int32, _vp, _vp, _vp, C.c_int32, _ip, _fp, _fp, C.c_float, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
        C.c_int,
    ),
    "vbd_soft_contacts_table": (
        [C.c_int32, _vp, _vp, _vp, C.POINTER(VbdShapeTable), C.c_float, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
        C.c_int,
    ),
    "vbd_mesh_create": ([_fp, C.c_int32, _ip, C.c_int32, C.POINTER(_vp)], C.c_int),
    "vbd_shape_set_create": ([C.POINTER(VbdShapeTable), C.POINTER(_vp)], C.c_int),
    "vbd_shape_set_destroy": ([_vp], C.c_int),
    "vbd_shape_set_use_parameter_table": ([_vp, C.c_int32], C.c_int),
    "vbd_soft_contacts_set": (
        [_vp, C.c_int32, _vp, _vp, _vp, _vp, _vp, C.c_float, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
        C.c_int,
    ),
    "vbd_mesh_destroy": ([_vp], C.c_int),
    "vbd_soft_contacts": (
        [C.c_int32, _vp, _vp, _vp, C.c_int32, _ip, _fp, _fp, _fp, C.c_float, C.c_int32, _vp, _vp, _vp, _vp, _vp,
         _vp, _vp],
        C.c_int,
    ),
}

_lib = None


class VbdError(RuntimeError):
    pass


def load():
    """Load the CUDA library; raise ImportError if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "(there is no CPU fallback for the VBD solver)"
            )
        lib = C.CDLL(LIB_PATH)
        for name, (argtypes, restype) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = restype
        _lib = lib
    return _lib


def check(rc: int, what: str):
    if rc == VBD_OK:
        return
    names = {
        VBD_ERR_INVALID_ARGUMENT: "invalid argument",
        VBD_ERR_CUDA: "CUDA error",
        VBD_ERR_OUT_OF_MEMORY: "out of device memory",
        VBD_ERR_UNSUPPORTED: "unsupported",
        VBD_ERR_EMPTY_COLORING: "empty coloring",
        VBD_ERR_TOO_LARGE: "model too large for the fixed buffers",
    }
    raise VbdError(f"{what} failed: {names.get(rc, rc)} ({rc})")
