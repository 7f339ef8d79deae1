"""ctypes binding of libsors_b200.so (the C ABI declared in include/sors_b200.h).

The CUDA library is the only compute path: when it cannot be loaded the
import raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

SORS_OK = 0
ERRORS = {1: "ARG", 2: "INVERTED", 3: "NOT_CONVERGED", 4: "PCG_BREAKDOWN", 5: "CUDA", 6: "OOM", 7: "LINESEARCH",
          8: "UNSUPPORTED"}


class SorsSettings(C.Structure):
    _fields_ = [
        ("time_stepping", C.c_int32),
        ("solver_method", C.c_int32),
        ("dt", C.c_double),
        ("substeps", C.c_int32),
        ("cfl", C.c_int32),
        ("grav", C.c_double * 3),
        ("damping_alpha", C.c_double),
        ("precision", C.c_int32),
        ("project_spd", C.c_int32),
        ("material", C.c_int32),
        ("newton_dx_tol", C.c_double),
        ("newton_res_tol", C.c_double),
        ("newton_max_iter", C.c_int32),
        ("pcg_rel_tol", C.c_double),
        ("pcg_max_iter", C.c_int32),
        ("device", C.c_int32),
        ("newton_predictor", C.c_int32),
        ("max_blocks", C.c_int32),
        ("newton_safeguard", C.c_int32),
        ("two_level", C.c_int32),
        ("linear_solver", C.c_int32),
        ("pressure_jac_exact", C.c_int32),
    ]


class SorsStepStats(C.Structure):
    _fields_ = [
        ("newton_iters", C.c_int32),
        ("pcg_iters", C.c_int32),
        ("substeps", C.c_int32),
        ("residual_norm", C.c_double),
        ("dx_norm", C.c_double),
    ]


class SorsKernelProfile(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("assemble_ms", "spmv_ms", "pcg_update_ms", "energy_ms", "assemble_bytes",
                                          "spmv_bytes", "pcg_update_bytes", "energy_bytes", "tl_restrict_ms",
                                          "tl_coarse_z_ms", "tl_restrict_bytes", "tl_coarse_z_bytes",
                                          "form_p_ms", "form_p_bytes", "assemble_grad_ms")]


# (name, restype, argtypes) of every exported symbol declared in include/sors_b200.h
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_h = C.c_void_p
SIGNATURES = [
    ("sors_default_settings", None, [C.POINTER(SorsSettings)]),
    ("sors_create", C.c_int, [_dp, C.c_int32, _ip, C.c_int32, C.c_int32, _dp, _dp, _dp, C.POINTER(SorsSettings),
                              C.POINTER(C.c_void_p)]),
    ("sors_destroy", None, [_h]),
    ("sors_last_error", C.c_int, [C.c_char_p, C.c_size_t]),
    ("sors_set_neumann", C.c_int, [_h, _ip, _dp]),
    ("sors_set_pressure_faces", C.c_int, [_h, _ip, C.c_int32, C.c_int32, _ip, C.c_int32]),
    ("sors_enable_vertex_force", C.c_int, [_h, C.c_int32]),
    ("sors_set_muscles", C.c_int, [_h, _ip, _dp, _dp, C.c_int32]),
    ("sors_set_material", C.c_int, [_h, _dp, _dp]),
    ("sors_set_plane_contact", C.c_int, [_h, _dp, _dp, C.c_int32, _ip, C.c_int32]),
    ("sors_set_disk_contact", C.c_int, [_h, _dp, _dp, _dp, C.c_int32, _ip, C.c_int32]),
    ("sors_set_disk_contact_groups", C.c_int, [_h, _dp, _dp, _dp, C.c_int32, _ip, _ip]),
    ("sors_set_disk", C.c_int, [_h, C.c_int32, _dp, _dp, C.c_double]),
    ("sors_set_max_distance", C.c_int, [_h, _ip, _ip, _dp, C.c_int32]),
    ("sors_held_pairs", C.c_int32, [_h, _ip, _dp, C.c_int32]),
    ("sors_adjoint_set_pairs", C.c_int, [_h, _ip, _dp, C.c_int32]),
    ("sors_active_contacts", C.c_int32, [_h]),
    ("sors_held_contacts", C.c_int32, [_h, _ip, _dp, C.c_int32]),
    ("sors_get_contact_state", C.c_int32, [_h, _ip, C.c_int32]),
    ("sors_set_contact_state", C.c_int, [_h, _ip, C.c_int32]),
    ("sors_adjoint_step", C.c_int, [_h, _dp, C.c_double, _dp, _ip, _dp, C.c_int32, _dp, _dp, _dp, _dp, _dp,
                                    C.POINTER(SorsStepStats)]),
    ("sors_adjoint_pressure_grad", C.c_int, [_h, _dp, C.c_int32]),
    ("sors_adjoint_step_cn", C.c_int, [_h, _dp, C.c_double, _dp, _dp, _ip, _dp, C.c_int32, _dp, _dp, _dp, _dp, _dp,
                                       _dp, C.POINTER(SorsStepStats)]),
    ("sors_get_prev_force", C.c_int, [_h, _dp]),
    ("sors_set_prev_force", C.c_int, [_h, _dp]),
    ("sors_set_actuation", C.c_int, [_h, C.c_char_p, _dp, C.c_int64]),
    ("sors_set_initial_deformation", C.c_int, [_h, _dp]),
    ("sors_set_initial_velocity", C.c_int, [_h, _dp]),
    ("sors_get_state", C.c_int, [_h, _dp, _dp]),
    ("sors_energy", C.c_int, [_h, _dp, C.c_double, _dp]),
    ("sors_gradient", C.c_int, [_h, _dp, C.c_double, _dp]),
    ("sors_hessian_bsr", C.c_int, [_h, _dp, C.c_double, _ip, _ip, _dp, _lp]),
    ("sors_elem_eval", C.c_int, [_h, _dp, C.c_int32, _dp, _dp, _dp]),
    ("sors_step", C.c_int, [_h, _dp, _dp, C.c_double, C.c_int32, C.POINTER(SorsStepStats)]),
    ("sors_step_device", C.c_int, [_h, C.c_void_p, C.c_double, C.c_int32, C.POINTER(SorsStepStats)]),
    ("sors_update_state", C.c_int, [_h, _dp, C.c_double]),
    ("sors_device_bytes", C.c_int64, [_h]),
    ("sors_sizes", C.c_int, [_h, _lp, _lp, _lp]),
    ("sors_profile_kernels", C.c_int, [_h, C.c_int32, C.POINTER(SorsKernelProfile)]),
    ("sors_kernel_launch_count", C.c_int64, []),
    ("sors_evaluation_count", C.c_int64, [_h, C.c_int32]),
    ("sors_set_assembly_variant", C.c_int, [_h, C.c_int32]),
    ("sors_assembly_chunks", C.c_int64, [_h]),
    ("sors_last_step_curvature", C.c_int, [_h, C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    ("sors_set_members", C.c_int, [_h, C.POINTER(C.c_int32), C.c_int32]),
    ("sors_elem_energy_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]),
    ("sors_stream", C.c_void_p, [_h]),
]

_lib = None


def lib_path() -> str:
    return _build.LIB


def load():
    """Load (building first when the sources are newer) libsors_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    if _build.needs_build():
        _build.build()
    path = _build.LIB
    if not os.path.exists(path):
        raise RuntimeError(f"libsors_b200.so not found at {path}; run `python -m sors_b200.build`")
    L = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    load().sors_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != SORS_OK:
        raise RuntimeError(last_error() or f"sors error {ERRORS.get(status, status)}")


def default_settings() -> SorsSettings:
    s = SorsSettings()
    load().sors_default_settings(C.byref(s))
    return s
