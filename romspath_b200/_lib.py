"""ctypes declarations of the C ABI in ``include/romspath_gpu.h``.

Loading fails loudly: there is no CPU fallback for the particle step.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

MAXNGRID = 5
NOALLOC_MAX_PARTICLES = 1048576
RP_OK = 0
ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_UNSUPPORTED, ERR_NOEXT = -1, -2, -3, -4, -5, -6
ERRORS = {-1: "RP_ERR_ARG", -2: "RP_ERR_CUDA", -3: "RP_ERR_STATE", -4: "RP_ERR_NOMEM",
          -5: "RP_ERR_UNSUPPORTED", -6: "RP_ERR_NOEXT"}
FIELD_F64, FIELD_F32, FIELD_MIXED, FIELD_MIXED_I16 = 0, 1, 2, 3
FLAG_OOB, FLAG_NODE, FLAG_WBOT, FLAG_WTOP, FLAG_SPLINE = 1, 2, 4, 8, 16
DIAG_SALTTEMP, DIAG_SALTTEMP_MEAN, DIAG_BOTTOM = 1, 2, 4

EXPORTS = [
    "rp_create", "rp_upload_frame", "rp_upload_frame_f32", "rp_set_particles", "rp_locate_particles",
    "rp_step", "rp_get_particles", "rp_set_id_base", "rp_set_step_index", "rp_set_noise_hook", "rp_synchronize",
    "rp_last_error", "rp_destroy", "rp_device_state_get", "rp_last_step_stats", "rp_kernel_launches",
    "rp_step_noalloc", "rp_version", "rp_adj_frames", "rp_adj_set_frame", "rp_forward", "rp_backward",
    "rp_tangent", "rp_adj_replay", "rp_step_n", "rp_set_launch", "rp_upload_frame_ext", "rp_upload_frame_ext_f32",
    "rp_get_diagnostics", "rp_reset_diagnostics", "rp_set_grid_lonlat", "rp_output_record", "rp_upload_frame_desc",
    "rp_set_behavior", "rp_get_behavior", "rp_set_grid_angle", "rp_locate_lonlat", "rp_nest_maps",
    "rp_output_record_async", "rp_output_wait", "rp_count_spline_passes", "rp_spline_pass_counts",
    "rp_set_kernel_form",
]

PD = C.POINTER(C.c_double)
PF = C.POINTER(C.c_float)
PI32 = C.POINTER(C.c_int32)
PU32 = C.POINTER(C.c_uint32)


class RpParams(C.Structure):
    _fields_ = [
        ("numpar", C.c_int32), ("idt", C.c_int32), ("dt", C.c_int32), ("scheme", C.c_int32),
        ("nsb", C.c_int32), ("vturb_on", C.c_int32), ("hturb_on", C.c_int32),
        ("open_ocean_boundary", C.c_int32), ("behavior", C.c_int32), ("stokes", C.c_int32),
        ("field_dtype", C.c_int32), ("spline_max_iter", C.c_int32),
        ("vertdist", C.c_double), ("serr", C.c_double), ("smth", C.c_double), ("sub", C.c_double),
        ("deltat", C.c_double), ("aksback", C.c_double),
        ("constant_hturb", C.c_double * MAXNGRID),
        ("seed", C.c_uint64), ("device", C.c_int32), ("reserved", C.c_int32 * 7),
    ]


class RpFrame(C.Structure):
    _fields_ = [("f32", C.c_int32)] + [(k, C.c_void_p) for k in (
        "zeta", "u", "v", "w", "aks", "su", "sv", "salt", "temp", "bustr", "bvstr")] + [
        (k, PD) for k in ("wetdry_rho", "wetdry_u", "wetdry_v")] + [
        (k, C.c_void_p) for k in ("turbaccel", "turbvort", "waveaccelu", "waveaccelv")]


FUCHS = ("vort_cr", "vort_sat", "b0pv", "b1pv", "b0wv", "b1w", "acc_cr", "acc_sat", "b0pa", "b1pa", "b0wa")


class RpBehavior(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("behavior", "process_va", "process_wa", "va_flag")] + [
        ("swimfast", C.c_double), ("initsize", C.c_double)] + [(k, C.c_double) for k in FUCHS]


class RpGrid(C.Structure):
    _fields_ = [
        ("xi_rho", C.c_int32), ("eta_rho", C.c_int32), ("n_rho", C.c_int32), ("vtransform", C.c_int32),
        ("hc", C.c_double),
        ("h", PD), ("pm", PD), ("pn", PD),
        ("mask_rho", PI32), ("mask_u", PI32), ("mask_v", PI32),
        ("s_rho", PD), ("cs_r", PD), ("s_w", PD), ("cs_w", PD),
        ("scl", PD), ("off", PD),
    ]


class RpAdjStep(C.Structure):
    _fields_ = [
        ("ex", C.c_double * 3), ("ix", C.c_double * 3), ("ets", C.c_int32),
        ("frame_b", C.c_int32), ("frame_c", C.c_int32), ("frame_f", C.c_int32), ("step_index", C.c_uint64),
    ]


class RpDeviceState(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("age", C.c_void_p), ("dob", C.c_void_p),
        ("status", C.c_void_p), ("wd", C.c_void_p), ("zeta", C.c_void_p), ("bath", C.c_void_p),
        ("gid", C.c_void_p), ("isin", C.c_void_p), ("pid", C.c_void_p), ("flags", C.c_void_p),
        ("stream", C.c_void_p),
    ]


_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the sm_100a library (building it with nvcc if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"romspath_b200: CUDA library missing at {path}")
        _build.build()
    L = C.CDLL(path)
    _declare(L)
    _lib = L
    return L


def _declare(L):
    P = C.c_void_p
    L.rp_create.argtypes = [C.POINTER(RpParams), C.c_int32, C.POINTER(RpGrid), C.POINTER(P)]
    L.rp_upload_frame.argtypes = [P, C.c_int32, C.c_int32] + [PD] * 7
    L.rp_upload_frame_f32.argtypes = [P, C.c_int32, C.c_int32] + [PF] * 7
    L.rp_upload_frame_ext.argtypes = [P, C.c_int32, C.c_int32] + [PD] * 11
    L.rp_upload_frame_ext_f32.argtypes = [P, C.c_int32, C.c_int32] + [PF] * 11
    L.rp_get_diagnostics.argtypes = [P, C.c_int64] + [PD] * 7
    L.rp_reset_diagnostics.argtypes = [P]
    L.rp_set_grid_lonlat.argtypes = [P, C.c_int32, PD, PD]
    L.rp_upload_frame_desc.argtypes = [P, C.c_int32, C.c_int32, C.POINTER(RpFrame)]
    L.rp_set_behavior.argtypes = [P, C.POINTER(RpBehavior)]
    L.rp_set_grid_angle.argtypes = [P, C.c_int32, PD, C.c_int32]
    L.rp_locate_lonlat.argtypes = [P, C.c_int64, PD, PD, PD, PD, C.c_int32, PD, PD]
    L.rp_nest_maps.argtypes = [C.c_int32, PI32, PI32, C.POINTER(PD), C.POINTER(PD), PD, PD, PD]
    L.rp_get_behavior.argtypes = [P, C.c_int64] + [PD] * 4
    L.rp_output_record.argtypes = [P, C.c_int64, C.c_int32] + [PD] * 11
    L.rp_output_record_async.argtypes = [P, C.c_int64, C.c_int32] + [PD] * 11
    L.rp_output_wait.argtypes = [P]
    L.rp_set_particles.argtypes = [P, C.c_int64] + [PD] * 7 + [PI32]
    L.rp_locate_particles.argtypes = [P, C.c_int64, PD, PD, PD, PD, C.c_int32]
    L.rp_step.argtypes = [P, PD, PD, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    L.rp_get_particles.argtypes = [P, C.c_int64] + [PD] * 6 + [PI32, PD, PD, PD, PU32]
    L.rp_set_step_index.argtypes = [P, C.c_uint64]
    L.rp_set_id_base.argtypes = [P, C.c_uint32]
    L.rp_set_noise_hook.argtypes = [P, PD, C.c_int64]
    L.rp_synchronize.argtypes = [P]
    L.rp_last_error.argtypes = [P, C.c_char_p, C.c_int32]
    L.rp_destroy.argtypes = [P]
    L.rp_device_state_get.argtypes = [P, C.POINTER(RpDeviceState)]
    L.rp_last_step_stats.argtypes = [P, C.POINTER(C.c_float), C.POINTER(C.c_int32)]
    L.rp_kernel_launches.argtypes = [P, C.POINTER(C.c_int64)]
    L.rp_count_spline_passes.argtypes = [P, C.c_int32]
    L.rp_spline_pass_counts.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.rp_step_noalloc.argtypes = [P, C.POINTER(RpDeviceState), PD, PD, C.c_int32, C.c_int32, C.c_int32,
                                  C.c_int32]
    L.rp_step_n.argtypes = [P, C.c_int32, PD, PD, PI32, PI32, PI32, PI32]
    L.rp_set_launch.argtypes = [P, C.c_int32, C.c_int32]
    L.rp_set_kernel_form.argtypes = [P, C.c_int32]
    L.rp_adj_frames.argtypes = [P, C.c_int32]
    L.rp_adj_set_frame.argtypes = [P, C.c_int32, C.c_int32] + [PD] * 7
    L.rp_forward.argtypes = [P, C.c_int32, C.POINTER(RpAdjStep), C.c_double, C.c_int32]
    L.rp_backward.argtypes = [P] + [PD] * 6 + [PD]
    L.rp_tangent.argtypes = [P, C.c_double, PD]
    L.rp_adj_replay.argtypes = [P, PD, PD, PD, C.c_double, PD, PD, PD]
    L.rp_version.restype = C.c_char_p
    for name in EXPORTS:
        if name != "rp_version":
            getattr(L, name).restype = C.c_int
