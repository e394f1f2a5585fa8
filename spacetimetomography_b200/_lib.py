"""ctypes binding of libstt.so (the C ABI declared in include/stt.h).

The CUDA library is the only implementation: importing this module without a
built ``libstt.so`` raises, and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libstt.so"


class STTError(RuntimeError):
    """A libstt call returned a non-zero stt_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"stt status {status}: {message}")
        self.status = status


STATUS = {0: "STT_OK", 1: "STT_ERR_INVALID", 2: "STT_ERR_CUDA", 3: "STT_ERR_NOMEM",
          4: "STT_ERR_STATE", 5: "STT_ERR_UNSUPPORTED", 6: "STT_ERR_TIMEOUT"}


class Geometry(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("sx", C.c_double), ("sy", C.c_double), ("sz", C.c_double),
                ("W", C.c_int), ("H", C.c_int), ("ds", C.c_double),
                ("sid", C.c_double), ("sdd", C.c_double), ("off", C.c_double * 3),
                ("n_views", C.c_int), ("angles_rad", C.POINTER(C.c_double))]


class PdParams(C.Structure):
    _fields_ = [("sigma", C.c_float), ("tau", C.c_float), ("tv_w", C.c_float),
                ("tp_w", C.c_float), ("bc_w", C.c_float), ("huber_factor", C.c_float),
                ("gmax", C.c_float), ("cut", C.c_int * 8)]


class SolveCfg(C.Structure):
    _fields_ = [("n_frames", C.c_int), ("views_per_frame", C.c_int), ("bp_mode", C.c_int),
                ("alpha", C.c_double), ("pd", PdParams), ("roi_cut", C.c_int * 8),
                ("seed", C.c_ulonglong), ("mode", C.c_int), ("halo", C.c_int), ("frame_offset", C.c_int),
                ("total_frames", C.c_int), ("autotune", C.c_int), ("storage", C.c_int)]


class PdState(C.Structure):
    _fields_ = [("vol", C.c_void_p), ("xbar", C.c_void_p), ("xprev", C.c_void_p),
                ("ytv", C.c_void_p), ("ytp", C.c_void_p), ("ybc", C.c_void_p),
                ("flow", C.c_void_p), ("proj", C.c_void_p), ("ytp_halo", C.c_void_p),
                ("ybc_halo", C.c_void_p), ("flow_halo", C.c_void_p)]


class FlowParams(C.Structure):
    _fields_ = [("tol", C.c_float), ("lam", C.c_float), ("huber", C.c_float), ("eta", C.c_float),
                ("sigma", C.c_float), ("max_iter", C.c_int), ("norm", C.c_int), ("n_warps", C.c_int),
                ("scales", C.c_int), ("cut", C.c_int * 6)]


class OpNorm(C.Structure):
    _fields_ = [("norm_A", C.c_double), ("norm_K", C.c_double), ("sigma", C.c_double), ("tau", C.c_double),
                ("iterations", C.c_int), ("rel_change", C.c_double)]


class Instance(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("vol", C.c_void_p), ("proj", C.c_void_p), ("n_views", C.c_int),
                ("bp_mode", C.c_int), ("alpha", C.c_double), ("pd", PdParams), ("roi_cut", C.c_int * 8),
                ("seed", C.c_ulonglong), ("autotune", C.c_int), ("storage", C.c_int)]


class Tuning(C.Structure):
    """stt_tuning (include/stt.h): launch choices and the autotuner's timings."""
    _fields_ = [("fp_variant", C.c_int), ("slab_variant", C.c_int), ("bp_variant", C.c_int),
                ("staged_bins", C.c_uint), ("tuned", C.c_int), ("from_cache", C.c_int),
                ("fp_us", C.c_float * 12), ("slab_us", C.c_float * 8), ("bp_us", C.c_float * 8),
                ("ray_variant", C.c_int), ("ray_us", C.c_float * 2), ("staged_bins_bf16", C.c_uint),
                ("fp_variant_bf16", C.c_int), ("fp16_us", C.c_float * 2)]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is not built; run `python spacetimetomography_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    vp, i, d, f = C.c_void_p, C.c_int, C.c_double, C.c_float
    sigs = {
        "stt_create": [C.POINTER(vp), i],
        "stt_destroy": [vp],
        "stt_set_geometry": [vp, C.POINTER(Geometry)],
        "stt_views_from_rounds": [i, vp, i, d, vp],
        "stt_lds_angles": [i, i, i, i, vp],
        "stt_permutation": [C.c_ulonglong, i, vp],
        "stt_fp": [vp, vp, vp, vp, vp, i, i, vp],
        "stt_fp_correction": [vp, vp, vp, vp, vp, i, vp],
        "stt_fp_vjp": [vp, vp, vp, i, i, vp],
        "stt_bp_voxel": [vp, vp, vp, d, f, i, vp],
        "stt_bp_ray": [vp, vp, vp, f, i, vp],
        "stt_bp_ray_scatter": [vp, vp, vp, vp, i, vp],
        "stt_gather_ceiling": [vp, vp, i, i, vp, vp, vp],
        "stt_fp_texture_ok": [vp, vp, vp],
        "stt_fp_texture_ok_typed": [vp, vp, i, vp],
        "stt_sart_sweep_typed": [vp, vp, i, vp, vp, i, i, d, f, i, vp, vp, vp],
        "stt_bp_voxel_typed": [vp, vp, vp, i, d, f, i, vp],
        "stt_bp_ray_typed": [vp, vp, vp, i, f, i, vp],
        "stt_warp_typed": [vp, vp, vp, i, i, f, vp, vp],
        "stt_sart_sweep": [vp, vp, vp, vp, i, i, d, f, i, vp, vp, vp],
        "stt_pd_dual": [vp, C.POINTER(PdParams), vp, vp, vp, vp, vp, vp, vp],
        "stt_pd_primal": [vp, C.POINTER(PdParams), i, vp, vp, vp, vp, vp, vp, vp, vp],
        "stt_pd_extrapolate": [vp, vp, vp, vp, vp, vp],
        "stt_roi_mask": [vp, vp, vp, vp],
        "stt_warp": [vp, vp, vp, i, f, vp, vp],
        "stt_warp_vjp": [vp, vp, vp, i, f, vp, vp, vp, vp],
        "stt_solver_create": [vp, C.POINTER(SolveCfg), C.POINTER(PdState), C.POINTER(vp)],
        "stt_solver_iterate": [vp, i, vp],
        "stt_solver_iterate_phase": [vp, i, vp],
        "stt_solver_stats": [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_ulonglong)],
        "stt_solver_persistent_info": [vp, C.POINTER(i), C.POINTER(i)],
        "stt_solver_destroy": [vp],
        "stt_solver_frame_order": [C.c_ulonglong, C.c_ulonglong, i, i, i, vp],
        "stt_fp_typed": [vp, vp, i, vp, vp, vp, i, i, vp],
        "stt_sart_view": [vp, vp, vp, i, d, f, i, vp, vp],
        "stt_opnorm_power_iter": [vp, i, C.c_ulonglong, C.POINTER(OpNorm), vp],
        "stt_batch_create": [vp, i, i, C.POINTER(vp)],
        "stt_batch_iterate": [vp, i, vp],
        "stt_batch_destroy": [vp],
        "stt_batch_staging": [vp, vp, vp, vp, vp],
        "stt_ctx_dims": [vp, vp],
        "stt_warp_box": [vp, vp, vp, vp, i, f, vp, vp],
        "stt_image_gradient": [vp, vp, vp, vp],
        "stt_flow_create": [i, vp, C.POINTER(FlowParams), C.POINTER(vp)],
        "stt_flow_destroy": [vp],
        "stt_flow_multiscale": [vp, vp, vp, vp, vp, vp],
        "stt_flow_level": [vp, vp, vp, vp, vp, vp, vp, vp, vp],
        "stt_flow_stats": [vp, C.POINTER(i), vp, vp],
        "stt_flow_blur": [vp, vp, i, f, vp, vp],
        "stt_flow_resize": [vp, vp, i, vp, vp, vp, vp],
        "stt_poll_status": [vp, vp],
        "stt_solver_poll_status": [vp, vp],
        "stt_batch_poll_status": [vp, vp],
        "stt_warp_poll_status": [vp],
        "stt_autotune": [vp, C.POINTER(Tuning), vp],
        "stt_get_tuning": [vp, C.POINTER(Tuning)],
        "stt_set_tuning": [vp, C.POINTER(Tuning)],
        "stt_solver_set_iteration": [vp, C.c_ulonglong, vp],
    }
    for name, argtypes in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = C.c_int
    lib.stt_last_error.argtypes = [vp]
    lib.stt_last_error.restype = C.c_char_p
    lib.stt_solver_last_error.argtypes = [vp]
    lib.stt_solver_last_error.restype = C.c_char_p
    lib.stt_batch_last_error.argtypes = [vp]
    lib.stt_batch_last_error.restype = C.c_char_p
    lib.stt_flow_last_error.argtypes = [vp]
    lib.stt_flow_last_error.restype = C.c_char_p
    lib.stt_tuning_variant_name.argtypes = [i, i]
    lib.stt_tuning_variant_name.restype = C.c_char_p
    lib.stt_version.argtypes = []
    lib.stt_version.restype = C.c_char_p
    return lib


lib = _load()


def check(status: int, ctx=None) -> None:
    if status != 0:
        msg = lib.stt_last_error(ctx)
        raise STTError(status, (msg or b"").decode(errors="replace"))
