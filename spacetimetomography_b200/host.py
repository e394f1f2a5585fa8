"""Python side of the host-buffer entry points of libstt_facade.so
(include/stt_host.h): the space-time solve on volumes, flows and projection
stacks held in host memory, as a host application of the reference holds
them (ST_Tomography::Render's image phase, ST_Tomography.cpp:475-607).

Arrays are C-contiguous float32 host arrays (numpy, or torch CPU tensors --
pinned ones make the copies asynchronous), shapes as in api.py:
vol (F, nz, ny, nx), flow (F, 3, nz, ny, nx), proj (F, V, H, W).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import _PKG, Geometry, SolveCfg, STTError
from .api import REFERENCE_CUT, SOLVE_GRAPH, PdParams

FACADE_PATH = _PKG / "libstt_facade.so"
_lib = None


def facade():
    """libstt_facade.so (raises if it is not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not FACADE_PATH.exists():
            raise ImportError(f"{FACADE_PATH} is not built; run `python spacetimetomography_b200/build.py`")
        lib = C.CDLL(str(FACADE_PATH))
        vp, i = C.c_void_p, C.c_int
        for name, args in {"stt_host_set_device": [i],
                           "stt_host_solver_create": [C.POINTER(Geometry), C.POINTER(SolveCfg), i, C.POINTER(vp)],
                           "stt_host_solver_submit": [vp, vp, vp, vp, i, vp],
                           "stt_host_solver_wait": [vp], "stt_host_solver_pending": [vp],
                           "stt_host_solver_destroy": [vp]}.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = C.c_int
        lib.stt_host_last_error.argtypes = []
        lib.stt_host_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def _host_ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):  # torch CPU tensor
        if a.is_cuda or not a.is_contiguous() or a.dtype.itemsize != 4:
            raise ValueError("host arrays must be contiguous float32 CPU tensors")
        return C.c_void_p(a.data_ptr())
    if not (a.flags["C_CONTIGUOUS"] and a.dtype == np.float32):
        raise ValueError("host arrays must be C-contiguous float32")
    return C.c_void_p(a.ctypes.data)


class HostSolver:
    """stt_host_solver: submit() enqueues one step (upload, n_iters
    iterations, read-back) on the next of `slots` device states; wait()
    completes the oldest pending step.  Keep the arrays of a step alive and
    unread until its wait().  `autotune` (stt_solve_cfg.autotune): the
    launch choices are timed on this geometry when the solver is created."""

    def __init__(self, dims, spacing, det, ds, sid, sdd, angles, n_frames, views_per_frame, pd: PdParams,
                 alpha=0.3, bp_mode=0, roi_cut=REFERENCE_CUT, seed=0, mode=SOLVE_GRAPH, slots=2, device=0,
                 offset=(0.0, 0.0, 0.0), autotune=True):
        lib = facade()
        self._ang = np.ascontiguousarray(angles, dtype=np.float64)
        g = Geometry(int(dims[0]), int(dims[1]), int(dims[2]), *map(float, spacing), int(det[0]), int(det[1]),
                     float(ds), float(sid), float(sdd), (C.c_double * 3)(*map(float, offset)), len(self._ang),
                     self._ang.ctypes.data_as(C.POINTER(C.c_double)))
        cfg = SolveCfg(n_frames, views_per_frame, bp_mode, float(alpha), pd.c(), (C.c_int * 8)(*map(int, roi_cut)),
                       C.c_ulonglong(seed), mode, 0, 0, 0, int(bool(autotune)))
        self._chk(lib.stt_host_set_device(int(device)))
        h = C.c_void_p()
        self._chk(lib.stt_host_solver_create(C.byref(g), C.byref(cfg), int(slots), C.byref(h)))
        self._h = h
        self._keep = []

    @staticmethod
    def _chk(rc):
        if rc != 0:
            raise STTError(rc, (facade().stt_host_last_error() or b"").decode(errors="replace"))

    def _trim(self):
        # the arrays of the pending steps, oldest first (submit may complete older steps itself)
        while len(self._keep) > self.pending():
            self._keep.pop(0)

    def submit(self, vol, flow, proj, n_iters=1, vol_out=None):
        self._keep.append((vol, flow, proj, vol_out))
        try:
            self._chk(facade().stt_host_solver_submit(self._h, _host_ptr(vol), _host_ptr(flow), _host_ptr(proj),
                                                      int(n_iters), _host_ptr(vol_out)))
        finally:
            self._trim()

    def wait(self):
        try:
            self._chk(facade().stt_host_solver_wait(self._h))
        finally:
            self._trim()

    def pending(self) -> int:
        return facade().stt_host_solver_pending(self._h)

    def close(self):
        if getattr(self, "_h", None):
            facade().stt_host_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
