"""ctypes bindings of the checkers: oracle/liboracle.so (CPU restatement) and,
when it was built, oracle/_ref/libstt_ref.so (the reference's own code).

Test infrastructure only: the product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_SO = ROOT / "oracle" / "liboracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libstt_ref.so"

P = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731


class OGeom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("sx", C.c_double),
                ("sy", C.c_double), ("sz", C.c_double), ("W", C.c_int), ("H", C.c_int),
                ("ds", C.c_double), ("sid", C.c_double), ("sdd", C.c_double),
                ("off", C.c_double * 3)]


class OView(C.Structure):
    _fields_ = [("angle", C.c_double), ("quat", C.c_float * 4)]


class OPd(C.Structure):
    _fields_ = [("sigma", C.c_float), ("tau", C.c_float), ("tv_w", C.c_float), ("tp_w", C.c_float),
                ("bc_w", C.c_float), ("huber_factor", C.c_float), ("gmax", C.c_float),
                ("cut", C.c_int * 8)]


def _ensure_built():
    if not ORACLE_SO.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "all"], check=True)


_ensure_built()
O = C.CDLL(str(ORACLE_SO))
_vp, _i, _d, _f = C.c_void_p, C.c_int, C.c_double, C.c_float
O.orc_view_from_round.argtypes = [_d, _i, C.POINTER(OView)]
O.orc_view_from_angle.argtypes = [_d, C.POINTER(OView)]
O.orc_fp_f32.argtypes = [C.POINTER(OGeom), _i, C.POINTER(OView), _vp, _vp, _vp, _vp, _i]
O.orc_fp_f64.argtypes = [C.POINTER(OGeom), C.POINTER(OView), _vp, _vp, _vp, _vp, _i]
O.orc_fp_rows_f64.argtypes = [C.POINTER(OGeom), C.POINTER(OView), _vp, _i, _i, _vp, _i]
O.orc_fp_rows_f32.argtypes = [C.POINTER(OGeom), _i, C.POINTER(OView), _vp, _i, _i, _vp, _i]
O.orc_bp_ray_scatter_f32.argtypes = [C.POINTER(OGeom), _i, C.POINTER(OView), _vp, _vp, _vp]
O.orc_fp_adjoint_f64.argtypes = [C.POINTER(OGeom), C.POINTER(OView), _vp, _vp]
O.orc_fp_adjoint_f32.argtypes = [C.POINTER(OGeom), _i, C.POINTER(OView), _vp, _vp]
O.orc_bp_voxel_f32.argtypes = [C.POINTER(OGeom), _i, C.POINTER(OView), _vp, _d, _f, _vp, _i]
O.orc_bp_voxel_f64.argtypes = [C.POINTER(OGeom), C.POINTER(OView), _vp, _d, _d, _vp, _i]
O.orc_correction_f32.argtypes = [_i, _vp, _vp, _vp, _vp]
O.orc_bp_ray_update_f32.argtypes = [C.c_long, _vp, _vp, _f, _vp]
O.orc_sart_f32.argtypes = [C.POINTER(OGeom), _i, _vp, _vp, _i, _vp, _d, _f, _i, _vp, _vp, _vp, _i]
O.orc_sart_f64.argtypes = [C.POINTER(OGeom), _vp, _vp, _i, _vp, _d, _d, _i, _vp, _vp, _vp, _i]
O.orc_roi_mask_f32.argtypes = [_vp, _vp, _vp]
O.orc_permutation.argtypes = [C.c_ulonglong, _i, _vp]
O.orc_pd_dual_f32.argtypes = [_vp, C.POINTER(OPd), _vp, _vp, _vp, _vp, _vp, _vp]
O.orc_pd_primal_f32.argtypes = [_vp, C.POINTER(OPd), _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
O.orc_pd_extrapolate_f32.argtypes = [_vp, _vp, _vp, _vp, _vp]
O.orc_pd_dual_f64.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
O.orc_pd_primal_f64.argtypes = [_vp, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
O.orc_pd_extrapolate_f64.argtypes = [_vp, _vp, _vp, _vp, _vp]
O.orc_warp_f32.argtypes = [_vp, _vp, _vp, _i, _f, _vp, _i]
O.orc_warp_f64.argtypes = [_vp, _vp, _vp, _i, _d, _vp, _i]
O.orc_warp_vjp_f64.argtypes = [_vp, _vp, _vp, _i, _d, _vp, _vp, _vp]
O.orc_cubic_at_f32.argtypes = [_vp, _vp, _f, _f, _f]
O.orc_cubic_at_f32.restype = _f
O.orc_cubic_at_f64.argtypes = [_vp, _vp, _d, _d, _d]
O.orc_cubic_at_f64.restype = _d
O.orc_warp_box_f32.argtypes = [_vp, _vp, _vp, _vp, _i, _f, _vp, _i]
O.orc_blur_f32.argtypes = [_vp, _i, _f, _vp]
O.orc_resize_f32.argtypes = [_vp, _i, _vp, _vp, _vp]
O.orc_gradient_f32.argtypes = [_vp, _vp, _vp, _vp, _vp]
O.orc_flow_level_f32.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _i, _i, _i, _f, _vp, _vp]
O.orc_flow_multiscale_f32.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _i, _i, _i, _f, _f, _i, _f,
                                      _vp]
O.orc_view_matrices_f32.argtypes = [C.POINTER(OGeom), C.POINTER(OView), _vp]

REF = None
if REF_SO.exists():
    REF = C.CDLL(str(REF_SO))
    REF.ref_fp_view.argtypes = [_vp, _vp, _i, _i, _d, _d, _d, _vp, _d, _i, _vp, _vp, _vp, _vp, _vp, _i]
    REF.ref_bp_ray_view.argtypes = [_vp, _vp, _i, _i, _d, _d, _d, _vp, _d, _i, _vp, _vp, _vp, _vp]
    REF.ref_warp.argtypes = [_vp, _vp, _vp, _i, _f, _vp]
    REF.ref_cubic_at.argtypes = [_vp, _vp, _i, _vp, _vp, _vp, _vp]
    REF.ref_warp_box.argtypes = [_vp, _vp, _vp, _vp, _i, _f, _vp]
    REF.ref_gradient.argtypes = [_vp, _vp, _vp, _vp, _vp]
    REF.ref_blur.argtypes = [_vp, _i, _vp, _f, _vp]
    REF.ref_resize_cubic.argtypes = [_vp, _i, _vp, _vp, _vp]
    REF.ref_flow_level.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _i, _i, _i, _f,
                                   _vp, _i]
    REF.ref_flow_multiscale.argtypes = [_vp, _vp, _vp, _vp, _vp, _f, _f, _i, _i, _i, _f, _f, _i, _f, _vp, _i]


REF_ST_SO = ROOT / "oracle" / "_ref" / "libstt_ref_st.so"


class RefStCfg(C.Structure):
    """ref_st_cfg of oracle/ref_st_driver.cpp."""
    _fields_ = [("dims", C.c_int * 3), ("sp", C.c_float * 3), ("W", C.c_int), ("H", C.c_int), ("ds", C.c_double),
                ("sid", C.c_double), ("sdd", C.c_double), ("oxyz", C.c_double * 3), ("nframes", C.c_int),
                ("nrounds", C.c_int), ("bp_mode", C.c_int), ("alpha", C.c_double), ("tv_w", C.c_double),
                ("tp_w", C.c_double), ("bc_w", C.c_double), ("huber", C.c_double), ("cut", C.c_int * 8),
                ("joint_iters", C.c_int), ("gmax", C.c_float), ("threads", C.c_int)]


REF_ST = None
if REF_ST_SO.exists():
    REF_ST = C.CDLL(str(REF_ST_SO))
    REF_ST.ref_st_run.argtypes = [C.POINTER(RefStCfg), _vp, C.c_char_p] + [_vp] * 3 + [_i] + [_vp] * 7 + [_vp, _vp,
                                                                                                        _vp]
    REF_ST.ref_st_shuffle.argtypes = [C.c_uint, _i, _vp]
    REF_ST.ref_st_last_run_seconds.argtypes = []
    REF_ST.ref_st_last_run_seconds.restype = C.c_double


class Scan:
    """One scan geometry, as both checkers and libstt take it."""

    def __init__(self, n, det, sid=600.0, sdd=1000.0, spacing=1.0, ds=1.0, off=(0.0, 0.0, 0.0)):
        self.dims = tuple(n) if hasattr(n, "__len__") else (n, n, n)
        self.det = tuple(det) if hasattr(det, "__len__") else (det, det)
        self.sp = tuple(spacing) if hasattr(spacing, "__len__") else (spacing,) * 3
        self.ds, self.sid, self.sdd, self.off = ds, sid, sdd, tuple(off)

    def ogeom(self) -> OGeom:
        nx, ny, nz = self.dims
        W, H = self.det
        return OGeom(nx, ny, nz, *map(float, self.sp), W, H, float(self.ds), float(self.sid),
                     float(self.sdd), (C.c_double * 3)(*self.off))


def view_round(start_deg: float, k: int) -> OView:
    v = OView()
    O.orc_view_from_round(float(start_deg), int(k), C.byref(v))
    return v


def view_angle(angle: float) -> OView:
    v = OView()
    O.orc_view_from_angle(float(angle), C.byref(v))
    return v


def views_array(views):
    arr = (OView * len(views))()
    for i, v in enumerate(views):
        arr[i] = v
    return arr


def fp32(scan: Scan, view: OView, vol: np.ndarray, gmode: int = 0, threads: int = 0):
    W, H = scan.det
    img = np.zeros((H, W), np.float32)
    rl = np.zeros_like(img)
    wt = np.zeros_like(img)
    g = scan.ogeom()
    O.orc_fp_f32(C.byref(g), gmode, C.byref(view), P(np.ascontiguousarray(vol, np.float32)), P(img),
                 P(rl), P(wt), threads)
    return img, rl, wt


def fp64(scan: Scan, view: OView, vol: np.ndarray, threads: int = 0):
    W, H = scan.det
    img = np.zeros((H, W), np.float64)
    rl = np.zeros_like(img)
    wt = np.zeros_like(img)
    g = scan.ogeom()
    O.orc_fp_f64(C.byref(g), C.byref(view), P(np.ascontiguousarray(vol, np.float64)), P(img), P(rl),
                 P(wt), threads)
    return img, rl, wt


def fp64_rows(scan: Scan, view: OView, vol: np.ndarray, row0: int, nrows: int, threads: int = 0):
    """FP64 projection of detector rows [row0, row0 + nrows) only: (nrows, W)."""
    W, H = scan.det
    img = np.zeros((H, W), np.float64)
    g = scan.ogeom()
    if O.orc_fp_rows_f64(C.byref(g), C.byref(view), P(np.ascontiguousarray(vol, np.float64)), row0, row0 + nrows,
                         P(img), threads) != 0:
        raise ValueError("bad row range")
    return img[row0:row0 + nrows].copy()


def fp32_rows(scan: Scan, view: OView, vol: np.ndarray, row0: int, nrows: int, gmode: int = 1, threads: int = 0):
    """The band in the reference's FP32 arithmetic (gmode 1: FP64 ray set-up, FP32 march, as the GPU)."""
    W, H = scan.det
    img = np.zeros((H, W), np.float32)
    g = scan.ogeom()
    if O.orc_fp_rows_f32(C.byref(g), gmode, C.byref(view), P(np.ascontiguousarray(vol, np.float32)), row0,
                         row0 + nrows, P(img), threads) != 0:
        raise ValueError("bad row range")
    return img[row0:row0 + nrows].copy()


def ref_fp(scan: Scan, start_deg: float, k: int, vol: np.ndarray, threads: int = 0):
    W, H = scan.det
    img = np.zeros((H, W), np.float32)
    rl = np.zeros_like(img)
    wt = np.zeros_like(img)
    dims = np.array(scan.dims, np.int32)
    sp = np.array(scan.sp, np.float32)
    off = np.array(scan.off, np.float64)
    REF.ref_fp_view(P(dims), P(sp), W, H, scan.ds, scan.sid, scan.sdd, P(off), float(start_deg), int(k),
                    P(np.ascontiguousarray(vol, np.float32)), P(img), P(rl), P(wt), None, threads)
    return img, rl, wt


def ref_bp_ray(scan: Scan, start_deg: float, k: int, corr: np.ndarray):
    nx, ny, nz = scan.dims
    W, H = scan.det
    c = np.zeros((nz, ny, nx), np.float32)
    w = np.zeros_like(c)
    dims = np.array(scan.dims, np.int32)
    sp = np.array(scan.sp, np.float32)
    off = np.array(scan.off, np.float64)
    REF.ref_bp_ray_view(P(dims), P(sp), W, H, scan.ds, scan.sid, scan.sdd, P(off), float(start_deg),
                        int(k), P(np.ascontiguousarray(corr, np.float32)), P(c), P(w), None)
    return c, w


def bp_ray_scatter32(scan: Scan, view: OView, corr: np.ndarray, gmode: int = 0):
    nx, ny, nz = scan.dims
    c = np.zeros((nz, ny, nx), np.float32)
    w = np.zeros_like(c)
    g = scan.ogeom()
    O.orc_bp_ray_scatter_f32(C.byref(g), gmode, C.byref(view), P(np.ascontiguousarray(corr, np.float32)),
                             P(c), P(w))
    return c, w


def fp_adjoint64(scan: Scan, view: OView, proj_bar: np.ndarray):
    nx, ny, nz = scan.dims
    out = np.zeros((nz, ny, nx), np.float64)
    g = scan.ogeom()
    O.orc_fp_adjoint_f64(C.byref(g), C.byref(view), P(np.ascontiguousarray(proj_bar, np.float64)), P(out))
    return out


def fp_adjoint32(scan: Scan, view: OView, proj_bar: np.ndarray, gmode: int = 1):
    nx, ny, nz = scan.dims
    out = np.zeros((nz, ny, nx), np.float32)
    g = scan.ogeom()
    O.orc_fp_adjoint_f32(C.byref(g), gmode, C.byref(view), P(np.ascontiguousarray(proj_bar, np.float32)), P(out))
    return out


def bp_voxel32(scan, view, corr, alpha, gmax, vol, gmode=0):
    v = np.array(vol, np.float32, copy=True)
    g = scan.ogeom()
    O.orc_bp_voxel_f32(C.byref(g), gmode, C.byref(view), P(np.ascontiguousarray(corr, np.float32)),
                       float(alpha), float(gmax), P(v), 0)
    return v


def bp_voxel64(scan, view, corr, alpha, gmax, vol):
    v = np.array(vol, np.float64, copy=True)
    g = scan.ogeom()
    O.orc_bp_voxel_f64(C.byref(g), C.byref(view), P(np.ascontiguousarray(corr, np.float64)),
                       float(alpha), float(gmax), P(v), 0)
    return v


def sart64(scan, views, perm, proj, alpha, gmax, bp_mode, vol, raylen=None, roi=None, threads=0):
    v = np.array(vol, np.float64, copy=True)
    W, H = scan.det
    rl = np.zeros((H, W), np.float64) if raylen is None else raylen
    g = scan.ogeom()
    va = views_array(views)
    pm = np.ascontiguousarray(perm, np.int32)
    O.orc_sart_f64(C.byref(g), va, P(pm), len(pm), P(np.ascontiguousarray(proj, np.float64)), float(alpha),
                   float(gmax), int(bp_mode), P(v), P(rl),
                   None if roi is None else P(np.ascontiguousarray(roi, np.float64)), threads)
    return v, rl


def sart32(scan, views, perm, proj, alpha, gmax, bp_mode, vol, raylen=None, roi=None, gmode=1,
           threads=0):
    v = np.array(vol, np.float32, copy=True)
    W, H = scan.det
    rl = np.zeros((H, W), np.float32) if raylen is None else raylen
    g = scan.ogeom()
    va = views_array(views)
    pm = np.ascontiguousarray(perm, np.int32)
    O.orc_sart_f32(C.byref(g), gmode, va, P(pm), len(pm), P(np.ascontiguousarray(proj, np.float32)),
                   float(alpha), float(gmax), int(bp_mode), P(v), P(rl),
                   None if roi is None else P(np.ascontiguousarray(roi, np.float32)), threads)
    return v, rl


def roi_mask(dims, cut):
    nx, ny, nz = dims
    r = np.zeros((nz, ny, nx), np.float32)
    O.orc_roi_mask_f32(P(np.array(dims, np.int32)), P(np.array(cut, np.int32)), P(r))
    return r


def permutation(seed, n):
    out = np.zeros(n, np.int32)
    O.orc_permutation(C.c_ulonglong(seed), n, P(out))
    return out


def warp32(vel, src, dt, threads=0):
    nc = 1 if src.ndim == 3 else src.shape[0]
    nz, ny, nx = src.shape[-3:]
    out = np.zeros_like(src, dtype=np.float32)
    O.orc_warp_f32(P(np.array([nx, ny, nz], np.int32)), P(np.ascontiguousarray(vel, np.float32)),
                   P(np.ascontiguousarray(src, np.float32)), nc, float(dt), P(out), threads)
    return out


def warp64(vel, src, dt, threads=0):
    nc = 1 if src.ndim == 3 else src.shape[0]
    nz, ny, nx = src.shape[-3:]
    out = np.zeros(src.shape, np.float64)
    O.orc_warp_f64(P(np.array([nx, ny, nz], np.int32)), P(np.ascontiguousarray(vel, np.float64)),
                   P(np.ascontiguousarray(src, np.float64)), nc, float(dt), P(out), threads)
    return out


def warp_vjp64(vel, src, dt, out_bar):
    nc = 1 if src.ndim == 3 else src.shape[0]
    nz, ny, nx = src.shape[-3:]
    sb = np.zeros(src.shape, np.float64)
    vb = np.zeros(vel.shape, np.float64)
    O.orc_warp_vjp_f64(P(np.array([nx, ny, nz], np.int32)), P(np.ascontiguousarray(vel, np.float64)),
                       P(np.ascontiguousarray(src, np.float64)), nc, float(dt),
                       P(np.ascontiguousarray(out_bar, np.float64)), P(sb), P(vb))
    return sb, vb


def ref_warp(vel, src, dt):
    nc = 1 if src.ndim == 3 else src.shape[0]
    nz, ny, nx = src.shape[-3:]
    out = np.zeros_like(src, dtype=np.float32)
    REF.ref_warp(P(np.array([nx, ny, nz], np.int32)), P(np.ascontiguousarray(vel, np.float32)),
                 P(np.ascontiguousarray(src, np.float32)), nc, float(dt), P(out))
    return out


def pd_dual32(dims, p: OPd, xf, xf1, bw, ytv, ytp, ybc):
    ytv, ytp, ybc = (np.array(a, np.float32, copy=True) for a in (ytv, ytp, ybc))
    O.orc_pd_dual_f32(P(np.array(dims, np.int32)), C.byref(p), P(xf), P(xf1), P(bw), P(ytv), P(ytp), P(ybc))
    return ytv, ytp, ybc


def pd_primal32(dims, p: OPd, first, ytp_prev, ytp, fw, ybc, ytv, vol):
    v = np.array(vol, np.float32, copy=True)
    xprev = np.zeros_like(v)
    O.orc_pd_primal_f32(P(np.array(dims, np.int32)), C.byref(p), int(first), P(ytp_prev), P(ytp), P(fw),
                        P(ybc), P(ytv), P(v), P(xprev))
    return v, xprev


def pd_extrapolate32(dims, cut, vol, xprev, xbar):
    xb = np.array(xbar, np.float32, copy=True)
    O.orc_pd_extrapolate_f32(P(np.array(dims, np.int32)), P(np.array(cut, np.int32)), P(vol), P(xprev), P(xb))
    return xb


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def pd_dual64(dims, pp, cut, xf, xf1, bw, ytv, ytp, ybc):
    ytv, ytp, ybc = (np.array(a, np.float64, copy=True) for a in (ytv, ytp, ybc))
    O.orc_pd_dual_f64(P(np.array(dims, np.int32)), P(np.array(pp, np.float64)), P(np.array(cut, np.int32)),
                      P(np.ascontiguousarray(xf, np.float64)), P(np.ascontiguousarray(xf1, np.float64)),
                      P(np.ascontiguousarray(bw, np.float64)), P(ytv), P(ytp), P(ybc))
    return ytv, ytp, ybc


def pd_primal64(dims, pp, cut, first, ytp_prev, ytp, fw, ybc, ytv, vol):
    v = np.array(vol, np.float64, copy=True)
    xprev = np.zeros_like(v)
    z = np.zeros_like(v)
    O.orc_pd_primal_f64(P(np.array(dims, np.int32)), P(np.array(pp, np.float64)), P(np.array(cut, np.int32)),
                        int(first), P(np.ascontiguousarray(z if ytp_prev is None else ytp_prev, np.float64)),
                        P(np.ascontiguousarray(ytp, np.float64)),
                        P(np.ascontiguousarray(z if fw is None else fw, np.float64)),
                        P(np.ascontiguousarray(ybc, np.float64)), P(np.ascontiguousarray(ytv, np.float64)),
                        P(v), P(xprev))
    return v, xprev


def pd_extrapolate64(dims, cut, vol, xprev, xbar):
    xb = np.array(xbar, np.float64, copy=True)
    O.orc_pd_extrapolate_f64(P(np.array(dims, np.int32)), P(np.array(cut, np.int32)),
                             P(np.ascontiguousarray(vol, np.float64)), P(np.ascontiguousarray(xprev, np.float64)),
                             P(xb))
    return xb


def pd_iteration(scan, angles, st, F, V, pp, pd_cut, roi_cut, alpha, bp_mode, orders, raylen, fp64=True):
    """One primal-dual iteration of ST_Tomography::Render (ST_Tomography.cpp:492-607)
    in the reference's sequential frame order.  fp64=True: the FP64 oracle;
    fp64=False: the reference's FP32 arithmetic (float march on FP64 ray setup).
    st: dict of arrays (vol (F+1), xbar (F+1), xprev F, ytv F x 3, ytp F, ybc F,
    flow F x 3, proj F x V); orders[f] is frame f's view order; raylen[f] the
    sticky ray-length state.  pp = (sigma, tau, tv_w, tp_w, bc_w, huber_factor, gmax)."""
    dims = scan.dims
    dt = np.float64 if fp64 else np.float32
    st = {k: np.array(v, dt, copy=True) for k, v in st.items()}
    roi = roi_mask(dims, roi_cut).astype(dt)
    views = [view_angle(a) for a in angles]
    opd = OPd(*pp, (C.c_int * 8)(*pd_cut))
    for f in range(F):
        if fp64:
            bw = warp64(st["flow"][f], st["xbar"][f + 1], -1.0)
            st["ytv"][f], st["ytp"][f], st["ybc"][f] = pd_dual64(dims, pp, pd_cut, st["xbar"][f], st["xbar"][f + 1],
                                                                 bw, st["ytv"][f], st["ytp"][f], st["ybc"][f])
            fw = None if f == 0 else warp64(st["flow"][f - 1], st["ybc"][f - 1], 1.0)
            st["vol"][f], st["xprev"][f] = pd_primal64(dims, pp, pd_cut, f == 0,
                                                       None if f == 0 else st["ytp"][f - 1], st["ytp"][f], fw,
                                                       st["ybc"][f], st["ytv"][f], st["vol"][f])
            st["vol"][f], raylen[f] = sart64(scan, views[f * V:(f + 1) * V], orders[f], st["proj"][f], alpha, pp[6],
                                             bp_mode, st["vol"][f], raylen=raylen[f], roi=roi)
            st["xbar"][f] = pd_extrapolate64(dims, pd_cut, st["vol"][f], st["xprev"][f], st["xbar"][f])
        else:
            bw = warp32(st["flow"][f], st["xbar"][f + 1], -1.0)
            st["ytv"][f], st["ytp"][f], st["ybc"][f] = pd_dual32(dims, opd, st["xbar"][f], st["xbar"][f + 1], bw,
                                                                 st["ytv"][f], st["ytp"][f], st["ybc"][f])
            z = np.zeros_like(st["vol"][f])
            fw = z if f == 0 else warp32(st["flow"][f - 1], st["ybc"][f - 1], 1.0)
            st["vol"][f], st["xprev"][f] = pd_primal32(dims, opd, f == 0, z if f == 0 else st["ytp"][f - 1],
                                                       st["ytp"][f], fw, st["ybc"][f], st["ytv"][f], st["vol"][f])
            st["vol"][f], raylen[f] = sart32(scan, views[f * V:(f + 1) * V], orders[f], st["proj"][f], alpha, pp[6],
                                             bp_mode, st["vol"][f], raylen=raylen[f], roi=roi, gmode=1)
            st["xbar"][f] = pd_extrapolate32(dims, pd_cut, st["vol"][f], st["xprev"][f], st["xbar"][f])
    return st


def bf16_round(a) -> np.ndarray:
    """FP32 values rounded to the nearest BF16 (ties to even), as FP32: what a
    BF16 store keeps (finite inputs)."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(np.shape(a))


def pd_iteration_bf16(scan, angles, st, F, V, pp, pd_cut, roi_cut, alpha, bp_mode, orders, raylen):
    """pd_iteration in the FP32 arithmetic with BF16 storage of the primal
    volumes (vol, xbar, xprev): every value stored into them is rounded to the
    nearest BF16 -- after the primal step, after each view's backprojection
    inside SART, and after the over-relaxation -- while the duals, the warped
    volumes and the ray lengths stay FP32.  st["proj"] (and the volumes) must
    already hold BF16 values.  The rounding after each view is why SART runs
    here one view per call."""
    dims = scan.dims
    st = {k: np.array(v, np.float32, copy=True) for k, v in st.items()}
    roi = roi_mask(dims, roi_cut)
    views = [view_angle(a) for a in angles]
    opd = OPd(*pp, (C.c_int * 8)(*pd_cut))
    for f in range(F):
        bw = warp32(st["flow"][f], st["xbar"][f + 1], -1.0)
        st["ytv"][f], st["ytp"][f], st["ybc"][f] = pd_dual32(dims, opd, st["xbar"][f], st["xbar"][f + 1], bw,
                                                             st["ytv"][f], st["ytp"][f], st["ybc"][f])
        z = np.zeros_like(st["vol"][f])
        fw = z if f == 0 else warp32(st["flow"][f - 1], st["ybc"][f - 1], 1.0)
        v, xp = pd_primal32(dims, opd, f == 0, z if f == 0 else st["ytp"][f - 1], st["ytp"][f], fw, st["ybc"][f],
                            st["ytv"][f], st["vol"][f])
        v, st["xprev"][f] = bf16_round(v), bf16_round(xp)
        for k in orders[f]:
            v, raylen[f] = sart32(scan, views[f * V:(f + 1) * V], [int(k)], st["proj"][f], alpha, pp[6], bp_mode, v,
                                  raylen=raylen[f], gmode=1)
            v = bf16_round(v)
        st["vol"][f] = bf16_round(v * roi)
        st["xbar"][f] = bf16_round(pd_extrapolate32(dims, pd_cut, st["vol"][f], st["xprev"][f], st["xbar"][f]))
    return st


def view_matrices32(scan: Scan, view: OView) -> np.ndarray:
    """P2M, M2V, model-view, V2M of the reference's FP32 pipeline (64 floats)."""
    out = np.zeros(64, np.float32)
    g = scan.ogeom()
    O.orc_view_matrices_f32(C.byref(g), C.byref(view), P(out))
    return out


# ---- optical flow and the CImg operations it uses --------------------------

def _dim(a):
    nz, ny, nx = a.shape[-3:]
    return np.array([nx, ny, nz], np.int32)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def warp_box32(vel, src, dt, box):
    nc = 1 if src.ndim == 3 else src.shape[0]
    out = np.zeros(src.shape, np.float32)
    O.orc_warp_box_f32(P(_dim(src)), P(np.array(box, np.float32)), P(_f32(vel)), P(_f32(src)), nc, float(dt),
                       P(out), 0)
    return out


def ref_warp_box(vel, src, dt, box):
    nc = 1 if src.ndim == 3 else src.shape[0]
    out = np.zeros(src.shape, np.float32)
    REF.ref_warp_box(P(_dim(src)), P(np.array(box, np.float32)), P(_f32(vel)), P(_f32(src)), nc, float(dt),
                     P(out))
    return out


def blur32(img, sigma):
    nc = 1 if img.ndim == 3 else img.shape[0]
    out = np.array(img, np.float32, copy=True)
    O.orc_blur_f32(P(_dim(img)), nc, float(sigma), P(out))
    return out


def ref_blur(img, sigma):
    nc = 1 if img.ndim == 3 else img.shape[0]
    out = np.zeros(img.shape, np.float32)
    REF.ref_blur(P(_dim(img)), nc, P(_f32(img)), float(sigma), P(out))
    return out


def resize32(img, odim):
    """odim = (nx, ny, nz)."""
    nc = 1 if img.ndim == 3 else img.shape[0]
    shape = (odim[2], odim[1], odim[0]) if img.ndim == 3 else (nc, odim[2], odim[1], odim[0])
    out = np.zeros(shape, np.float32)
    O.orc_resize_f32(P(_dim(img)), nc, P(_f32(img)), P(np.array(odim, np.int32)), P(out))
    return out


def ref_resize(img, odim):
    nc = 1 if img.ndim == 3 else img.shape[0]
    shape = (odim[2], odim[1], odim[0]) if img.ndim == 3 else (nc, odim[2], odim[1], odim[0])
    out = np.zeros(shape, np.float32)
    REF.ref_resize_cubic(P(_dim(img)), nc, P(_f32(img)), P(np.array(odim, np.int32)), P(out))
    return out


def gradient32(img):
    g = np.zeros((3,) + img.shape, np.float32)
    O.orc_gradient_f32(P(_dim(img)), P(_f32(img)), P(g[0]), P(g[1]), P(g[2]))
    return g


def ref_gradient(img):
    g = np.zeros((3,) + img.shape, np.float32)
    REF.ref_gradient(P(_dim(img)), P(_f32(img)), P(g[0]), P(g[1]), P(g[2]))
    return g


def flow_level32(I1, I2, V, Y, roi, box=None, tol=0.0, lam=1.2, max_iter=20, norm=4, n_warps=2, huber=1.0,
                 errs=False):
    """Returns (V, Y, iterations per warp[, last residual per warp]); Y is 10 channels (Y1|Y2|Y3|Y4)."""
    d = _dim(I1)
    box = np.array(d if box is None else box, np.float32)
    V = np.array(V, np.float32, copy=True)
    Y = np.array(Y, np.float32, copy=True)
    its = np.zeros(n_warps, np.int32)
    err = np.zeros(n_warps, np.float32)
    O.orc_flow_level_f32(P(d), P(box), P(np.array(roi, np.int32)), P(_f32(I1)), P(_f32(I2)), P(V), P(Y),
                         float(tol), float(lam), int(max_iter), int(norm), int(n_warps), float(huber), P(its),
                         P(err))
    return (V, Y, its, err) if errs else (V, Y, its)


def ref_flow_level(I1, I2, V, Y, roi, box=None, tol=0.0, lam=1.2, max_iter=20, norm=4, n_warps=2, huber=1.0,
                   threads=1):
    d = _dim(I1)
    box = np.array(d if box is None else box, np.int32)
    V = np.array(V, np.float32, copy=True)
    Y = np.array(Y, np.float32, copy=True)
    y1, y2, y3, y4 = (np.ascontiguousarray(Y[a:b]) for a, b in ((0, 3), (3, 6), (6, 9), (9, 10)))
    REF.ref_flow_level(P(d), P(box), P(_f32(I1)), P(_f32(I2)), P(V), P(y1), P(y2), P(y3), P(y4), float(tol),
                       float(lam), int(max_iter), int(norm), int(n_warps), float(huber),
                       P(np.array(roi, np.int32)), threads)
    return V, np.concatenate([y1, y2, y3, y4])


def flow_multiscale32(I1, I2, V, cut, Y=None, tol=0.0, lam=1.2, max_iter=20, norm=4, n_warps=2, eta=0.65,
                      sigma=0.5, scales=3, huber=1.0):
    d = _dim(I1)
    out = np.zeros((3,) + I1.shape, np.float32)
    O.orc_flow_multiscale_f32(P(d), P(_f32(I1)), P(_f32(I2)), P(_f32(V)), None if Y is None else P(_f32(Y)),
                              P(out), float(tol), float(lam), int(max_iter), int(norm), int(n_warps), float(eta),
                              float(sigma), int(scales), float(huber), P(np.array(cut, np.int32)))
    return out


def ref_flow_multiscale(I1, I2, V, cut, tol=0.0, lam=1.2, max_iter=20, norm=4, n_warps=2, eta=0.65, sigma=0.5,
                        scales=3, huber=1.0, threads=1):
    d = _dim(I1)
    out = np.zeros((3,) + I1.shape, np.float32)
    c8 = np.zeros(8, np.int32)
    c8[:6] = cut[:6]
    REF.ref_flow_multiscale(P(d), P(_f32(I1)), P(_f32(I2)), P(_f32(V)), P(out), float(tol), float(lam),
                            int(max_iter), int(norm), int(n_warps), float(eta), float(sigma), int(scales),
                            float(huber), P(c8), threads)
    return out


# ---- the reference's own ST_Tomography (oracle/_ref/libstt_ref_st.so) -------

def ref_st_run(scan: Scan, start_deg, proj, vols, flows, *, rounds=1, bp_mode=0, alpha=0.3, tv_w=0.05, tp_w=0.3,
               bc_w=0.2, huber=0.01, cut=(3, 3, 3, 5, 3, 3, 6, 5), mode=0, joint_iters=2, gmax=0.0, threads=1,
               full=True):
    """Runs the reference's ST_Tomography: mode 0 = SART(f) for every frame,
    mode 1 = Render (the joint loop).  start_deg: (F, rounds); proj: (F, V, H, W)
    with V = 10 * rounds; vols: (F, nz, ny, nx); flows: (F, 3, nz, ny, nx).
    Returns a dict of the outputs (only `vol` unless full), the srand seeds,
    G_Max and the seconds the SART calls / Render took."""
    import tempfile

    F = len(vols)
    nx, ny, nz = scan.dims
    W, H = scan.det
    cfg = RefStCfg((C.c_int * 3)(*scan.dims), (C.c_float * 3)(*scan.sp), W, H, float(scan.ds), float(scan.sid),
                   float(scan.sdd), (C.c_double * 3)(*scan.off), F, rounds, bp_mode, float(alpha), float(tv_w),
                   float(tp_w), float(bc_w), float(huber), (C.c_int * 8)(*cut), joint_iters, float(gmax), threads)
    sd = np.ascontiguousarray(np.asarray(start_deg, np.float32).reshape(F, rounds))
    pr = np.ascontiguousarray(proj, np.float32)
    vo = np.ascontiguousarray(vols, np.float32)
    fl = np.ascontiguousarray(flows, np.float32)
    out = dict(vol=np.zeros((F, nz, ny, nx), np.float32))
    if full:
        out.update(xbar=np.zeros((F + 1, nz, ny, nx), np.float32), xprev=np.zeros((F + 1, nz, ny, nx), np.float32),
                   ytv=np.zeros((F + 1, 3, nz, ny, nx), np.float32), ytp=np.zeros((F + 1, nz, ny, nx), np.float32),
                   ybc=np.zeros((F + 1, nz, ny, nx), np.float32), flow=np.zeros((F, 3, nz, ny, nx), np.float32))
    g = out.get
    seeds = np.zeros(4096, np.uint32)
    nseeds = C.c_int(len(seeds))
    gm = C.c_float()
    with tempfile.TemporaryDirectory() as wd:
        (Path(wd) / "FlowOutput").mkdir()
        rc = REF_ST.ref_st_run(C.byref(cfg), P(sd), wd.encode(), P(pr), P(vo), P(fl), mode, P(out["vol"]),
                               P(g("xbar")), P(g("xprev")), P(g("ytv")), P(g("ytp")), P(g("ybc")),
                               P(g("flow")), P(seeds), C.byref(nseeds), C.byref(gm))
    if rc != 0:
        raise RuntimeError(f"ref_st_run failed: {rc}")
    out["seeds"] = seeds[:nseeds.value].copy()
    out["gmax"] = float(gm.value)
    out["seconds"] = float(REF_ST.ref_st_last_run_seconds())
    return out


def ref_st_shuffle(seed: int, n: int) -> np.ndarray:
    """The view order the reference's SART draws after srand(seed)."""
    out = np.zeros(n, np.int32)
    REF_ST.ref_st_shuffle(int(seed), n, P(out))
    return out
