"""Python side of the libstt C ABI (include/stt.h), on torch CUDA tensors.

Shapes (C order, x fastest as in the reference's CImg layout):
  volume            (nz, ny, nx)        float32
  projection stack  (nviews, H, W)      float32
  flow / velocity   (3, nz, ny, nx)     float32, planar channels
  dual TV variable  (3, nz, ny, nx)     float32
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from ._lib import FlowParams, Geometry, Instance, OpNorm, PdState, SolveCfg, STTError, Tuning, check, lib
from ._lib import PdParams as _PdParams

# ROI cut of the reference (ST_Tomography.cpp:114)
REFERENCE_CUT = (8, 8, 8, 45, 8, 8, 30, 20)


def _dtype_code(t) -> int:
    """stt_dtype of a tensor's storage: float32 -> STT_DTYPE_F32, bfloat16 -> STT_DTYPE_BF16."""
    import torch

    if t.dtype == torch.float32:
        return 0
    if t.dtype == torch.bfloat16:
        return 1
    raise ValueError(f"libstt stores float32 or bfloat16, not {t.dtype}")


def _ptr(t) -> C.c_void_p | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("libstt works on CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return C.c_void_p(t.data_ptr())


def _stream(stream) -> C.c_void_p | None:
    if stream is None:
        import torch

        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream) if stream.cuda_stream else None


def views_from_rounds(start_deg: Sequence[float], views_per_round: int = 10,
                      step_deg: float = 36.0) -> np.ndarray:
    """Angles (rad) of the reference's view list (InitViews, ST_Tomography.cpp:887-934)."""
    s = np.ascontiguousarray(start_deg, dtype=np.float64)
    out = np.zeros(len(s) * views_per_round, dtype=np.float64)
    check(lib.stt_views_from_rounds(len(s), s.ctypes.data_as(C.c_void_p), views_per_round,
                                    float(step_deg), out.ctypes.data_as(C.c_void_p)))
    return out


def lds_angles(n: int, segments: int = 10, base: int = 2, zero_every: int = 10000) -> np.ndarray:
    """Low_discrepency_squence.m:38-67 (degrees)."""
    out = np.zeros(n, dtype=np.float64)
    check(lib.stt_lds_angles(n, segments, base, zero_every, out.ctypes.data_as(C.c_void_p)))
    return out


def permutation(seed: int, n: int) -> np.ndarray:
    """Seeded view order (SplitMix64 + Fisher-Yates) used in place of time(0)."""
    out = np.zeros(n, dtype=np.int32)
    check(lib.stt_permutation(C.c_ulonglong(seed), n, out.ctypes.data_as(C.c_void_p)))
    return out


@dataclass
class PdParams:
    """Primal-dual parameters as ST_Tomography uses them (ST_Tomography.cpp:99-120, 215-219)."""

    sigma: float = 0.9 / 8.0
    tau: float = 1.0
    tv_w: float = 0.1
    tp_w: float = 0.5
    bc_w: float = 0.5
    huber_factor: float = 1.0
    gmax: float = 10.0
    cut: tuple = field(default=REFERENCE_CUT)

    def c(self) -> _PdParams:
        p = _PdParams(self.sigma, self.tau, self.tv_w, self.tp_w, self.bc_w, self.huber_factor,
                      self.gmax)
        for k in range(8):
            p.cut[k] = int(self.cut[k])
        return p


class Context:
    """One libstt context (stt_create/stt_destroy) on one device."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.stt_create(C.byref(h), int(device)))
        self._h = h
        self.device = device
        self.dims = None
        self.det = None
        self.n_views = 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.stt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st: int) -> None:
        check(st, self._h)

    def set_geometry(self, dims, spacing, det, ds, sid, sdd, angles, offset=(0.0, 0.0, 0.0)):
        """dims=(nx,ny,nz), spacing=(sx,sy,sz) mm, det=(W,H), angles in radians."""
        ang = np.ascontiguousarray(angles, dtype=np.float64)
        self._angles = ang  # keep alive for the call
        g = Geometry(int(dims[0]), int(dims[1]), int(dims[2]), float(spacing[0]), float(spacing[1]),
                     float(spacing[2]), int(det[0]), int(det[1]), float(ds), float(sid), float(sdd),
                     (C.c_double * 3)(*map(float, offset)), len(ang),
                     ang.ctypes.data_as(C.POINTER(C.c_double)))
        self._chk(lib.stt_set_geometry(self._h, C.byref(g)))
        self.dims = tuple(int(x) for x in dims)
        self.det = (int(det[0]), int(det[1]))
        self.n_views = len(ang)

    # ---- projector ---------------------------------------------------------
    def fp(self, vol, proj, view0=0, nviews=None, raylen=None, weight=None, stream=None):
        nviews = self.n_views - view0 if nviews is None else nviews
        self._chk(lib.stt_fp(self._h, _ptr(vol), _ptr(proj), _ptr(raylen), _ptr(weight), view0,
                             nviews, _stream(stream)))
        return proj

    def fp_typed(self, vol, proj, view0=0, nviews=None, raylen=None, weight=None, stream=None):
        """Forward projection of a float32 or bfloat16 volume (stt_fp_typed)."""
        import torch

        dtype = {torch.float32: 0, torch.bfloat16: 1}[vol.dtype]
        nviews = self.n_views - view0 if nviews is None else nviews
        self._chk(lib.stt_fp_typed(self._h, _ptr(vol), dtype, _ptr(proj), _ptr(raylen), _ptr(weight), view0, nviews,
                                   _stream(stream)))
        return proj

    def sart_view(self, vol, b, view, alpha, gmax, bp_mode, raylen_state, stream=None):
        """One SART view: FP + correction against b (H, W), then backprojection."""
        self._chk(lib.stt_sart_view(self._h, _ptr(vol), _ptr(b), int(view), float(alpha), float(gmax), int(bp_mode),
                                    _ptr(raylen_state), _stream(stream)))

    def opnorm(self, n_iter=50, seed=0, stream=None) -> dict:
        """||A|| by FP64 power iteration on A^T A, and the steps it implies."""
        o = OpNorm()
        self._chk(lib.stt_opnorm_power_iter(self._h, int(n_iter), C.c_ulonglong(seed), C.byref(o), _stream(stream)))
        return {"norm_A": o.norm_A, "norm_K": o.norm_K, "sigma": o.sigma, "tau": o.tau,
                "iterations": o.iterations, "rel_change": o.rel_change}

    def poll_status(self, stream=None):
        """Raises STTError (STT_ERR_TIMEOUT) if a bounded device-side wait of
        this context's launches gave up since the last poll; synchronises."""
        self._chk(lib.stt_poll_status(self._h, _stream(stream)))

    # ---- launch choices (stt_autotune / stt_get_tuning / stt_set_tuning) ----
    @staticmethod
    def _tuning_dict(t: Tuning) -> dict:
        return {"fp_variant": t.fp_variant, "slab_variant": t.slab_variant, "bp_variant": t.bp_variant,
                "staged_bins": t.staged_bins, "tuned": bool(t.tuned), "from_cache": bool(t.from_cache),
                "fp_us": list(t.fp_us)[:12], "slab_us": list(t.slab_us)[:8], "bp_us": list(t.bp_us)[:5],
                "ray_variant": t.ray_variant, "ray_us": list(t.ray_us), "staged_bins_bf16": t.staged_bins_bf16,
                "fp_variant_bf16": t.fp_variant_bf16, "fp16_us": list(t.fp16_us),
                "fp16": (lib.stt_tuning_variant_name(4, t.fp_variant_bf16) or b"").decode(),
                "ray": (lib.stt_tuning_variant_name(3, t.ray_variant) or b"").decode(),
                "fp": (lib.stt_tuning_variant_name(0, t.fp_variant) or b"").decode(),
                "slab": (lib.stt_tuning_variant_name(1, t.slab_variant) or b"").decode(),
                "bp": (lib.stt_tuning_variant_name(2, t.bp_variant) or b"").decode()}

    def autotune(self, stream=None) -> dict:
        """Times the launch variants on this geometry and keeps the fastest."""
        t = Tuning()
        self._chk(lib.stt_autotune(self._h, C.byref(t), _stream(stream)))
        return self._tuning_dict(t)

    def get_tuning(self) -> dict:
        t = Tuning()
        self._chk(lib.stt_get_tuning(self._h, C.byref(t)))
        return self._tuning_dict(t)

    def set_tuning(self, fp_variant=0, slab_variant=0, bp_variant=0, staged_bins=0x1E0, ray_variant=None,
                   staged_bins_bf16=None, fp_variant_bf16=None):
        """ray_variant and fp_variant_bf16 None keep the context's current
        choices; staged_bins_bf16 None takes staged_bins."""
        cur = self.get_tuning() if ray_variant is None or fp_variant_bf16 is None else None
        if ray_variant is None:
            ray_variant = cur["ray_variant"]
        if fp_variant_bf16 is None:
            fp_variant_bf16 = cur["fp_variant_bf16"]
        t = Tuning(int(fp_variant), int(slab_variant), int(bp_variant), int(staged_bins), 1, 0)
        t.ray_variant = int(ray_variant)
        t.staged_bins_bf16 = int(staged_bins if staged_bins_bf16 is None else staged_bins_bf16)
        t.fp_variant_bf16 = int(fp_variant_bf16)
        self._chk(lib.stt_set_tuning(self._h, C.byref(t)))

    def fp_correction(self, vol, b, raylen_state, corr, view, stream=None):
        self._chk(lib.stt_fp_correction(self._h, _ptr(vol), _ptr(b), _ptr(raylen_state), _ptr(corr),
                                        view, _stream(stream)))
        return corr

    def fp_vjp(self, proj_bar, vol_bar, view0=0, nviews=None, stream=None):
        nviews = self.n_views - view0 if nviews is None else nviews
        self._chk(lib.stt_fp_vjp(self._h, _ptr(proj_bar), _ptr(vol_bar), view0, nviews,
                                 _stream(stream)))
        return vol_bar

    def bp_voxel(self, corr, vol, alpha, gmax, view, stream=None):
        """vol: float32, or bfloat16 (BF16 storage, stt_bp_voxel_typed)."""
        self._chk(lib.stt_bp_voxel_typed(self._h, _ptr(corr), _ptr(vol), _dtype_code(vol), float(alpha),
                                         float(gmax), view, _stream(stream)))
        return vol

    def bp_ray(self, corr, vol, gmax, view, stream=None):
        """vol: float32, or bfloat16 (BF16 storage, stt_bp_ray_typed)."""
        self._chk(lib.stt_bp_ray_typed(self._h, _ptr(corr), _ptr(vol), _dtype_code(vol), float(gmax), view,
                                       _stream(stream)))
        return vol

    def gather_ceiling(self, vol, view, out, count=None, packed=True, stream=None, texture=False):
        """stt_gather_ceiling: the projector's gathers and interpolation alone
        along view `view`'s rays (a measurement kernel); `texture`: the
        corners as tld4 gathers (packed pairs)."""
        mode = 2 | 1 if texture else int(bool(packed))
        self._chk(lib.stt_gather_ceiling(self._h, _ptr(vol), view, mode, _ptr(out),
                                         _ptr(count) if count is not None else None, _stream(stream)))

    def fp_texture_ok(self, vol) -> bool:
        """Whether the tld4 gather forms bind `vol` as textures on this device
        (fp_variant 10, 11 for float32; fp_variant_bf16 1 for bfloat16;
        stt_fp_texture_ok_typed); else they run as loads."""
        ok = C.c_int(0)
        self._chk(lib.stt_fp_texture_ok_typed(self._h, _ptr(vol), _dtype_code(vol), C.byref(ok)))
        return bool(ok.value)

    def bp_ray_scatter(self, corr, contrib, wsum, view, stream=None):
        """The ray-driven backprojection's raw accumulation: contrib += c*w and
        wsum += w over every sample's 8 corners (stt_bp_ray_scatter)."""
        self._chk(lib.stt_bp_ray_scatter(self._h, _ptr(corr), _ptr(contrib), _ptr(wsum), view, _stream(stream)))

    def sart_sweep(self, vol, proj_stack, perm, alpha, gmax, bp_mode, raylen_state,
                   view_offset=0, roi_cut=None, stream=None):
        """vol and proj_stack: both float32, or both bfloat16 (BF16 storage,
        stt_sart_sweep_typed)."""
        perm = np.ascontiguousarray(perm, dtype=np.int32)
        cut = None if roi_cut is None else (C.c_int * 8)(*map(int, roi_cut))
        code = _dtype_code(vol)
        if _dtype_code(proj_stack) != code:
            raise ValueError("vol and proj_stack must have the same dtype")
        self._chk(lib.stt_sart_sweep_typed(self._h, _ptr(vol), code, _ptr(proj_stack),
                                           perm.ctypes.data_as(C.c_void_p), len(perm), view_offset,
                                           float(alpha), float(gmax), int(bp_mode), _ptr(raylen_state),
                                           cut, _stream(stream)))
        return vol

    # ---- primal-dual -------------------------------------------------------
    def pd_dual(self, p: PdParams, xbar_f, xbar_f1, bw, ytv, ytp, ybc, stream=None):
        pc = p.c()
        self._chk(lib.stt_pd_dual(self._h, C.byref(pc), _ptr(xbar_f), _ptr(xbar_f1), _ptr(bw),
                                  _ptr(ytv), _ptr(ytp), _ptr(ybc), _stream(stream)))

    def pd_primal(self, p: PdParams, first_frame, ytp_prev, ytp, fw, ybc, ytv, vol, xprev,
                  stream=None):
        pc = p.c()
        self._chk(lib.stt_pd_primal(self._h, C.byref(pc), int(bool(first_frame)), _ptr(ytp_prev),
                                    _ptr(ytp), _ptr(fw), _ptr(ybc), _ptr(ytv), _ptr(vol),
                                    _ptr(xprev), _stream(stream)))

    def pd_extrapolate(self, cut, vol, xprev, xbar, stream=None):
        c = (C.c_int * 8)(*map(int, cut))
        self._chk(lib.stt_pd_extrapolate(self._h, c, _ptr(vol), _ptr(xprev), _ptr(xbar),
                                         _stream(stream)))

    def roi_mask(self, cut, roi, stream=None):
        c = (C.c_int * 8)(*map(int, cut))
        self._chk(lib.stt_roi_mask(self._h, c, _ptr(roi), _stream(stream)))
        return roi


def warp(flow, src, dt, out=None, stream=None):
    """warping::warp (warping.h:116-145) with aabb = [0, dim]; src (nc, nz, ny, nx) or (nz, ny, nx)."""
    import torch

    nc = 1 if src.dim() == 3 else src.shape[0]
    nz, ny, nx = src.shape[-3:]
    dim = (C.c_int * 3)(nx, ny, nz)
    if out is None:
        out = torch.empty_like(src, dtype=torch.float32)
    check(lib.stt_warp_typed(dim, _ptr(flow), _ptr(src), _dtype_code(src), nc, float(dt), _ptr(out),
                             _stream(stream)))
    return out


def warp_poll_status(stream=None):
    """Raises STTError (STT_ERR_TIMEOUT) if a bounded wait of a standalone warp
    on the current device gave up since the last poll; synchronises."""
    check(lib.stt_warp_poll_status(_stream(stream)))


def warp_vjp(flow, src, dt, out_bar, src_bar=None, flow_bar=None, stream=None):
    """Accumulates J_src^T out_bar into src_bar and J_flow^T out_bar into flow_bar."""
    nc = 1 if src.dim() == 3 else src.shape[0]
    nz, ny, nx = src.shape[-3:]
    dim = (C.c_int * 3)(nx, ny, nz)
    check(lib.stt_warp_vjp(dim, _ptr(flow), _ptr(src), nc, float(dt), _ptr(out_bar), _ptr(src_bar),
                           _ptr(flow_bar), _stream(stream)))
    return src_bar, flow_bar


def _dim3(t):
    nz, ny, nx = t.shape[-3:]
    return (C.c_int * 3)(nx, ny, nz)


def warp_box(flow, src, dt, box, out=None, stream=None):
    """warping::warp with aabb = [0, box] (box = (bx, by, bz)); bit-exact CImg sampling."""
    import torch

    nc = 1 if src.dim() == 3 else src.shape[0]
    if out is None:
        out = torch.empty_like(src)
    check(lib.stt_warp_box(_dim3(src), (C.c_float * 3)(*map(float, box)), _ptr(flow), _ptr(src), nc, float(dt),
                           _ptr(out), _stream(stream)))
    return out


def image_gradient(img, out=None, stream=None):
    """CImg::get_gradient("xyz", 0) of a (nz, ny, nx) volume -> (3, nz, ny, nx)."""
    import torch

    if out is None:
        out = torch.empty((3,) + tuple(img.shape), device=img.device, dtype=img.dtype)
    check(lib.stt_image_gradient(_dim3(img), _ptr(img), _ptr(out), _stream(stream)))
    return out


@dataclass
class FlowParams_:
    """Parameters of optical_flow::L1Huber_OF_MultiScale3D; defaults are the
    values ST_Tomography::Render passes (ST_Tomography.cpp:440-456)."""

    tol: float = 0.1
    lam: float = 1.2
    huber: float = 1.0
    eta: float = 0.65
    sigma: float = 0.5
    max_iter: int = 3000
    norm: int = 4
    n_warps: int = 3
    scales: int = 3
    cut: Sequence[int] = field(default_factory=lambda: tuple(REFERENCE_CUT[:6]))

    def c(self) -> FlowParams:
        return FlowParams(float(self.tol), float(self.lam), float(self.huber), float(self.eta), float(self.sigma),
                          int(self.max_iter), int(self.norm), int(self.n_warps), int(self.scales),
                          (C.c_int * 6)(*map(int, self.cut[:6])))


class Flow:
    """stt_flow: the 3D TV-L1/Huber optical flow of optical_flow.h on one GPU.

    Images (nz, ny, nx), flow V (3, nz, ny, nx), dual Y (10, nz, ny, nx); all
    torch CUDA float32 tensors."""

    def __init__(self, shape, params: FlowParams_ | None = None, device: int = 0):
        """shape = (nz, ny, nx) of the full-size images."""
        self.params = params or FlowParams_()
        self.shape = tuple(int(v) for v in shape)
        nz, ny, nx = self.shape
        h = C.c_void_p()
        pc = self.params.c()
        rc = lib.stt_flow_create(int(device), (C.c_int * 3)(nx, ny, nz), C.byref(pc), C.byref(h))
        if rc != 0:
            raise STTError(rc, (lib.stt_last_error(None) or b"flow create failed").decode())
        self._h = h

    def _chk(self, rc):
        if rc != 0:
            raise STTError(rc, (lib.stt_flow_last_error(self._h) or b"").decode(errors="replace"))

    def multiscale(self, I1, I2, V, Y0=None, stream=None):
        """V: initial flow in, finest flow out (in place)."""
        shp = self.shape
        if tuple(I1.shape) != shp or tuple(I2.shape) != shp or tuple(V.shape) != (3,) + shp or (
                Y0 is not None and tuple(Y0.shape) != (10,) + shp):
            raise ValueError(f"multiscale expects images {shp}, V (3,)+{shp}, Y0 (10,)+{shp}")
        self._chk(lib.stt_flow_multiscale(self._h, _ptr(I1), _ptr(I2), _ptr(V), _ptr(Y0), _stream(stream)))
        return V

    def level(self, I1, I2, V, Y, roi, box=None, stream=None):
        nz, ny, nx = I1.shape
        shp = tuple(I1.shape)
        if tuple(I2.shape) != shp or tuple(V.shape) != (3,) + shp or tuple(Y.shape) != (10,) + shp:
            raise ValueError("level expects I1, I2 of one shape, V (3,)+shape and Y (10,)+shape")
        box = (nx, ny, nz) if box is None else box
        self._chk(lib.stt_flow_level(self._h, _dim3(I1), (C.c_float * 3)(*map(float, box)),
                                     (C.c_int * 6)(*map(int, roi)), _ptr(I1), _ptr(I2), _ptr(V), _ptr(Y),
                                     _stream(stream)))
        return V, Y

    def stats(self):
        """(iterations, residual) per (level, warp) of the last call; synchronises."""
        n = C.c_int()
        self._chk(lib.stt_flow_stats(self._h, C.byref(n), None, None))
        its = np.zeros(max(n.value, 1), np.int32)
        err = np.zeros(max(n.value, 1), np.float32)
        self._chk(lib.stt_flow_stats(self._h, C.byref(n), its.ctypes.data_as(C.c_void_p),
                                     err.ctypes.data_as(C.c_void_p)))
        return its[:n.value], err[:n.value]

    def blur(self, img, sigma, stream=None):
        """CImg::blur(sigma) in place on (nz, ny, nx) or (nc, nz, ny, nx)."""
        nc = 1 if img.dim() == 3 else img.shape[0]
        self._chk(lib.stt_flow_blur(self._h, _dim3(img), nc, float(sigma), _ptr(img), _stream(stream)))
        return img

    def resize(self, img, odim, out=None, stream=None):
        """CImg::get_resize(odim=(nx, ny, nz), nc, 5)."""
        import torch

        nc = 1 if img.dim() == 3 else img.shape[0]
        ox, oy, oz = odim
        shape = (oz, oy, ox) if img.dim() == 3 else (nc, oz, oy, ox)
        if out is None:
            out = torch.empty(shape, device=img.device, dtype=img.dtype)
        self._chk(lib.stt_flow_resize(self._h, _dim3(img), nc, _ptr(img), (C.c_int * 3)(ox, oy, oz), _ptr(out),
                                      _stream(stream)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib.stt_flow_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SOLVE_PLAIN, SOLVE_STREAMS, SOLVE_GRAPH, SOLVE_PERSISTENT = 0, 1, 2, 3


def frame_order(seed: int, iteration: int, n_frames: int, frame: int, views: int) -> np.ndarray:
    """View order of SART(frame) in PD iteration `iteration` (matches the device draw)."""
    out = np.zeros(views, dtype=np.int32)
    check(lib.stt_solver_frame_order(C.c_ulonglong(seed), C.c_ulonglong(iteration), n_frames, frame,
                                     views, out.ctypes.data_as(C.c_void_p)))
    return out


class Solver:
    """stt_solver: the space-time primal-dual iteration of ST_Tomography::Render.

    `state` holds torch CUDA tensors: vol (F+1,nz,ny,nx), xbar (F+1,...), xprev
    (F,...), ytv (F,3,...), ytp (F,...), ybc (F,...), flow (F,3,...), proj (F,V,H,W).
    """

    def __init__(self, ctx: Context, state: dict, n_frames: int, views_per_frame: int,
                 pd: PdParams, alpha: float = 0.3, bp_mode: int = 0, roi_cut=REFERENCE_CUT,
                 seed: int = 0, mode: int = SOLVE_GRAPH, halo: bool = False, frame_offset: int = 0,
                 total_frames: int = 0, autotune: bool = False, storage: str = "f32"):
        """halo=True: local frame 0 continues a previous shard (state needs
        ytp_halo, ybc_halo, flow_halo; see spacetimetomography_b200.halo).
        frame_offset / total_frames: the shard's place in the whole sequence
        (its view orders are those of the unsharded solve).  autotune: tune
        the context's launch choices first (Context.autotune).
        storage="bf16": vol, xbar, xprev and proj are torch.bfloat16 tensors
        (stt_solve_cfg.storage = STT_DTYPE_BF16); every other array stays
        float32."""
        import torch

        if storage not in ("f32", "bf16"):
            raise ValueError("storage must be 'f32' or 'bf16'")
        want = torch.bfloat16 if storage == "bf16" else torch.float32
        for k in ("vol", "xbar", "xprev", "proj"):
            if state[k].dtype != want:
                raise ValueError(f"state[{k!r}] must be {want} for storage={storage!r}")
        self.ctx = ctx
        self.state = state  # keeps the tensors alive
        cfg = SolveCfg(n_frames, views_per_frame, bp_mode, float(alpha), pd.c(),
                       (C.c_int * 8)(*map(int, roi_cut)), C.c_ulonglong(seed), mode, int(bool(halo)),
                       int(frame_offset), int(total_frames), int(bool(autotune)), 1 if storage == "bf16" else 0)
        keys = ("vol", "xbar", "xprev", "ytv", "ytp", "ybc", "flow", "proj", "ytp_halo", "ybc_halo",
                "flow_halo")
        st = PdState(*[state[k].data_ptr() if k in state else None for k in keys])
        h = C.c_void_p()
        rc = lib.stt_solver_create(ctx._h, C.byref(cfg), C.byref(st), C.byref(h))
        if rc != 0:
            raise STTError(rc, (lib.stt_last_error(ctx._h) or b"solver create failed").decode())
        self._h = h

    def iterate(self, n: int = 1, stream=None):
        rc = lib.stt_solver_iterate(self._h, int(n), _stream(stream))
        if rc != 0:
            raise STTError(rc, lib.stt_solver_last_error(self._h).decode())

    def iterate_phase(self, phase: int, stream=None):
        rc = lib.stt_solver_iterate_phase(self._h, int(phase), _stream(stream))
        if rc != 0:
            raise STTError(rc, lib.stt_solver_last_error(self._h).decode())

    def poll_status(self, stream=None):
        """See Context.poll_status."""
        rc = lib.stt_solver_poll_status(self._h, _stream(stream))
        if rc != 0:
            raise STTError(rc, lib.stt_solver_last_error(self._h).decode())

    def stats(self):
        nl, it = C.c_longlong(), C.c_ulonglong()
        check(lib.stt_solver_stats(self._h, C.byref(nl), C.byref(it)))
        return nl.value, it.value

    def persistent_info(self):
        """SOLVE_PERSISTENT: (blocks of the persistent launch, True if the
        iteration replays a captured graph); (0, False) in the other modes."""
        b, g = C.c_int(), C.c_int()
        check(lib.stt_solver_persistent_info(self._h, C.byref(b), C.byref(g)))
        return b.value, bool(g.value)

    def close(self):
        if getattr(self, "_h", None):
            lib.stt_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """stt_batch: independent single-frame TV + SART solves of uneven size,
    iterated together (concurrent streams, or one captured CUDA graph).

    Each instance is a dict: ctx (Context with its geometry), vol (nz, ny, nx)
    CUDA tensor (start in, result out), proj (V, H, W) CUDA tensor, and
    optionally bp_mode, alpha, pd (PdParams), roi_cut, seed, autotune and
    storage ("f32", or "bf16" with vol and proj torch.bfloat16 tensors)."""

    def __init__(self, instances, mode: int = SOLVE_GRAPH):
        import torch

        self._keep = instances
        arr = (Instance * len(instances))()
        for k, d in enumerate(instances):
            pd = d.get("pd", PdParams())
            storage = d.get("storage", "f32")
            want = {"f32": torch.float32, "bf16": torch.bfloat16}.get(storage)
            if want is None or d["vol"].dtype != want or d["proj"].dtype != want:
                raise ValueError(f"instance {k}: vol and proj must be {want} for storage={storage!r}")
            arr[k] = Instance(d["ctx"]._h, d["vol"].data_ptr(), d["proj"].data_ptr(), int(d["proj"].shape[0]),
                              int(d.get("bp_mode", 0)), float(d.get("alpha", 0.3)), pd.c(),
                              (C.c_int * 8)(*map(int, d.get("roi_cut", REFERENCE_CUT))),
                              C.c_ulonglong(int(d.get("seed", 0))), int(bool(d.get("autotune", False))),
                              1 if storage == "bf16" else 0)
        h = C.c_void_p()
        rc = lib.stt_batch_create(arr, len(instances), int(mode), C.byref(h))
        if rc != 0:
            raise STTError(rc, (lib.stt_last_error(None) or b"batch create failed").decode())
        self._h = h

    def staging(self) -> dict:
        """stt_batch_staging: the batch-level choice between the instances'
        tuned projector split and every view gathering."""
        timed, gather = C.c_int(), C.c_int()
        ms_split, ms_gather = C.c_float(), C.c_float()
        check(lib.stt_batch_staging(self._h, C.byref(timed), C.byref(gather), C.byref(ms_split), C.byref(ms_gather)))
        return {"timed": bool(timed.value), "all_gather": bool(gather.value), "ms_split": ms_split.value,
                "ms_gather": ms_gather.value}

    def iterate(self, n: int = 1, stream=None):
        rc = lib.stt_batch_iterate(self._h, int(n), _stream(stream))
        if rc != 0:
            raise STTError(rc, (lib.stt_batch_last_error(self._h) or b"").decode())

    def poll_status(self, stream=None):
        """See Context.poll_status."""
        rc = lib.stt_batch_poll_status(self._h, _stream(stream))
        if rc != 0:
            raise STTError(rc, (lib.stt_batch_last_error(self._h) or b"").decode())

    def close(self):
        if getattr(self, "_h", None):
            lib.stt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
