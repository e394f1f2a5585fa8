"""Generates tests/golden/reference_golden.npz from the reference's own code.

Run from the repository root after `make -C oracle ref` (which compiles the
reference's projector, warp and CImg sampler from its sources into
oracle/_ref/libstt_ref.so):

    python tests/golden/gen_golden.py

The fixtures are small (a few hundred KB) and seeded.  They pin the oracle's
FP32 restatement bit-for-bit where the reference tree is not available.
Cases: forward projection (image, ray length, sample count) of three views on
an off-centre, non-unit-spacing, non-square scan; the geometry matrices of
those views; the ray-driven backprojection scatter (contributions, weights);
warping::warp of a 2-channel volume for two time steps; CImg's cubic sampler
at points including edges and corners.  tests/golden/reference_flow_golden.npz:
CImg's Deriche blur, cubic/moving-average resize and gradient, the warp over a
general bounding box, four single-level optical-flow solves (with and without
an ROI, a full-size bounding box, residual iterations and a tolerance stop)
and one three-level multiscale solve.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
import oracle_bind as ob  # noqa: E402

OUT = HERE / "reference_golden.npz"

FP_SCAN = dict(n=(20, 18, 16), det=(24, 20), spacing=1.1, off=(0.5, -0.3, 0.8))
FP_VIEWS = [(0.0, 0), (33.3, 4), (250.0, 7)]
BP_SCAN = dict(n=(12, 11, 10), det=(18, 16), spacing=1.0, off=(0.2, 0.1, -0.4))
BP_VIEWS = [(15.0, 2), (300.5, 9)]
WARP_DIM = (10, 9, 8)
WARP_DT = (1.0, -1.0)


def main():
    if ob.REF is None:
        raise SystemExit("oracle/_ref/libstt_ref.so is missing: run `make -C oracle ref` first")
    rng = np.random.default_rng(20261203)
    out = {}
    # forward projection
    s = ob.Scan(FP_SCAN["n"], FP_SCAN["det"], spacing=FP_SCAN["spacing"], off=FP_SCAN["off"])
    nx, ny, nz = s.dims
    vol = rng.uniform(0, 1, (nz, ny, nx)).astype(np.float32)
    vol[:, :, :3] = 0.0
    out["fp_vol"] = vol
    imgs, rls, wts, mats = [], [], [], []
    dims = np.array(s.dims, np.int32)
    sp = np.array(s.sp, np.float32)
    off = np.array(s.off, np.float64)
    for sd, k in FP_VIEWS:
        img, rl, wt = ob.ref_fp(s, sd, k, vol, threads=1)
        m = np.zeros(96, np.float32)
        ob.REF.ref_fp_view(ob.P(dims), ob.P(sp), s.det[0], s.det[1], s.ds, s.sid, s.sdd, ob.P(off), sd, k,
                           ob.P(vol), None, None, None, ob.P(m), 1)
        imgs.append(img)
        rls.append(rl)
        wts.append(wt)
        mats.append(m)
    out.update(fp_img=np.stack(imgs), fp_raylen=np.stack(rls), fp_weight=np.stack(wts), fp_mats=np.stack(mats),
               fp_views=np.array(FP_VIEWS, np.float64))
    # ray-driven BP scatter
    s = ob.Scan(BP_SCAN["n"], BP_SCAN["det"], spacing=BP_SCAN["spacing"], off=BP_SCAN["off"])
    corr = rng.normal(size=(s.det[1], s.det[0])).astype(np.float32)
    cs, ws = [], []
    for sd, k in BP_VIEWS:
        c, w = ob.ref_bp_ray(s, sd, k, corr)
        cs.append(c)
        ws.append(w)
    out.update(bp_corr=corr, bp_contrib=np.stack(cs), bp_wsum=np.stack(ws), bp_views=np.array(BP_VIEWS, np.float64))
    # warp
    nx, ny, nz = WARP_DIM
    vel = (rng.normal(size=(3, nz, ny, nx)) * 1.3).astype(np.float32)
    src = rng.normal(size=(2, nz, ny, nx)).astype(np.float32)
    out.update(warp_vel=vel, warp_src=src,
               warp_out=np.stack([ob.ref_warp(vel, src, dt) for dt in WARP_DT]), warp_dt=np.array(WARP_DT))
    # CImg cubic sampler
    cdim = np.array([9, 7, 8], np.int32)
    img = rng.normal(size=(8, 7, 9)).astype(np.float32)
    pts = np.stack([rng.uniform(-1, 10, 96), rng.uniform(-1, 8, 96), rng.uniform(-1, 9, 96)]).astype(np.float32)
    pts[:, :6] = np.array([[0, 0, 0], [8, 6, 7], [3, 3, 3], [8.0, 2.5, 7], [4.5, 6, 0], [7.999, 5.5, 6.25]]).T
    vals = np.zeros(96, np.float32)
    ob.REF.ref_cubic_at(ob.P(cdim), ob.P(img), 96, ob.P(pts[0].copy()), ob.P(pts[1].copy()), ob.P(pts[2].copy()),
                        ob.P(vals))
    out.update(cubic_dim=cdim, cubic_img=img, cubic_pts=pts, cubic_val=vals)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    flow_fixtures()


FLOW_OUT = HERE / "reference_flow_golden.npz"
FLOW_DIM = (11, 10, 9)  # nx, ny, nz
# roi (x0 x1 y0 y1 z0 z1), box, max_iter, tol.  A case that stops on the
# residual uses no ROI: the reference's residual also sums gradient arrays it
# leaves unset outside the ROI (optical_flow.h:263-290), so with an ROI its
# stopping iteration depends on uninitialised memory.
FLOW_LEVEL_CASES = [
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 20, 0.0),
    ((2, 1, 1, 3, 2, 2), (16, 13, 12), 30, 0.0),
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 120, 1e-3),
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 130, 1e30),
]
FLOW_MS_DIM = (20, 18, 19)
FLOW_MS_CUT = (3, 2, 2, 4, 1, 3)


def flow_fixtures():
    """Optical flow and the CImg operations under it, from the reference's
    optical_flow.h / warping.h / CImg.h compiled into oracle/_ref (one thread)."""
    rng = np.random.default_rng(20261204)
    nx, ny, nz = FLOW_DIM
    out = {}
    img = rng.normal(size=(2, nz, ny, nx)).astype(np.float32)
    out["img"] = img
    out["blur_05"] = ob.ref_blur(img, 0.5)
    out["blur_13"] = ob.ref_blur(img, 1.3)
    for key, od in (("down", (7, 6, 8)), ("up", (16, 15, 12)), ("mixed", (11, 5, 20))):
        out[f"resize_{key}"] = ob.ref_resize(img, od)
        out[f"resize_{key}_dim"] = np.array(od, np.int32)
    out["grad"] = ob.ref_gradient(img[0])
    vel = (rng.normal(size=(3, nz, ny, nx)) * 1.5).astype(np.float32)
    out["vel"] = vel
    out["warp_box"] = ob.ref_warp_box(vel, img, -1.0, (17, 15, 13))
    i1 = ob.ref_blur(rng.uniform(0, 1, (nz, ny, nx)).astype(np.float32), 1.0)
    i2 = ob.ref_blur(rng.uniform(0, 1, (nz, ny, nx)).astype(np.float32), 1.0)
    v0 = (rng.normal(size=(3, nz, ny, nx)) * 0.3).astype(np.float32)
    y0 = (rng.normal(size=(10, nz, ny, nx)) * 0.1).astype(np.float32)
    out.update(I1=i1, I2=i2, V0=v0, Y0=y0)
    for c, (roi, box, mi, tol) in enumerate(FLOW_LEVEL_CASES):
        v, y = ob.ref_flow_level(i1, i2, v0, y0, roi, box=box, max_iter=mi, tol=tol, threads=1)
        out[f"level{c}_V"], out[f"level{c}_Y"] = v, y
    mx, my, mz = FLOW_MS_DIM
    m1 = ob.ref_blur(rng.uniform(0, 1, (mz, my, mx)).astype(np.float32), 1.5)
    m2 = ob.ref_blur(rng.uniform(0, 1, (mz, my, mx)).astype(np.float32), 1.5)
    mv = (rng.normal(size=(3, mz, my, mx)) * 0.3).astype(np.float32)
    out.update(ms_I1=m1, ms_I2=m2, ms_V0=mv)
    out["ms_V"] = ob.ref_flow_multiscale(m1, m2, mv, FLOW_MS_CUT, max_iter=12, threads=1)
    np.savez_compressed(FLOW_OUT, **out)
    print(f"wrote {FLOW_OUT} ({FLOW_OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
