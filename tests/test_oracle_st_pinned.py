"""The oracle's restatement of ST_Tomography.cpp is pinned to the reference's
own code: oracle/_ref/libstt_ref_st.so is the reference's ST_Tomography class
compiled where it lies (oracle/Makefile `ref`, compile-only stand-ins for
Eigen, libtiff and GL), driven by oracle/ref_st_driver.cpp.

* SART(f) (ST_Tomography.cpp:616-808): forward projection, correction,
  voxel-driven (bicubic) or ray-driven backprojection, ROI mask;
* Render() (:397-614): the image phase of the joint loop, two primal-dual
  passes over every frame (backward warp + dual step, forward warp + primal
  step, SART, over-relaxation), after the reference's own flow phase.

Both are compared bit for bit with the FP32 restatement (oracle/stt_oracle.cpp)
run on the same inputs, the same view order (the reference's srand seeds,
replayed) and the same flows.  No GPU."""
import ctypes as C

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.skipif(ob.REF_ST is None, reason="reference build (oracle/_ref/libstt_ref_st.so) not present")

CUT = (3, 3, 3, 5, 3, 3, 6, 5)


def _problem(seed, dims, det, frames, rounds, spacing=1.0, off=(0.3, -0.2, 0.4)):
    rng = np.random.default_rng(seed)
    scan = ob.Scan(dims, det, spacing=spacing, off=off)
    nx, ny, nz = scan.dims
    W, H = scan.det
    V = 10 * rounds
    start = rng.uniform(0.0, 360.0, (frames, rounds)).astype(np.float32)
    base = rng.uniform(0, 1, (nz, ny, nx)).astype(np.float32)
    vols = np.stack([base * np.float32(0.8 + 0.1 * f) for f in range(frames)]).astype(np.float32)
    proj = rng.uniform(0, 30, (frames, V, H, W)).astype(np.float32)
    flows = np.zeros((frames, 3, nz, ny, nx), np.float32)
    return scan, start, vols, proj, flows


def _views(start, f, rounds):
    return [ob.view_round(float(start[f, r]), k) for r in range(rounds) for k in range(10)]


@pytest.mark.parametrize("bp_mode", [0, 1])
@pytest.mark.parametrize("case", [dict(dims=(22, 20, 24), det=(40, 36), rounds=1, spacing=1.0),
                                  dict(dims=(18, 16, 20), det=(36, 30), rounds=2, spacing=1.1)])
def test_sart_restatement_equals_reference_sart(bp_mode, case):
    F = 2
    scan, start, vols, proj, flows = _problem(11, case["dims"], case["det"], F, case["rounds"], case["spacing"])
    V = 10 * case["rounds"]
    out = ob.ref_st_run(scan, start, proj, vols, flows, rounds=case["rounds"], bp_mode=bp_mode, alpha=0.3, cut=CUT,
                        mode=0, threads=1)
    assert len(out["seeds"]) == F  # one srand(time(0)) per SART call
    roi = ob.roi_mask(scan.dims, CUT)
    W, H = scan.det
    raylen = np.zeros((H, W), np.float32)  # one producer for all frames: the ray-length state carries over
    for f in range(F):
        perm = ob.ref_st_shuffle(out["seeds"][f], V)
        assert sorted(perm) == list(range(V))
        vol, raylen = ob.sart32(scan, _views(start, f, case["rounds"]), perm, proj[f], 0.3, out["gmax"], bp_mode,
                                vols[f], raylen=raylen, roi=roi, gmode=0)
        np.testing.assert_array_equal(vol, out["vol"][f], err_msg=f"frame {f}")


@pytest.mark.parametrize("bp_mode", [0, 1])
def test_primal_dual_restatement_equals_reference_render(bp_mode):
    """Render with two joint iterations: the reference's flow phase (its own
    optical flow, kept as it comes out) and then two primal-dual passes; the
    restatement replays the passes from the same start with those flows."""
    F, rounds = 3, 1
    V = 10 * rounds
    scan, start, vols, proj, flows = _problem(5, (20, 18, 22), (40, 36), F, rounds)
    tv, tp, bc, hub = 0.05, 0.3, 0.2, 0.01
    out = ob.ref_st_run(scan, start, proj, vols, flows, rounds=rounds, bp_mode=bp_mode, alpha=0.3, tv_w=tv, tp_w=tp,
                        bc_w=bc, huber=hub, cut=CUT, mode=1, joint_iters=2, threads=1)
    assert len(out["seeds"]) == 2 * F  # two passes over the frames, one SART call each
    # CP_sigma = .9/(L*CP_tau) and m_huberfactor as the reference forms them (ST_Tomography.cpp:97-102, 219)
    sigma = np.float32(0.9 / np.float32(8.0))
    hf = np.float32(1.0 / (1.0 + float(sigma) * hub / tv))
    opd = ob.OPd(float(sigma), 1.0, tv, tp, bc, float(hf), out["gmax"], (C.c_int * 8)(*CUT))
    nx, ny, nz = scan.dims
    W, H = scan.det
    roi = ob.roi_mask(scan.dims, CUT)
    full = np.concatenate([vols, vols[-1:]])  # the duplicated last frame (VolumeData.cpp:124-126)
    st = dict(vol=full.copy(), xbar=full.copy(), xprev=np.zeros_like(full),
              ytv=np.zeros((F + 1, 3, nz, ny, nx), np.float32), ytp=np.zeros_like(full), ybc=np.zeros_like(full))
    fl = out["flow"]
    raylen = np.zeros((H, W), np.float32)
    dims = scan.dims
    k = 0
    for _ in range(2):
        for f in range(F):
            bw = ob.warp32(fl[f], st["xbar"][f + 1], -1.0, threads=1)
            st["ytv"][f], st["ytp"][f], st["ybc"][f] = ob.pd_dual32(dims, opd, st["xbar"][f], st["xbar"][f + 1], bw,
                                                                     st["ytv"][f], st["ytp"][f], st["ybc"][f])
            z = np.zeros_like(st["vol"][f])
            fw = z if f == 0 else ob.warp32(fl[f - 1], st["ybc"][f - 1], 1.0, threads=1)
            st["vol"][f], st["xprev"][f] = ob.pd_primal32(dims, opd, f == 0, z if f == 0 else st["ytp"][f - 1],
                                                           st["ytp"][f], fw, st["ybc"][f], st["ytv"][f], st["vol"][f])
            perm = ob.ref_st_shuffle(out["seeds"][k], V)
            k += 1
            st["vol"][f], raylen = ob.sart32(scan, _views(start, f, rounds), perm, proj[f], 0.3, out["gmax"], bp_mode,
                                             st["vol"][f], raylen=raylen, roi=roi, gmode=0)
            st["xbar"][f] = ob.pd_extrapolate32(dims, CUT, st["vol"][f], st["xprev"][f], st["xbar"][f])
    assert np.abs(fl[:F - 1]).max() > 0  # the reference's flow phase ran and moved something
    for key in ("vol", "xbar", "xprev", "ytv", "ytp", "ybc"):
        np.testing.assert_array_equal(st[key][:F], out[key][:F], err_msg=key)
