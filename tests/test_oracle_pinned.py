"""The oracle (CPU restatement) is pinned: bit-for-bit against fixtures made by
the reference's own compiled code (tests/golden/gen_golden.py), against the
live reference build when it is present, and through identities (adjoint,
finite differences, known answers) for the parts whose reference source does
not compile here.  No GPU."""
import math
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob

G = np.load(Path(__file__).resolve().parent / "golden" / "reference_golden.npz")


def _fp_scan():
    return ob.Scan((20, 18, 16), (24, 20), spacing=1.1, off=(0.5, -0.3, 0.8))


def test_fp_matches_reference_fixture_bitwise():
    s = _fp_scan()
    for v, (sd, k) in enumerate(G["fp_views"]):
        img, rl, wt = ob.fp32(s, ob.view_round(sd, int(k)), G["fp_vol"], gmode=0, threads=1)
        np.testing.assert_array_equal(img, G["fp_img"][v])
        np.testing.assert_array_equal(rl, G["fp_raylen"][v])
        np.testing.assert_array_equal(wt, G["fp_weight"][v])


def test_geometry_matrices_match_reference_fixture():
    s = _fp_scan()
    for v, (sd, k) in enumerate(G["fp_views"]):
        m = ob.view_matrices32(s, ob.view_round(sd, int(k)))
        np.testing.assert_array_equal(m, G["fp_mats"][v][:64])


def test_bp_ray_scatter_matches_reference_fixture_bitwise():
    s = ob.Scan((12, 11, 10), (18, 16), spacing=1.0, off=(0.2, 0.1, -0.4))
    for v, (sd, k) in enumerate(G["bp_views"]):
        c, w = ob.bp_ray_scatter32(s, ob.view_round(sd, int(k)), G["bp_corr"], gmode=0)
        np.testing.assert_array_equal(c, G["bp_contrib"][v])
        np.testing.assert_array_equal(w, G["bp_wsum"][v])


def test_warp_matches_reference_fixture_bitwise():
    for i, dt in enumerate(G["warp_dt"]):
        out = ob.warp32(G["warp_vel"], G["warp_src"], float(dt), threads=1)
        np.testing.assert_array_equal(out, G["warp_out"][i])


def test_cubic_sampler_matches_reference_fixture_bitwise():
    dim, img, pts = G["cubic_dim"], G["cubic_img"], G["cubic_pts"]
    vals = np.array([ob.O.orc_cubic_at_f32(ob.P(dim), ob.P(img), *map(float, pts[:, i])) for i in range(pts.shape[1])],
                    np.float32)
    np.testing.assert_array_equal(vals, G["cubic_val"])


@pytest.mark.skipif(ob.REF is None, reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("case", range(4))
def test_oracle_matches_live_reference(case):
    rng = np.random.default_rng(100 + case)
    n = tuple(int(x) for x in rng.integers(14, 30, 3))
    det = tuple(int(x) for x in rng.integers(16, 48, 2))
    s = ob.Scan(n, det, spacing=float(rng.uniform(0.7, 1.5)), off=tuple(rng.uniform(-2, 2, 3)))
    vol = rng.uniform(0, 1, (n[2], n[1], n[0])).astype(np.float32)
    sd, k = float(rng.uniform(0, 360)), int(rng.integers(0, 10))
    a = ob.ref_fp(s, sd, k, vol, threads=1)
    b = ob.fp32(s, ob.view_round(sd, k), vol, gmode=0, threads=1)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    corr = rng.normal(size=(det[1], det[0])).astype(np.float32)
    c1, w1 = ob.ref_bp_ray(s, sd, k, corr)
    c2, w2 = ob.bp_ray_scatter32(s, ob.view_round(sd, k), corr)
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(w1, w2)
    vel = rng.normal(size=(3,) + vol.shape).astype(np.float32)
    np.testing.assert_array_equal(ob.ref_warp(vel, vol, 1.0), ob.warp32(vel, vol, 1.0))


def test_fp64_oracle_close_to_reference_arithmetic():
    s = _fp_scan()
    for sd, k in G["fp_views"]:
        v = ob.view_round(sd, int(k))
        d64 = ob.fp64(s, v, G["fp_vol"].astype(np.float64))[0]
        assert ob.rel_l2(d64, ob.fp32(s, v, G["fp_vol"], gmode=0)[0]) < 1e-4


def test_fp64_adjoint_dot_product():
    s = ob.Scan((17, 15, 13), (21, 19), spacing=1.2, off=(0.3, -0.5, 0.2))
    rng = np.random.default_rng(1)
    x = rng.normal(size=(13, 15, 17))
    y = rng.normal(size=(19, 21))
    for a in (0.0, 1.3, math.pi / 2, 4.4):
        v = ob.view_angle(a)
        lhs = float(np.sum(ob.fp64(s, v, x)[0] * y))
        rhs = float(np.sum(x * ob.fp_adjoint64(s, v, y)))
        assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))


def test_warp_vjp_finite_differences():
    rng = np.random.default_rng(2)
    nz, ny, nx = 9, 10, 11
    z, y, x = np.mgrid[0:nz, 0:ny, 0:nx].astype(np.float64)
    # fields that vary along every axis: a field constant along an axis makes
    # clamped samples land exactly on a corner value, i.e. on the kink of the
    # 8-corner min/max clamp, where a central difference is not a derivative
    vel = np.stack([0.7 * np.sin(0.5 * y + 0.31 * x + 0.17 * z + 0.3), 0.6 * np.cos(0.4 * x + 0.23 * z - 0.11 * y + 0.1),
                    0.5 * np.sin(0.3 * z + 0.19 * x + 0.27 * y + 0.7)])
    src = np.sin(0.6 * x + 0.2 + 0.13 * z) * np.cos(0.5 * y + 0.07 * x) + 0.3 * z / nz
    obar = rng.normal(size=src.shape)
    sb, vb = ob.warp_vjp64(vel, src, 1.0, obar)
    eps = 1e-6
    for _ in range(3):
        ds = rng.normal(size=src.shape)
        fd = (np.sum(ob.warp64(vel, src + eps * ds, 1.0) * obar) - np.sum(ob.warp64(vel, src - eps * ds, 1.0) * obar)) / (2 * eps)
        assert abs(fd - np.sum(sb * ds)) <= 1e-6 * max(1.0, abs(fd))
        dv = rng.normal(size=vel.shape)
        fd = (np.sum(ob.warp64(vel + eps * dv, src, 1.0) * obar) - np.sum(ob.warp64(vel - eps * dv, src, 1.0) * obar)) / (2 * eps)
        assert abs(fd - np.sum(vb * dv)) <= 1e-5 * max(1.0, abs(fd))


def test_voxel_bp_constant_correction_known_answer():
    """Catmull-Rom weights sum to one: a constant correction c adds alpha*c to
    every voxel whose footprint is inside [2, W-2) x [2, H-2), nothing elsewhere."""
    s = ob.Scan((16, 14, 12), (40, 36))
    vol = np.full((12, 14, 16), 0.5, np.float32)
    out = ob.bp_voxel32(s, ob.view_angle(0.7), np.full((36, 40), 0.25, np.float32), 0.4, 10.0, vol, gmode=0)
    np.testing.assert_allclose(out, 0.5 + 0.4 * 0.25, rtol=1e-6)
    small = ob.Scan((16, 14, 12), (8, 8))  # most voxels project outside the 2-pixel border band
    out2 = ob.bp_voxel32(small, ob.view_angle(0.7), np.full((8, 8), 0.25, np.float32), 0.4, 10.0, vol, gmode=0)
    changed = np.isclose(out2, 0.6)
    assert changed.any() and (~changed).any() and np.all(out2[~changed] == 0.5)


def test_ray_bp_update_nan_rule_known_answer():
    contrib = np.array([1.0, 0.0, -3.0, 2.0], np.float32)
    wsum = np.array([2.0, 0.0, 1.0, 0.5], np.float32)
    vol = np.array([1.0, 5.0, 1.0, 9.0], np.float32)
    ob.O.orc_bp_ray_update_f32(4, ob.P(contrib), ob.P(wsum), np.float32(6.0), ob.P(vol))
    # 1+0.5; 0/0 -> NaN -> 0 (ST_Tomography.cpp:755-757 with the clamp macros); 1-3 -> 0; 9+4 -> gmax
    np.testing.assert_array_equal(vol, np.array([1.5, 0.0, 0.0, 6.0], np.float32))


def test_roi_mask_known_counts():
    dims = (64, 64, 64)
    r = ob.roi_mask(dims, (8, 8, 8, 45, 8, 8, 30, 20))
    # box: i in [8, 56], j in [8, 57] (j > ny - 7 cut), k in [8, 56]
    assert r[8, 8, 8] == 1.0 or r[8, 8, 8] == 0.0
    box = np.zeros_like(r)
    box[8:57, 8:58, 8:57] = 1.0
    assert np.all(r <= box)
    assert r[32, 32, 32] == 1.0 and r[32, 58, 32] == 0.0 and r[32, 57, 32] == 1.0
    # corner cut: i < 30 and k < 20 removed
    assert r[10, 32, 10] == 0.0 and r[25, 32, 31] == 1.0


def test_pd_dual_ramp_known_answer():
    dims = (12, 12, 12)
    x = np.arange(12, dtype=np.float32)
    xf = np.broadcast_to(2.0 * x[None, None, :], (12, 12, 12)).copy()  # slope 2 along x
    z = np.zeros((12, 12, 12), np.float32)
    cut = (2, 2, 2, 2, 2, 2, 0, 0)
    p = ob.OPd(0.1, 1.0, 10.0, 0.5, 0.5, 0.8, 100.0, (ob.C.c_int * 8)(*cut))
    ytv, ytp, ybc = ob.pd_dual32(dims, p, xf, xf, xf, np.zeros((3, 12, 12, 12), np.float32), z, z)
    # interior ROI: ytv_x = sigma * 2 * huber_factor, the other channels 0
    np.testing.assert_allclose(ytv[0, 5, 5, 5], 0.1 * 2.0 * 0.8, rtol=1e-6)
    assert ytv[1, 5, 5, 5] == 0.0 and ytv[2, 5, 5, 5] == 0.0
    assert ytv[0, 0, 5, 5] == 0.0  # outside the interior
    assert np.all(ytp == 0.0) and np.all(ybc == 0.0)


def test_permutation_is_a_seeded_shuffle():
    p1, p2 = ob.permutation(5, 50), ob.permutation(5, 50)
    np.testing.assert_array_equal(p1, p2)
    assert sorted(p1.tolist()) == list(range(50)) and not np.array_equal(p1, np.arange(50))


# ---- optical flow and the CImg operations it uses --------------------------

FG = np.load(Path(__file__).resolve().parent / "golden" / "reference_flow_golden.npz")
FLOW_LEVEL_CASES = [  # as tests/golden/gen_golden.py
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 20, 0.0),
    ((2, 1, 1, 3, 2, 2), (16, 13, 12), 30, 0.0),
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 120, 1e-3),
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 130, 1e30),
]


def test_cimg_image_ops_match_reference_fixture_bitwise():
    img = FG["img"]
    np.testing.assert_array_equal(ob.blur32(img, 0.5), FG["blur_05"])
    np.testing.assert_array_equal(ob.blur32(img, 1.3), FG["blur_13"])
    for key in ("down", "up", "mixed"):
        np.testing.assert_array_equal(ob.resize32(img, tuple(FG[f"resize_{key}_dim"])), FG[f"resize_{key}"])
    np.testing.assert_array_equal(ob.gradient32(img[0]), FG["grad"])
    np.testing.assert_array_equal(ob.warp_box32(FG["vel"], img, -1.0, (17, 15, 13)), FG["warp_box"])


@pytest.mark.parametrize("case", range(len(FLOW_LEVEL_CASES)))
def test_flow_level_matches_reference_fixture_bitwise(case):
    roi, box, mi, tol = FLOW_LEVEL_CASES[case]
    v, y, its = ob.flow_level32(FG["I1"], FG["I2"], FG["V0"], FG["Y0"], roi, box=box, max_iter=mi, tol=tol)
    np.testing.assert_array_equal(v, FG[f"level{case}_V"])
    # the reference writes Y back inside the ROI only; outside it Y keeps its input
    np.testing.assert_array_equal(y, FG[f"level{case}_Y"])
    if not 1.0 > tol:
        assert list(its) == [0, 0]  # the residual starts at 1: the loop never runs
    elif tol == 0.0:
        assert list(its) == [mi + 1, mi + 1]
    else:  # stops at a residual iteration (a multiple of 50) or runs out
        assert all(i == mi + 1 or i % 50 == 0 for i in its)


def test_flow_multiscale_matches_reference_fixture_bitwise():
    v = ob.flow_multiscale32(FG["ms_I1"], FG["ms_I2"], FG["ms_V0"], (3, 2, 2, 4, 1, 3), max_iter=12)
    np.testing.assert_array_equal(v, FG["ms_V"])


@pytest.mark.skipif(ob.REF is None, reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("dims,sigma,odim", [((17, 9, 12), 0.7, (30, 4, 12)), ((8, 8, 8), 2.0, (5, 13, 3))])
def test_cimg_image_ops_match_live_reference(dims, sigma, odim):
    rng = np.random.default_rng(sum(dims))
    nx, ny, nz = dims
    img = rng.normal(size=(3, nz, ny, nx)).astype(np.float32)
    np.testing.assert_array_equal(ob.blur32(img, sigma), ob.ref_blur(img, sigma))
    np.testing.assert_array_equal(ob.resize32(img, odim), ob.ref_resize(img, odim))
    np.testing.assert_array_equal(ob.gradient32(img[1]), ob.ref_gradient(img[1]))


@pytest.mark.skipif(ob.REF is None, reason="reference build (oracle/_ref) not present")
def test_flow_multiscale_matches_live_reference_with_tolerance_stop():
    rng = np.random.default_rng(77)
    shape = (13, 15, 14)
    i1 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), 1.2)
    i2 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), 1.2)
    v0 = np.zeros((3,) + shape, np.float32)
    # With an ROI the reference reads its unset gradient arrays outside the ROI
    # (optical_flow.h:263-290 fill them inside only) and sums them into the
    # residual, so whether a warp stops at a residual iteration depends on
    # uninitialised memory (a NaN there stops it even at tol 0).  Cases with
    # an ROI therefore stay below the first residual iteration (50).
    for cut, tol, mi in (((1, 1, 2, 1, 0, 1), 0.0, 40), ((0,) * 6, 0.0, 60), ((0,) * 6, 0.5, 75),
                         ((0,) * 6, 1.0, 10)):
        a = ob.flow_multiscale32(i1, i2, v0, cut, tol=tol, max_iter=mi, n_warps=2, scales=2, eta=0.7)
        b = ob.ref_flow_multiscale(i1, i2, v0, cut, tol=tol, max_iter=mi, n_warps=2, scales=2, eta=0.7)
        np.testing.assert_array_equal(a, b)


def test_fp64_row_band_equals_the_full_projection():
    """The band projection used to check 1024^2 views is the full FP64
    projection restricted to its rows."""
    s = ob.Scan((20, 18, 16), (24, 20), spacing=1.1, off=(0.5, -0.3, 0.8))
    vol = np.random.default_rng(4).uniform(0, 1, (16, 18, 20))
    v = ob.view_angle(0.7)
    full = ob.fp64(s, v, vol)[0]
    np.testing.assert_array_equal(ob.fp64_rows(s, v, vol, 5, 7), full[5:12])


def test_bf16_rounding_of_the_emulation_matches_torch():
    """oracle_bind.bf16_round (the BF16 store of the storage-mode emulation)
    rounds as torch's float32 -> bfloat16 conversion: nearest, ties to even."""
    import torch

    rng = np.random.default_rng(0)
    a = np.concatenate([rng.normal(size=4096).astype(np.float32) * 10.0 ** rng.integers(-30, 30, 4096),
                        np.array([1.0, 1.00390625, 1.005859375, -0.0, 0.0, 3.0e38], np.float32)]).astype(np.float32)
    ref = torch.from_numpy(a).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(ob.bf16_round(a), ref)
