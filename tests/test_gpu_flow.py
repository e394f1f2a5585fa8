"""Parity of the optical flow (optical_flow.h) and the CImg operations under it
with the oracle, through the C ABI.

The flow kernels follow the reference's float arithmetic operation by
operation, so every comparison here is bit-for-bit: against the oracle's FP32
restatement (itself pinned bit-for-bit to the reference's compiled code) and
against the committed reference fixtures.  The one non-deterministic part of
the reference, the residual sum that decides when a warp stops, is exercised
with settings whose stopping iteration does not depend on rounding.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

FG = np.load(Path(__file__).resolve().parent / "golden" / "reference_flow_golden.npz")


def _stt():
    import spacetimetomography_b200 as stt

    return stt


def _t(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


def _np(t):
    import torch

    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def _flow(shape, **kw):
    """shape = (nz, ny, nx), the torch shape of one image."""
    stt = _stt()
    return stt.Flow(shape, stt.FlowParams(**kw))


def _images(shape, seed, smooth=1.2):
    rng = np.random.default_rng(seed)
    i1 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), smooth)
    i2 = ob.blur32(rng.uniform(0, 1, shape).astype(np.float32), smooth)
    return i1, i2, rng


@pytest.mark.parametrize("box", [None, (23.0, 20.0, 21.0), (9.5, 30.0, 14.0)])
def test_warp_box_bitwise(cuda, box):
    stt = _stt()
    rng = np.random.default_rng(5)
    nz, ny, nx = 14, 13, 15
    vel = (rng.normal(size=(3, nz, ny, nx)) * 1.5).astype(np.float32)
    src = rng.normal(size=(2, nz, ny, nx)).astype(np.float32)
    b = (nx, ny, nz) if box is None else box
    for dt in (-1.0, 0.7):
        out = _np(stt.warp_box(_t(vel, cuda), _t(src, cuda), dt, b))
        np.testing.assert_array_equal(out, ob.warp_box32(vel, src, dt, b))


def test_warp_box_matches_reference_fixture(cuda):
    stt = _stt()
    out = _np(stt.warp_box(_t(FG["vel"], cuda), _t(FG["img"], cuda), -1.0, (17, 15, 13)))
    np.testing.assert_array_equal(out, FG["warp_box"])


def test_gradient_bitwise(cuda):
    stt = _stt()
    img = np.random.default_rng(6).normal(size=(9, 7, 12)).astype(np.float32)
    np.testing.assert_array_equal(_np(stt.image_gradient(_t(img, cuda))), ob.gradient32(img))
    np.testing.assert_array_equal(_np(stt.image_gradient(_t(FG["img"][0], cuda))), FG["grad"])


@pytest.mark.parametrize("sigma", [0.05, 0.5, 1.3, 4.0])
def test_blur_bitwise(cuda, sigma):
    f = _flow((16, 16, 16))
    img = np.random.default_rng(7).normal(size=(2, 9, 11, 13)).astype(np.float32)
    g = _t(img, cuda)
    f.blur(g, sigma)
    np.testing.assert_array_equal(_np(g), ob.blur32(img, sigma))
    one = np.random.default_rng(8).normal(size=(1, 5, 17)).astype(np.float32)  # a unit extent is skipped
    g1 = _t(one, cuda)
    f.blur(g1, sigma)
    np.testing.assert_array_equal(_np(g1), ob.blur32(one, sigma))


def test_blur_matches_reference_fixture(cuda):
    f = _flow((16, 16, 16))
    for sigma, key in ((0.5, "blur_05"), (1.3, "blur_13")):
        g = _t(FG["img"], cuda)
        f.blur(g, sigma)
        np.testing.assert_array_equal(_np(g), FG[key])


@pytest.mark.parametrize("odim", [(7, 6, 8), (16, 15, 12), (11, 5, 20), (11, 10, 9), (3, 31, 9), (2, 2, 40)])
def test_resize_bitwise(cuda, odim):
    f = _flow((32, 32, 48))
    img = FG["img"]
    out = _np(f.resize(_t(img, cuda), odim))
    np.testing.assert_array_equal(out, ob.resize32(img, odim))


def test_resize_matches_reference_fixture(cuda):
    f = _flow((32, 32, 32))
    for key in ("down", "up", "mixed"):
        out = _np(f.resize(_t(FG["img"], cuda), tuple(FG[f"resize_{key}_dim"])))
        np.testing.assert_array_equal(out, FG[f"resize_{key}"])


FLOW_LEVEL_CASES = [  # as tests/golden/gen_golden.py
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 20, 0.0),
    ((2, 1, 1, 3, 2, 2), (16, 13, 12), 30, 0.0),
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 120, 1e-3),
    ((0, 0, 0, 0, 0, 0), (11, 10, 9), 130, 1e30),
]


@pytest.mark.parametrize("case", range(len(FLOW_LEVEL_CASES)))
def test_flow_level_matches_reference_fixture(cuda, case):
    roi, box, mi, tol = FLOW_LEVEL_CASES[case]
    f = _flow((9, 10, 11), max_iter=mi, tol=tol, n_warps=2)
    V, Y = _t(FG["V0"], cuda), _t(FG["Y0"], cuda)
    f.level(_t(FG["I1"], cuda), _t(FG["I2"], cuda), V, Y, roi, box=box)
    np.testing.assert_array_equal(_np(V), FG[f"level{case}_V"])
    np.testing.assert_array_equal(_np(Y), FG[f"level{case}_Y"])
    its, _ = f.stats()
    _, _, its_o = ob.flow_level32(FG["I1"], FG["I2"], FG["V0"], FG["Y0"], roi, box=box, max_iter=mi, tol=tol)
    np.testing.assert_array_equal(its, its_o)


@pytest.mark.parametrize("roi,norm,huber,lam", [((0, 0, 0, 0, 0, 0), 4, 1.0, 1.2), ((3, 2, 1, 4, 2, 3), 4, 0.5, 0.8),
                                                 ((1, 1, 1, 1, 1, 1), 1, 1.0, 1.2)])
def test_flow_level_bitwise_with_residual_iterations(cuda, roi, norm, huber, lam):
    """160 iterations per warp (three residual evaluations), tol 0: the loop
    never stops early, so values must agree exactly."""
    shape = (17, 19, 21)
    i1, i2, rng = _images(shape, 11)
    v0 = (rng.normal(size=(3,) + shape) * 0.4).astype(np.float32)
    y0 = (rng.normal(size=(10,) + shape) * 0.05).astype(np.float32)
    box = (25.0, 19.0, 30.0)
    f = _flow(shape, max_iter=159, tol=0.0, n_warps=3, norm=norm, huber=huber, lam=lam)
    V, Y = _t(v0, cuda), _t(y0, cuda)
    f.level(_t(i1, cuda), _t(i2, cuda), V, Y, roi, box=box)
    vo, yo, its = ob.flow_level32(i1, i2, v0, y0, roi, box=box, tol=0.0, lam=lam, max_iter=159, norm=norm,
                                  n_warps=3, huber=huber)
    np.testing.assert_array_equal(_np(V), vo)
    np.testing.assert_array_equal(_np(Y), yo)
    np.testing.assert_array_equal(f.stats()[0], [160, 160, 160])


def test_flow_level_tolerance_stop(cuda):
    """Stopping on the residual: tol 0.9 stops each warp at its first check
    (iteration 50), tol 0.0019 after more checks (the residuals at the checks
    are >= 8 % away from it, far beyond summation-order rounding), tol >= 1
    never enters the loop (the residual starts at 1)."""
    shape = (12, 14, 13)
    i1, i2, rng = _images(shape, 12)
    v0 = np.zeros((3,) + shape, np.float32)
    y0 = np.zeros((10,) + shape, np.float32)
    for tol in (0.9, 0.0019, 1.0):
        vo, yo, its_o, err_o = ob.flow_level32(i1, i2, v0, y0, (0,) * 6, tol=tol, max_iter=400, n_warps=2, errs=True)
        f = _flow(shape, max_iter=400, tol=tol, n_warps=2)
        V, Y = _t(v0, cuda), _t(y0, cuda)
        f.level(_t(i1, cuda), _t(i2, cuda), V, Y, (0,) * 6)
        np.testing.assert_array_equal(_np(V), vo)
        np.testing.assert_array_equal(_np(Y), yo)
        its, err = f.stats()
        np.testing.assert_array_equal(its, its_o)
        if tol < 1.0:
            assert its_o[0] in (50, 150) and its_o[0] < 401
            np.testing.assert_allclose(err, err_o, rtol=1e-4)
        else:
            assert list(its) == [0, 0]


def test_flow_multiscale_matches_reference_fixture(cuda):
    f = _flow(FG["ms_I1"].shape, max_iter=12, tol=0.0, n_warps=2, cut=(3, 2, 2, 4, 1, 3))
    V = _t(FG["ms_V0"], cuda)
    f.multiscale(_t(FG["ms_I1"], cuda), _t(FG["ms_I2"], cuda), V)
    np.testing.assert_array_equal(_np(V), FG["ms_V"])


@pytest.mark.parametrize("scales,eta,cut,y0", [(3, 0.65, (8, 8, 8, 45, 8, 8), False), (2, 0.8, (0,) * 6, True),
                                               (1, 0.65, (2, 3, 1, 2, 2, 1), True)])
def test_flow_multiscale_bitwise(cuda, scales, eta, cut, y0):
    shape = (40, 64, 48)
    i1, i2, rng = _images(shape, 13, smooth=2.0)
    v0 = (rng.normal(size=(3,) + shape) * 0.2).astype(np.float32)
    Y0 = (rng.normal(size=(10,) + shape) * 0.05).astype(np.float32) if y0 else None
    f = _flow(shape, max_iter=40, tol=0.0, n_warps=2, scales=scales, eta=eta, cut=cut)
    V = _t(v0, cuda)
    f.multiscale(_t(i1, cuda), _t(i2, cuda), V, None if Y0 is None else _t(Y0, cuda))
    ref = ob.flow_multiscale32(i1, i2, v0, cut, Y=Y0, tol=0.0, max_iter=40, n_warps=2, eta=eta, scales=scales)
    np.testing.assert_array_equal(_np(V), ref)
    its, _ = f.stats()
    assert len(its) == 2 * scales and np.all(its == 41)


def test_flow_recovers_a_translation(cuda):
    """Physical sanity: I2 = I1 shifted by (1.5, -1, 0.5) voxels; the recovered
    flow in the interior approaches the shift."""
    stt = _stt()
    import torch

    n = 48
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    c = (n - 1) / 2

    def blob(dx, dy, dz):
        r2 = ((x - c - dx) / 9.0) ** 2 + ((y - c - dy) / 7.0) ** 2 + ((z - c - dz) / 8.0) ** 2
        return np.exp(-r2).astype(np.float32)

    i1, i2 = blob(0, 0, 0), blob(1.5, -1.0, 0.5)
    f = _flow((n, n, n), max_iter=300, tol=0.0, n_warps=3, scales=3, lam=0.3, cut=(0,) * 6)
    V = torch.zeros((3, n, n, n), device=cuda)
    f.multiscale(_t(i1, cuda), _t(i2, cuda), V)
    v = _np(V)
    core = (slice(int(c) - 4, int(c) + 4),) * 3
    mean = [float(v[k][core].mean()) for k in range(3)]
    # warp(V, I2, -1) samples I2 at x + V, so V is the displacement from I1 to I2
    assert abs(mean[0] - 1.5) < 0.25 and abs(mean[1] + 1.0) < 0.25 and abs(mean[2] - 0.5) < 0.25, mean


def test_flow_argument_errors(cuda):
    stt = _stt()
    with pytest.raises(stt.STTError):
        stt.Flow((8, 8, 8), stt.FlowParams(scales=5, eta=0.5))  # a level below 3 voxels
    f = _flow((8, 8, 8))
    import torch

    a = torch.zeros((9, 9, 9), device=cuda)
    with pytest.raises(stt.STTError):
        f.level(a, a, torch.zeros((3, 9, 9, 9), device=cuda), torch.zeros((10, 9, 9, 9), device=cuda), (0,) * 6)
