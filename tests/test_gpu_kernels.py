"""Parity of every libstt kernel with the oracle, through the C ABI.

Tolerances: 1e-4 relative L2 against the FP64 oracle and against the
reference's own FP32 arithmetic (oracle FP32 flavour, bit-exact with the
compiled reference); tighter where the kernel has no accumulation.
"""
import math

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _stt():
    import spacetimetomography_b200 as stt

    return stt


def _t(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


def phantom(dims, seed, n=8, semi=None, zero_boundary=True):
    """Ellipsoid phantom; by default its outer voxel shell is zeroed.

    The reference's march restarts before the entry point when the entry
    coordinate of a descending axis lies in [0, 0.5) (RayCaster.core.h:70-76,
    137), re-walking clamped boundary samples.  Whether a ray takes that branch
    can differ between FP32 and FP64 evaluation for rays right at the 0.5
    threshold; with a zero boundary shell the branch adds nothing, so the FP64
    comparison is well-posed.  test_fp_nonzero_boundary covers the other case.
    """
    from spacetimetomography_b200 import phantom as ph

    s = semi or (0.06 * min(dims), 0.3 * min(dims))
    v = ph.ellipsoid_phantom(dims, n, seed, semi=s).numpy()
    if zero_boundary:
        v[0], v[-1], v[:, 0], v[:, -1], v[:, :, 0], v[:, :, -1] = 0, 0, 0, 0, 0, 0
    return v


SCANS = [
    dict(n=32, det=(48, 40), spacing=1.0, off=(0.0, 0.0, 0.0)),
    dict(n=(40, 36, 28), det=(61, 45), spacing=1.0, off=(1.5, -2.0, 0.7)),
    dict(n=30, det=(64, 64), spacing=1.3, off=(0.0, 0.0, 0.0)),
    dict(n=24, det=(120, 96), spacing=1.0, off=(0.0, 0.0, 0.0)),   # many rays miss the volume
]
ROUND_VIEWS = [(0.0, 0), (17.3, 3), (90.0, 0), (200.5, 7), (12.0, 9)]


def make_ctx(scan: ob.Scan, angles):
    stt = _stt()
    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    return ctx


@pytest.mark.parametrize("si", range(len(SCANS)))
def test_fp_parity(cuda, si):
    import torch

    stt = _stt()
    sc = SCANS[si]
    scan = ob.Scan(sc["n"], sc["det"], spacing=sc["spacing"], off=sc["off"])
    vol = phantom(scan.dims, seed=si)
    angles = stt.views_from_rounds([s for s, _ in ROUND_VIEWS], 10)
    idx = [r * 10 + k for r, (_, k) in enumerate(ROUND_VIEWS)]
    ctx = make_ctx(scan, angles[idx])
    W, H = scan.det
    nv = len(idx)
    proj = torch.zeros((nv, H, W), device=cuda)
    rl = torch.zeros_like(proj)
    wt = torch.zeros_like(proj)
    ctx.fp(_t(vol, cuda), proj, raylen=rl, weight=wt)
    torch.cuda.synchronize()
    proj, rl, wt = _np(proj), _np(rl), _np(wt)
    for v, (sd, k) in enumerate(ROUND_VIEWS):
        ref32, rl32, w32 = ob.fp32(scan, ob.view_round(sd, k), vol, gmode=0)
        d64, rl64, w64 = ob.fp64(scan, ob.view_round(sd, k), vol)
        assert ob.rel_l2(proj[v], d64) < TOL
        assert ob.rel_l2(proj[v], ref32) < TOL
        assert np.mean(wt[v] == w64) > 0.999
        assert np.mean(wt[v] == w32) > 0.999
        hit = (w64 > 0) & (wt[v] > 0)
        # tfar - tnear of two ~600 mm floats: ~1e-4 mm absolute rounding, as in the reference
        assert np.max(np.abs(rl[v][hit] - rl64[hit])) < 2e-4
        if ob.REF is not None:
            r_img, r_rl, r_w = ob.ref_fp(scan, sd, k, vol)
            np.testing.assert_array_equal(r_img, ref32)
            assert ob.rel_l2(proj[v], r_img) < TOL


def test_fp_nonzero_boundary(cuda):
    """Non-zero boundary voxels: the kernel takes the reference's FP32 branch decisions."""
    import torch

    stt = _stt()
    scan = ob.Scan(30, (64, 64), spacing=1.3)
    vol = phantom(scan.dims, seed=2, zero_boundary=False) + 0.25
    angles = stt.views_from_rounds([s for s, _ in ROUND_VIEWS], 10)
    idx = [r * 10 + k for r, (_, k) in enumerate(ROUND_VIEWS)]
    ctx = make_ctx(scan, angles[idx])
    proj = torch.zeros((len(idx), 64, 64), device=cuda)
    wt = torch.zeros_like(proj)
    ctx.fp(_t(vol, cuda), proj, weight=wt)
    proj, wt = _np(proj), _np(wt)
    for v, (sd, k) in enumerate(ROUND_VIEWS):
        ref32, _, w32 = ob.fp32(scan, ob.view_round(sd, k), vol, gmode=0)
        d64, _, w64 = ob.fp64(scan, ob.view_round(sd, k), vol)
        assert ob.rel_l2(proj[v], ref32) < TOL
        flip = wt[v] != w64
        assert np.mean(flip) < 2e-3
        assert ob.rel_l2(proj[v][~flip], d64[~flip]) < TOL


def test_fp_axis_aligned_and_odd_detector(cuda):
    """Odd W/H at 0 and 90 degrees: rays with exactly zero direction components."""
    import torch

    scan = ob.Scan(33, (35, 33))
    vol = phantom(scan.dims, seed=7)
    angles = np.array([0.0, math.pi / 2, math.pi, 1.5 * math.pi])
    ctx = make_ctx(scan, angles)
    proj = torch.zeros((4, 33, 35), device=cuda)
    wt = torch.zeros_like(proj)
    ctx.fp(_t(vol, cuda), proj, weight=wt)
    proj, wt = _np(proj), _np(wt)
    for v, a in enumerate(angles):
        d64, _, w64 = ob.fp64(scan, ob.view_angle(a), vol)
        assert ob.rel_l2(proj[v], d64) < TOL
        assert np.mean(wt[v] == w64) > 0.999


def test_fp_correction_sticky_raylength(cuda):
    import torch

    scan = ob.Scan(32, (80, 64))
    vol = phantom(scan.dims, seed=3)
    angles = np.array([0.3, 1.9, 4.0])
    ctx = make_ctx(scan, angles)
    W, H = scan.det
    rng = np.random.default_rng(0)
    b = rng.uniform(0, 20, (3, H, W)).astype(np.float32)
    state = torch.zeros((H, W), device=cuda)
    corr = torch.zeros((H, W), device=cuda)
    st_ref = np.zeros((H, W), np.float64)
    for v in range(3):
        ctx.fp_correction(_t(vol, cuda), _t(b[v], cuda), state, corr, v)
        d64, rl64, w64 = ob.fp64(scan, ob.view_angle(angles[v]), vol)
        st_ref = np.where(w64 > 0, rl64, st_ref)
        c_ref = (b[v] - d64) / (st_ref + 1.0)
        assert ob.rel_l2(_np(corr), c_ref) < TOL
        assert np.max(np.abs(_np(state) - st_ref)) < 2e-4


def test_fp_adjoint_dot_product(cuda):
    import torch

    scan = ob.Scan((36, 30, 34), (50, 44), off=(0.5, 1.0, -0.5))
    angles = np.array([0.1, 1.1, 2.6, 3.9])
    ctx = make_ctx(scan, angles)
    rng = np.random.default_rng(5)
    nx, ny, nz = scan.dims
    W, H = scan.det
    x = rng.normal(size=(nz, ny, nx)).astype(np.float32)
    y = rng.normal(size=(4, H, W)).astype(np.float32)
    ax = torch.zeros((4, H, W), device=cuda)
    ctx.fp(_t(x, cuda), ax)
    aty = torch.zeros((nz, ny, nx), device=cuda)
    ctx.fp_vjp(_t(y, cuda), aty)
    lhs = float(np.sum(_np(ax).astype(np.float64) * y))
    rhs = float(np.sum(x.astype(np.float64) * _np(aty)))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    ref64 = sum(ob.fp_adjoint64(scan, ob.view_angle(a), y[v]) for v, a in enumerate(angles))
    ref32 = sum(ob.fp_adjoint32(scan, ob.view_angle(a), y[v]).astype(np.float64) for v, a in enumerate(angles))
    # same FP32 march as the kernel: only the atomic summation order differs
    assert ob.rel_l2(_np(aty), ref32) < 1e-5
    # against the FP64 march: sample positions differ by float rounding, and
    # a random y gives each voxel few, sign-mixed contributions
    assert ob.rel_l2(_np(aty), ref64) < TOL


@pytest.mark.parametrize("alpha", [0.3, 1.0])
def test_bp_voxel(cuda, alpha):
    import torch

    scan = ob.Scan((34, 30, 32), (48, 40), off=(0.7, -0.4, 1.1))
    ctx = make_ctx(scan, np.array([0.7, 2.2]))
    rng = np.random.default_rng(1)
    nx, ny, nz = scan.dims
    corr = rng.normal(size=(40, 48)).astype(np.float32)
    vol = rng.uniform(0, 2, (nz, ny, nx)).astype(np.float32)
    gmax = 2.5
    for v, a in enumerate([0.7, 2.2]):
        g = _t(vol, cuda)
        ctx.bp_voxel(_t(corr, cuda), g, alpha, gmax, v)
        out = _np(g)
        ref = ob.bp_voxel64(scan, ob.view_angle(a), corr, alpha, gmax, vol)
        assert ob.rel_l2(out - vol, ref - vol) < TOL
        g2 = _t(vol, cuda)
        ctx.bp_voxel(_t(corr, cuda), g2, alpha, gmax, v)
        np.testing.assert_array_equal(_np(g2), out)  # deterministic gather


def test_bp_ray(cuda):
    scan = ob.Scan(28, (44, 40))
    ctx = make_ctx(scan, np.array([0.4, 3.3]))
    rng = np.random.default_rng(2)
    corr = rng.normal(size=(40, 44)).astype(np.float32)
    vol = rng.uniform(0, 1, (28, 28, 28)).astype(np.float32)
    gmax = 1.7
    for v, a in enumerate([0.4, 3.3]):
        g = _t(vol, cuda)
        ctx.bp_ray(_t(corr, cuda), g, gmax, v)
        c, w = ob.bp_ray_scatter32(scan, ob.view_angle(a), corr, gmode=1)
        with np.errstate(invalid="ignore", divide="ignore"):
            ref = np.clip(vol + c / w, 0, gmax)
        ref = np.where(np.isnan(vol + c / w), 0.0, ref)
        assert ob.rel_l2(_np(g), ref) < TOL


@pytest.mark.parametrize("bp_mode", [0, 1])
def test_sart_sweep(cuda, bp_mode):
    import torch

    stt = _stt()
    scan = ob.Scan(32, (48, 48))
    truth = phantom(scan.dims, seed=11)
    nv = 24
    angles = np.arange(nv) * (2 * math.pi / nv)
    ctx = make_ctx(scan, angles)
    proj = np.stack([ob.fp64(scan, ob.view_angle(a), truth)[0] for a in angles]).astype(np.float32)
    gmax = float(proj.max() / 4.0)
    perm = stt.permutation(1234, nv)
    vol0 = np.zeros_like(truth)
    roi_cut = (4, 4, 4, 6, 4, 4, 8, 6)
    roi = ob.roi_mask(scan.dims, roi_cut)
    g = _t(vol0, cuda)
    state = torch.zeros((48, 48), device=cuda)
    ctx.sart_sweep(g, _t(proj, cuda), perm, 0.3, gmax, bp_mode, state, roi_cut=roi_cut)
    ctx.sart_sweep(g, _t(proj, cuda), perm[::-1].copy(), 0.3, gmax, bp_mode, state, roi_cut=roi_cut)
    views = [ob.view_angle(a) for a in angles]
    ref, rl = ob.sart64(scan, views, perm, proj, 0.3, gmax, bp_mode, vol0, roi=roi)
    ref, rl = ob.sart64(scan, views, perm[::-1].copy(), proj, 0.3, gmax, bp_mode, ref, raylen=rl, roi=roi)
    assert ob.rel_l2(_np(g), ref) < TOL
    assert np.max(np.abs(_np(state) - rl)) < 2e-4


def test_pd_steps(cuda):
    import torch

    stt = _stt()
    dims = (40, 56, 36)
    nx, ny, nz = dims
    cut = (4, 4, 4, 9, 4, 4, 6, 5)
    scan = ob.Scan(dims, (48, 48))
    ctx = make_ctx(scan, np.array([0.0]))
    rng = np.random.default_rng(4)
    sh = (nz, ny, nx)
    xf, xf1, bw, ytp, ybc, ytp_prev, fw, vol = (rng.normal(size=sh).astype(np.float32) for _ in range(8))
    vol = np.abs(vol)
    ytv = rng.normal(size=(3,) + sh).astype(np.float32) * 0.05
    p = stt.PdParams(sigma=0.1125, tau=1.0, tv_w=0.05, tp_w=0.3, bc_w=0.4, huber_factor=0.9, gmax=1.5, cut=cut)
    op = ob.OPd(p.sigma, p.tau, p.tv_w, p.tp_w, p.bc_w, p.huber_factor, p.gmax, (ob.C.c_int * 8)(*cut))
    g_ytv, g_ytp, g_ybc = _t(ytv, cuda), _t(ytp, cuda), _t(ybc, cuda)
    ctx.pd_dual(p, _t(xf, cuda), _t(xf1, cuda), _t(bw, cuda), g_ytv, g_ytp, g_ybc)
    r_ytv, r_ytp, r_ybc = ob.pd_dual32(dims, op, xf, xf1, bw, ytv, ytp, ybc)
    for a, b in ((g_ytv, r_ytv), (g_ytp, r_ytp), (g_ybc, r_ybc)):
        assert ob.rel_l2(_np(a), b) < 1e-6
    for first in (1, 0):
        g_vol, g_xp = _t(vol, cuda), torch.zeros(sh, device=cuda)
        ctx.pd_primal(p, first, _t(ytp_prev, cuda), _t(r_ytp, cuda), _t(fw, cuda), _t(r_ybc, cuda),
                      _t(r_ytv, cuda), g_vol, g_xp)
        r_vol, r_xp = ob.pd_primal32(dims, op, first, ytp_prev, r_ytp, fw, r_ybc, r_ytv, vol)
        assert ob.rel_l2(_np(g_vol), r_vol) < 1e-6
        np.testing.assert_array_equal(_np(g_xp), r_xp)
    xbar = rng.normal(size=sh).astype(np.float32)
    g_xbar = _t(xbar, cuda)
    ctx.pd_extrapolate(cut, _t(r_vol, cuda), _t(r_xp, cuda), g_xbar)
    r_xbar = ob.pd_extrapolate32(dims, cut, r_vol, r_xp, xbar)
    np.testing.assert_allclose(_np(g_xbar), r_xbar, rtol=1e-6, atol=1e-6)
    roi = torch.zeros(sh, device=cuda)
    ctx.roi_mask((8, 8, 8, 45, 8, 8, 30, 20), roi)
    np.testing.assert_array_equal(_np(roi), ob.roi_mask(dims, (8, 8, 8, 45, 8, 8, 30, 20)))


@pytest.mark.parametrize("dim,nc,dt", [((24, 20, 16), 1, 1.0), ((33, 17, 21), 2, -1.0), ((20, 20, 20), 3, 0.37)])
def test_warp(cuda, dim, nc, dt):
    stt = _stt()
    rng = np.random.default_rng(9)
    nx, ny, nz = dim
    vel = (rng.normal(size=(3, nz, ny, nx)) * 1.5).astype(np.float32)
    src = rng.normal(size=(nc, nz, ny, nx)).astype(np.float32)
    out = _np(stt.warp(_t(vel, cuda), _t(src, cuda), dt))
    r32 = ob.warp32(vel, src, dt)
    r64 = ob.warp64(vel, src, dt)
    assert ob.rel_l2(out, r64) < 1e-5
    assert ob.rel_l2(out, r32) < 1e-5
    if ob.REF is not None:
        np.testing.assert_array_equal(ob.ref_warp(vel, src, dt), r32)


@pytest.mark.parametrize("rough,dt", [(False, 1.0), (False, -1.0), (True, 1.0)])
def test_warp_staged_equals_gathered(cuda, rough, dt):
    """stt_warp stages the velocity around each block with TMA when nx is a
    multiple of 4 and the flow is 16-byte aligned; a flow one float off that
    alignment takes the gather kernel.  Both must give the same bits, for a
    smooth flow (every stencil in its box) and a rough one (many fall back)."""
    import torch

    stt = _stt()
    nx, ny, nz = 48, 40, 36
    z, y, x = np.mgrid[0:nz, 0:ny, 0:nx].astype(np.float32)
    if rough:
        vel = (np.random.default_rng(12).normal(size=(3, nz, ny, nx)) * 3.0).astype(np.float32)
    else:
        vel = np.stack([2.5 * np.sin(0.2 * y + 0.1 * z), 1.5 * np.cos(0.15 * x), 1.2 * np.sin(0.1 * x + 0.2 * y)])
        vel = vel.astype(np.float32)
    src = np.random.default_rng(13).normal(size=(2, nz, ny, nx)).astype(np.float32)
    v_al = _t(vel, cuda)
    buf = torch.empty(vel.size + 1, device=cuda)
    v_off = buf[1:].view(vel.shape)
    v_off.copy_(v_al)
    assert v_al.data_ptr() % 16 == 0 and v_off.data_ptr() % 16 != 0
    s_d = _t(src, cuda)
    a = _np(stt.warp(v_al, s_d, dt))
    b = _np(stt.warp(v_off, s_d, dt))
    np.testing.assert_array_equal(a, b)
    assert ob.rel_l2(a, ob.warp64(vel, src, dt)) < 1e-5


def test_warp_vjp(cuda):
    import torch

    stt = _stt()
    rng = np.random.default_rng(10)
    nx, ny, nz = 20, 18, 16
    vel = (rng.normal(size=(3, nz, ny, nx)) * 0.8).astype(np.float32)
    src = rng.normal(size=(2, nz, ny, nx)).astype(np.float32)
    obar = rng.normal(size=(2, nz, ny, nx)).astype(np.float32)
    sb = torch.zeros((2, nz, ny, nx), device=cuda)
    vb = torch.zeros((3, nz, ny, nx), device=cuda)
    stt.warp_vjp(_t(vel, cuda), _t(src, cuda), 1.0, _t(obar, cuda), sb, vb)
    rs, rv = ob.warp_vjp64(vel.astype(np.float64), src.astype(np.float64), 1.0, obar.astype(np.float64))
    assert ob.rel_l2(_np(sb), rs) < 1e-5
    assert ob.rel_l2(_np(vb), rv) < 1e-4


@pytest.mark.parametrize("dims,det,off", [((96, 80, 112), (160, 144), (1.5, -0.7, 2.0)),
                                          ((128, 128, 128), (192, 192), (0.0, 0.0, 0.0))])
def test_bp_ray_scatter_slab_vs_sequential_oracle(cuda, dims, det, off):
    """The slab-staged scatter (shared-memory box per slab, k_bp_slab.cu)
    against the oracle's sequential scatter in FP32, on sizes where a block
    walks many slabs: views along both axes, oblique views, an off-centre
    volume and rays that miss."""
    import torch

    scan = ob.Scan(dims, det, off=off)
    angles = np.array([0.0, 0.2, 0.7, 1.3, 1.5708, 2.6, 3.9, 5.5])
    ctx = make_ctx(scan, angles)
    rng = np.random.default_rng(5)
    W, H = det
    nx, ny, nz = dims
    for v, a in enumerate(angles):
        corr = rng.normal(size=(H, W)).astype(np.float32)
        c = torch.zeros((nz, ny, nx), device=cuda)
        w = torch.zeros((nz, ny, nx), device=cuda)
        ctx.bp_ray_scatter(_t(corr, cuda), c, w, v)
        c_ref, w_ref = ob.bp_ray_scatter32(scan, ob.view_angle(a), corr, gmode=1)
        assert ob.rel_l2(_np(w), w_ref) < 1e-5, (v, ob.rel_l2(_np(w), w_ref))
        assert ob.rel_l2(_np(c), c_ref) < 1e-5, (v, ob.rel_l2(_np(c), c_ref))
    ctx.close()


def test_gather_ceiling_packed_pairs_equal_scalar(cuda):
    """The gather ceiling in packed FP32x2 pairs (fp_cell2/trilerp2, the
    helpers of the packed projector variants) gives the scalar form's bits,
    so does its tld4 form (fp_corners_tex, the corner fetch of the texture
    projector variants), and its sums track the projector's (same rays,
    nearly the same samples)."""
    import torch

    scan = ob.Scan((64, 56, 72), (96, 80), off=(0.7, -1.1, 0.4))
    angles = np.array([0.0, 0.3, 0.9, 1.5708, 2.4])
    ctx = make_ctx(scan, angles)
    vol = _t(phantom(scan.dims, seed=3), cuda)
    W, H = scan.det
    for v in range(len(angles)):
        a = torch.zeros((H, W), device=cuda)
        b = torch.zeros((H, W), device=cuda)
        n = torch.zeros((H, W), dtype=torch.int32, device=cuda)
        ctx.gather_ceiling(vol, v, a, n, packed=True)
        ctx.gather_ceiling(vol, v, b, packed=False)
        np.testing.assert_array_equal(_np(a), _np(b))
        assert ctx.fp_texture_ok(vol)
        ctx.gather_ceiling(vol, v, b, texture=True)
        np.testing.assert_array_equal(_np(a), _np(b))
        proj = torch.zeros((1, H, W), device=cuda)
        ctx.fp(vol, proj, view0=v, nviews=1)
        assert ob.rel_l2(_np(a), _np(proj)[0]) < 0.05
        assert int(n.sum()) > 0
    ctx.close()
