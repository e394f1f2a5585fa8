"""Parity at the single-frame workloads' full sizes (128^3 / 128^2 with 128
views; 256^3 / 512^2 with 360 views; 512^3 / 1024^2 with 720 views), through
the C ABI, on seeded samples the FP64 oracle finishes in seconds, and through
size-independent identities:

* SART sweeps against the FP64 oracle (relative L2 below 1e-4);
* the dot-product test <A x, y> = <x, A^T y> of the projector and its exact
  adjoint (stt_fp / stt_fp_vjp), accumulated in FP64;
* an FP64 finite-difference check of the data-term gradient
  A^T (A x - b) (GPU, FP32) against central differences of
  f(x) = |A x - b|^2 / 2 evaluated with the FP64 oracle's projector;
* at 512^3, where one FP64 projection of a 1024^2 view takes minutes, a
  64-row band of the forward projection and the voxel backprojection of one
  view's correction against the FP64 oracle.

Reference loops: ST_Tomography.cpp:616-808 (SART), :690-730 (voxel BP),
:733-764 (ray BP); TypicalRayProducer.core.h:123-268 (projector)."""
import math

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu


def _ctx(scan, angles):
    import spacetimetomography_b200 as stt

    c = stt.Context(0)
    c.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    return c


def _phantom(n, count, seed, cuda, porous=False):
    from spacetimetomography_b200 import phantom as ph

    dims = (n, n, n)
    s = n / 256.0
    bg = ph.porous_background(dims, 77, n ** 3 // 1000, device=cuda) if porous else None
    return ph.rasterize(ph.ellipsoid_params(count, dims, seed=seed, semi=(5.0 * s, 40.0 * s)), dims, cuda,
                        background=bg)


@pytest.mark.parametrize("n,det,views,nsweep,bp_mode", [(128, 128, 128, 128, 0), (256, 512, 360, 3, 0),
                                                        (256, 512, 360, 2, 1)])
def test_sart_sweep_at_full_size_vs_fp64(cuda, n, det, views, nsweep, bp_mode):
    import torch

    scan = ob.Scan(n, det)
    angles = np.arange(views) * (2 * math.pi / views)
    ctx = _ctx(scan, angles)
    truth = _phantom(n, 12 if n == 128 else 30, 101, cuda)
    proj = torch.empty((views, det, det), device=cuda)
    ctx.fp(truth, proj)
    torch.cuda.synchronize()
    gmax = float(proj.max()) / 4
    order = [int(v) for v in np.linspace(0, views - 1, nsweep)]
    start = (truth * 0.8).contiguous()
    vol = start.clone()
    state = torch.zeros((det, det), device=cuda)
    ctx.sart_sweep(vol, proj, order, 0.3, gmax, bp_mode, state)
    torch.cuda.synchronize()
    ctx.poll_status()
    views = [ob.view_angle(a) for a in angles]
    got = vol.cpu().numpy()
    # the reference's FP32 arithmetic (the restatement, pinned bit for bit to the
    # reference's SART): the same within float rounding (and atomic order)
    ref32, _ = ob.sart32(scan, views, order, proj.cpu().numpy(), 0.3, gmax, bp_mode, start.cpu().numpy(), gmode=1)
    assert ob.rel_l2(got, ref32) < 1e-5, ob.rel_l2(got, ref32)
    ref, _ = ob.sart64(scan, views, order, proj.cpu().numpy().astype(np.float64), 0.3,
                       gmax, bp_mode, start.cpu().numpy().astype(np.float64))
    e = ob.rel_l2(got, ref)
    if bp_mode == 0:
        assert e < 1e-4, e
    else:
        # The ray-driven update is contrib/weight per voxel: a voxel that one
        # evaluation's samples barely touch (weight ~1e-6) takes the whole
        # correction there and none in the other (0/0 -> 0).  Where the FP32
        # march and the FP64 one touch a voxel differently, the two differ by a
        # full correction value: the reference's FP32 arithmetic itself lies
        # about 1e-3 from FP64 at 256^3 / 512^2 (measured 8.4e-4), so the FP64
        # error of this path is held to 2e-3.
        assert e < 2e-3, e
    ctx.close()


@pytest.mark.parametrize("n,det,views", [(256, 512, 360), (512, 1024, 720)])
def test_dot_product_adjoint_at_full_size(cuda, n, det, views):
    import torch

    scan = ob.Scan(n, det)
    angles = np.arange(views) * (2 * math.pi / views)
    ctx = _ctx(scan, angles)
    g = torch.Generator(device=cuda)
    g.manual_seed(5)
    x = torch.rand((n, n, n), device=cuda, generator=g)
    sel = [0, views // 8, views // 3]  # 0, 45 and 120 degrees
    y = torch.rand((1, det, det), device=cuda, generator=g)
    for v in sel:
        ax = torch.zeros((1, det, det), device=cuda)
        ctx.fp(x, ax, view0=v, nviews=1)
        aty = torch.zeros((n, n, n), device=cuda)
        ctx.fp_vjp(y, aty, view0=v, nviews=1)
        torch.cuda.synchronize()
        lhs = float((ax.double() * y.double()).sum())
        rhs = float((x.double() * aty.double()).sum())
        assert abs(lhs - rhs) <= 2e-5 * abs(lhs), (v, lhs, rhs)
    ctx.close()


def test_data_gradient_fp64_finite_difference_256(cuda):
    """d/de f(x + e d) at e = 0 for f = |A x - b|^2 / 2 on one view: the GPU's
    <A^T (A x - b), d> against an FP64 central difference of the oracle's f
    (exact for this quadratic up to rounding).  The direction d is a second,
    non-negative phantom: a zero-mean random d would make the inner product a
    near-cancelling sum whose value the rounding of single samples decides."""
    import torch

    n, det = 256, 512
    scan = ob.Scan(n, det)
    angle = 0.7
    ctx = _ctx(scan, [angle])
    x = _phantom(n, 30, 7, cuda)
    d = (_phantom(n, 20, 8, cuda) + 0.05).contiguous()
    b = torch.zeros((1, det, det), device=cuda)
    ctx.fp((x * 1.1).contiguous(), b)
    ax = torch.zeros((1, det, det), device=cuda)
    ctx.fp(x, ax)
    grad = torch.zeros((n, n, n), device=cuda)
    ctx.fp_vjp((ax - b).contiguous(), grad)
    torch.cuda.synchronize()
    g_gpu = float((grad.double() * d.double()).sum())
    xs, ds, bs = x.cpu().numpy().astype(np.float64), d.cpu().numpy().astype(np.float64), b.cpu().numpy()[0]
    eps = 1e-3

    def f(e):
        p = ob.fp64(scan, ob.view_angle(angle), xs + e * ds)[0]
        return 0.5 * float(((p - bs) ** 2).sum())
    g_fd = (f(eps) - f(-eps)) / (2 * eps)
    assert abs(g_gpu - g_fd) <= 1e-4 * abs(g_fd), (g_gpu, g_fd)
    ctx.close()


def test_512_band_and_voxel_backprojection_vs_fp64(cuda):
    import torch

    n, det, views = 512, 1024, 720
    scan = ob.Scan(n, det)
    angles = np.arange(views) * (2 * math.pi / views)
    v = views // 8  # 45 degrees: the slab-staged projector's case
    ctx = _ctx(scan, angles)
    truth = _phantom(n, 100, 105, cuda, porous=True)
    img = torch.zeros((1, det, det), device=cuda)
    ctx.fp(truth, img, view0=v, nviews=1)
    torch.cuda.synchronize()
    t32 = truth.cpu().numpy()
    r0 = det // 2 - 32
    got = img[0, r0:r0 + 64].cpu().numpy()
    # the reference's FP32 arithmetic: the same within float rounding
    band32 = ob.fp32_rows(scan, ob.view_angle(angles[v]), t32, r0, 64)
    assert ob.rel_l2(got, band32) < 1e-5, ob.rel_l2(got, band32)
    # FP64: the reference's march steps its sample positions in FP32 (t += sd,
    # pos += step over ~600 samples per ray here), and at 512^3 the porous
    # background's sharp sphere edges turn that position drift into ~1e-4 of
    # the line integrals (measured 1.1e-4); held to 2e-4
    band = ob.fp64_rows(scan, ob.view_angle(angles[v]), t32.astype(np.float64), r0, 64)
    assert ob.rel_l2(got, band) < 2e-4, ob.rel_l2(got, band)
    # one view's correction and its voxel backprojection
    b = torch.zeros((det, det), device=cuda)
    ctx.fp(truth, b[None], view0=v, nviews=1)
    start = (truth * 0.8).contiguous()
    corr = torch.zeros((det, det), device=cuda)
    rl = torch.zeros((det, det), device=cuda)
    ctx.fp_correction(start, b, rl, corr, v)
    vol = start.clone()
    gmax = float(b.max()) / 4
    ctx.bp_voxel(corr, vol, 0.3, gmax, v)
    torch.cuda.synchronize()
    ctx.poll_status()
    s64 = start.cpu().numpy().astype(np.float64)
    ref = ob.bp_voxel64(scan, ob.view_angle(angles[v]), corr.cpu().numpy().astype(np.float64), 0.3, gmax, s64.copy())
    upd = vol.cpu().numpy().astype(np.float64) - s64
    assert ob.rel_l2(vol.cpu().numpy(), ref) < 1e-6
    assert ob.rel_l2(upd, ref - s64) < 1e-4
    ctx.close()
