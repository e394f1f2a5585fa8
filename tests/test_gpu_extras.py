"""The entries of the ABI around the projector that the reference has no
single function for: the BF16-stored forward projection, one SART view on
its own, and the FP64 power iteration for the operator norm."""
import math

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu


def _stt():
    import spacetimetomography_b200 as stt

    return stt


def _scan_ctx(scan, angles, cuda):
    stt = _stt()
    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    return ctx


def _phantom(dims, seed):
    from spacetimetomography_b200 import phantom as ph

    v = ph.ellipsoid_phantom(dims, 6, seed, semi=(2.0, 0.3 * min(dims))).numpy()  # (nz, ny, nx)
    return np.ascontiguousarray(v, np.float32)


def test_fp_bf16_storage(cuda):
    """BF16 storage: the FP32 projection of the widened volume (the taps are
    exact), and within the BF16 rounding of the FP32 projection."""
    import torch

    scan = ob.Scan((40, 36, 28), (61, 45), off=(1.5, -2.0, 0.7))
    angles = np.array([0.1, 0.9, 1.6, 2.7, 4.0])  # x- and z-dominant views
    ctx = _scan_ctx(scan, angles, cuda)
    nx, ny, nz = scan.dims
    vol = torch.from_numpy(_phantom((nx, ny, nz), 3) + 0.01).to(cuda)
    v16 = vol.to(torch.bfloat16)
    p16 = torch.zeros((len(angles), 45, 61), device=cuda)
    ctx.fp_typed(v16, p16)
    pw = torch.zeros_like(p16)
    ctx.fp(v16.float().contiguous(), pw)
    p32 = torch.zeros_like(p16)
    ctx.fp_typed(vol, p32)
    torch.cuda.synchronize()
    # the same taps; the compiler contracts the two instantiations' arithmetic
    # differently in a few places, so up to an ulp apart
    np.testing.assert_allclose(p16.cpu().numpy(), pw.cpu().numpy(), rtol=1e-6, atol=1e-6)
    ref = np.stack([ob.fp64(scan, ob.view_angle(a), vol.cpu().numpy().astype(np.float64))[0] for a in angles])
    e16 = ob.rel_l2(p16.cpu().numpy(), ref)
    e32 = ob.rel_l2(p32.cpu().numpy(), ref)
    assert e32 < 1e-4  # nonzero boundary: the FP32 march takes the reference's restart decisions
    assert e16 < 4e-3, e16


@pytest.mark.parametrize("bp_mode", [0, 1])
def test_sart_view_equals_a_one_view_sweep(cuda, bp_mode):
    import torch

    stt = _stt()
    scan = ob.Scan((32, 30, 28), (48, 44))
    angles = np.arange(6) * (2 * math.pi / 6) + 0.2
    ctx = _scan_ctx(scan, angles, cuda)
    nx, ny, nz = scan.dims
    truth = _phantom((nx, ny, nz), 4)
    proj = torch.zeros((6, 44, 48), device=cuda)
    ctx.fp(torch.from_numpy(truth).to(cuda), proj)
    order = [3, 0, 5, 1, 4, 2]
    gmax = float(proj.max().item() / 4)
    a = torch.zeros((nz, ny, nx), device=cuda)
    b = torch.zeros_like(a)
    ra = torch.zeros((44, 48), device=cuda)
    rb = torch.zeros_like(ra)
    for v in order:
        ctx.sart_view(a, proj[v].contiguous(), v, 0.3, gmax, bp_mode, ra)
    ctx.sart_sweep(b, proj, np.array(order, np.int32), 0.3, gmax, bp_mode, rb)
    torch.cuda.synchronize()
    if bp_mode == 0:
        np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    else:  # float atomics in the scatter
        assert ob.rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5
    assert a.abs().max().item() > 0


def test_opnorm_power_iteration_against_fp64_oracle(cuda):
    stt = _stt()
    scan = ob.Scan((20, 18, 16), (32, 28), spacing=1.1)
    angles = np.arange(8) * (2 * math.pi / 8) + 0.1
    ctx = _scan_ctx(scan, angles, cuda)
    r = ctx.opnorm(n_iter=80, seed=7)
    views = [ob.view_angle(a) for a in angles]
    x = np.ones((16, 18, 20))
    x /= np.linalg.norm(x)
    lam = 0.0
    for _ in range(80):
        ax = np.zeros_like(x)
        for v in views:
            ax += ob.fp_adjoint64(scan, v, ob.fp64(scan, v, x)[0])
        lam = float((x * ax).sum())
        x = ax / np.linalg.norm(ax)
    ref = math.sqrt(lam)
    assert abs(r["norm_A"] - ref) / ref < 1e-3, (r, ref)
    assert r["rel_change"] < 1e-4
    assert r["iterations"] == 80
    assert r["sigma"] * r["tau"] * r["norm_K"] ** 2 < 1.0
    assert abs(r["norm_K"] ** 2 - (r["norm_A"] ** 2 + 12.0)) < 1e-6 * r["norm_K"] ** 2
    with pytest.raises(stt.STTError):
        ctx.opnorm(n_iter=0)


INSTANCES = [  # dims (nx, ny, nz), views, detector (W, H), sid, sdd
    ((40, 36, 32), 12, (64, 56), 600.0, 1000.0),
    ((24, 24, 24), 8, (40, 40), 520.0, 950.0),
    ((48, 40, 36), 10, (72, 64), 680.0, 1080.0),
]


def _instance(k, cuda):
    import torch

    stt = _stt()
    dims, V, det, sid, sdd = INSTANCES[k]
    scan = ob.Scan(dims, det, sid=sid, sdd=sdd)
    angles = np.arange(V) * (2 * math.pi / V) + 0.13 * k
    ctx = _scan_ctx(scan, angles, cuda)
    truth = torch.from_numpy(_phantom(dims, 20 + k)).to(cuda)
    proj = torch.zeros((V, det[1], det[0]), device=cuda)
    ctx.fp(truth, proj)
    torch.cuda.synchronize()
    gmax = float(proj[0].max().item() / 4)
    pd = stt.PdParams(tv_w=0.01, tp_w=0.0, bc_w=0.0, huber_factor=0.9, gmax=gmax, cut=(2, 2, 2, 2, 2, 2, 3, 3))
    return ctx, proj, pd, truth


@pytest.mark.parametrize("bp_mode", [0, 1])
def test_batch_of_uneven_instances_equals_separate_solves(cuda, bp_mode):
    """Three instances of different volume, detector and view counts iterated
    as one graph (and as concurrent streams) give each instance's own
    single-frame solve."""
    import torch

    stt = _stt()
    made = [_instance(k, cuda) for k in range(len(INSTANCES))]
    cut = (2, 2, 2, 2, 2, 2, 3, 3)
    results = {}
    for mode in (stt.SOLVE_GRAPH, stt.SOLVE_STREAMS):
        inst = []
        for k, (ctx, proj, pd, truth) in enumerate(made):
            inst.append(dict(ctx=ctx, vol=torch.zeros_like(truth), proj=proj, bp_mode=bp_mode, alpha=0.3, pd=pd,
                             roi_cut=cut, seed=100 + k))
        b = stt.Batch(inst, mode=mode)
        b.iterate(3)
        torch.cuda.synchronize()
        results[mode] = [d["vol"].cpu().numpy() for d in inst]
        b.close()
    for k, (ctx, proj, pd, truth) in enumerate(made):
        n = truth.shape
        st = dict(vol=torch.zeros((2,) + n, device=cuda), xbar=torch.zeros((2,) + n, device=cuda),
                  xprev=torch.zeros((1,) + n, device=cuda), ytv=torch.zeros((1, 3) + n, device=cuda),
                  ytp=torch.zeros((1,) + n, device=cuda), ybc=torch.zeros((1,) + n, device=cuda),
                  flow=torch.zeros((1, 3) + n, device=cuda), proj=proj.unsqueeze(0).contiguous())
        solver = stt.Solver(ctx, st, 1, proj.shape[0], pd, alpha=0.3, bp_mode=bp_mode, roi_cut=cut, seed=100 + k,
                            mode=stt.SOLVE_GRAPH)
        solver.iterate(3)
        torch.cuda.synchronize()
        ref = st["vol"][0].cpu().numpy()
        solver.close()
        assert np.abs(ref).max() > 0
        for mode in results:
            if bp_mode == 0:
                np.testing.assert_array_equal(results[mode][k], ref)
            else:
                assert ob.rel_l2(results[mode][k], ref) < 1e-5
        # and it reconstructs: closer to the truth than the zero start
        assert ob.rel_l2(results[stt.SOLVE_GRAPH][k], truth.cpu().numpy()) < 0.9
