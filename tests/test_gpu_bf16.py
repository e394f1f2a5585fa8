"""BF16 storage of the solver's primal volumes and sinogram
(stt_solve_cfg.storage = STT_DTYPE_BF16) through the C ABI: the three
execution modes agree; one iteration equals the oracle's FP32 restatement with
every primal store rounded to BF16 (oracle_bind.pd_iteration_bf16); the error
against the FP64 oracle is stated; a batch of BF16 instances equals each
instance's own BF16 solve."""
import numpy as np
import pytest

import oracle_bind as ob
from test_gpu_solver import DET, F, N, PD_CUT, ROI_CUT, V, make_problem

pytestmark = pytest.mark.gpu

PRIMAL = ("vol", "xbar", "xprev", "proj")


def bf16_problem(seed):
    scan, angles, st, gmax = make_problem(seed)
    st = dict(st)
    for k in PRIMAL:
        st[k] = ob.bf16_round(st[k])
    return scan, angles, st, gmax


def run_bf16(scan, angles, st, gmax, mode, bp_mode, iters, cuda, seed=42, fp16=None):
    import torch

    import spacetimetomography_b200 as stt

    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    if fp16 is not None:
        ctx.set_tuning(0, 0, 0, staged_bins=0x1E0, fp_variant_bf16=fp16)
    g = {}
    for k, v in st.items():
        t = torch.from_numpy(np.ascontiguousarray(v)).to(cuda)
        g[k] = t.to(torch.bfloat16) if k in PRIMAL else t  # exact: the values are BF16 already
    pd = stt.PdParams(sigma=0.1125, tau=1.0, tv_w=0.05, tp_w=0.3, bc_w=0.2, huber_factor=0.9, gmax=gmax, cut=PD_CUT)
    if fp16:
        # frame f starts f * N^3 * 2 bytes on, a multiple of the texture alignment here
        assert ctx.fp_texture_ok(g["vol"]) and (N ** 3 * 2) % 512 == 0
    s = stt.Solver(ctx, g, F, V, pd, alpha=0.3, bp_mode=bp_mode, roi_cut=ROI_CUT, seed=seed, mode=mode,
                   storage="bf16")
    s.iterate(iters)
    torch.cuda.synchronize()
    s.poll_status()
    out = {k: v.float().cpu().numpy() for k, v in g.items()}
    s.close()
    ctx.close()
    return out


def test_bf16_storage_rejects_wrong_dtypes(cuda):
    import torch

    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = bf16_problem(0)
    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    g = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in st.items()}  # all float32
    with pytest.raises(ValueError):
        stt.Solver(ctx, g, F, V, stt.PdParams(gmax=gmax), storage="bf16")
    ctx.close()


@pytest.mark.parametrize("bp_mode", [0, 1])
def test_bf16_modes_agree(cuda, bp_mode):
    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = bf16_problem(1)
    res = {m: run_bf16(scan, angles, st, gmax, m, bp_mode, 2, cuda) for m in
           (stt.SOLVE_PLAIN, stt.SOLVE_STREAMS, stt.SOLVE_GRAPH)}
    base = res[stt.SOLVE_PLAIN]
    for m in (stt.SOLVE_STREAMS, stt.SOLVE_GRAPH):
        for k in ("vol", "xbar", "xprev", "ytv", "ytp", "ybc"):
            if bp_mode == 0:  # gathers only: the same bits in every mode
                np.testing.assert_array_equal(res[m][k], base[k], err_msg=k)
            else:  # float atomics: a sum order can flip a BF16 rounding
                assert ob.rel_l2(res[m][k], base[k]) < 5e-3, k


def test_bf16_texture_gathers_leave_the_solve_unchanged(cuda):
    """The BF16 solve with the gather projector's tld4 form (16-bit textures,
    fp_variant_bf16 1) gives the bits of its load form, in the graph mode."""
    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = bf16_problem(5)
    a = run_bf16(scan, angles, st, gmax, stt.SOLVE_GRAPH, 0, 2, cuda, fp16=0)
    b = run_bf16(scan, angles, st, gmax, stt.SOLVE_GRAPH, 0, 2, cuda, fp16=1)
    for k in ("vol", "xbar", "xprev", "ytv", "ytp", "ybc"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert np.abs(a["vol"]).max() > 0


@pytest.mark.parametrize("bp_mode", [0, 1])
def test_bf16_iteration_matches_rounded_restatement(cuda, bp_mode):
    """One iteration against the FP32 restatement that rounds every primal
    store to BF16.  Voxel BP: a rare FP32 difference between kernel and
    restatement (1e-7 relative, from the projector's summation) can move a
    value across a BF16 rounding boundary; those isolated flips (2^-8
    relative each) keep the volumes within 1e-3.  Ray BP adds float-atomic
    order to that."""
    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = bf16_problem(2)
    out = run_bf16(scan, angles, st, gmax, stt.SOLVE_GRAPH, bp_mode, 1, cuda, seed=9)
    pp = [0.1125, 1.0, 0.05, 0.3, 0.2, 0.9, gmax]
    raylen = [np.zeros((DET[1], DET[0]), np.float32) for _ in range(F)]
    orders = [stt.frame_order(9, 0, F, f, V) for f in range(F)]
    ref = ob.pd_iteration_bf16(scan, angles, st, F, V, pp, PD_CUT, ROI_CUT, 0.3, bp_mode, orders, raylen)
    tol = 1e-3 if bp_mode == 0 else 3e-3
    for k in ("vol", "xbar", "xprev", "ytv", "ytp", "ybc"):
        e = ob.rel_l2(out[k][:F], ref[k][:F])
        assert e < tol, (k, e)
    # every stored primal value is a BF16 value
    for k in ("vol", "xbar", "xprev"):
        np.testing.assert_array_equal(ob.bf16_round(out[k]), out[k])


def test_bf16_iteration_error_vs_fp64(cuda):
    """The BF16-storage solve against the FP64 oracle run from the same
    (BF16-valued) start: the volumes carry the BF16 rounding of every stored
    update, 2^-9 relative each, so they are held to 1e-2 (FP32 storage: 1e-4,
    test_gpu_solver)."""
    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = bf16_problem(3)
    out = run_bf16(scan, angles, st, gmax, stt.SOLVE_GRAPH, 0, 1, cuda, seed=5)
    pp = [0.1125, 1.0, 0.05, 0.3, 0.2, 0.9, gmax]
    raylen = [np.zeros((DET[1], DET[0]), np.float64) for _ in range(F)]
    orders = [stt.frame_order(5, 0, F, f, V) for f in range(F)]
    ref = ob.pd_iteration(scan, angles, st, F, V, pp, PD_CUT, ROI_CUT, 0.3, 0, orders, raylen, fp64=True)
    for k in ("vol", "xbar", "xprev"):
        e = ob.rel_l2(out[k][:F], ref[k][:F])
        assert e < 1e-2, (k, e)


def test_bf16_batch_equals_own_solves(cuda):
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    dims = [(32, 28, 24), (24, 24, 24)]
    dets = [(48, 40), (40, 36)]
    nviews = [10, 7]
    inst, ref = [], []
    for k, (d, det, nv) in enumerate(zip(dims, dets, nviews)):
        scan = ob.Scan(d, det)
        angles = np.linspace(0, 2 * np.pi, nv, endpoint=False)
        truth = ph.ellipsoid_phantom(d, 4, seed=k, semi=(2.0, 6.0)).numpy()
        proj = np.stack([ob.fp64(scan, ob.view_angle(a), truth)[0] for a in angles]).astype(np.float32)
        gmax = float(proj.max() / 4)
        cut = (2, 2, 2, 2, 2, 2, 3, 3)  # (the reference's cut would mask out these small volumes)
        pd = stt.PdParams(sigma=0.1125, tau=1.0, tv_w=0.05, huber_factor=0.9, gmax=gmax, cut=cut)
        for run in range(2):
            ctx = stt.Context(0)
            ctx.set_geometry(d, (1.0, 1.0, 1.0), det, 1.0, 600.0, 1000.0, angles)
            vol = torch.zeros(d[::-1], device=cuda, dtype=torch.bfloat16)
            p = torch.from_numpy(ob.bf16_round(proj)).to(cuda).to(torch.bfloat16)
            rec = dict(ctx=ctx, vol=vol, proj=p, pd=pd, roi_cut=cut, seed=3 + k, storage="bf16")
            (inst if run == 0 else ref).append(rec)
    b = stt.Batch(inst, mode=stt.SOLVE_GRAPH)
    b.iterate(2)
    torch.cuda.synchronize()
    b.close()
    for r in ref:  # each instance alone, one BF16 batch of one
        one = stt.Batch([r], mode=stt.SOLVE_STREAMS)
        one.iterate(2)
        torch.cuda.synchronize()
        one.close()
    for a, r in zip(inst, ref):
        np.testing.assert_array_equal(a["vol"].float().cpu().numpy(), r["vol"].float().cpu().numpy())
        assert float(a["vol"].float().abs().sum()) > 0
    for r in inst + ref:
        r["ctx"].close()


def _bf16(t):
    import torch

    return t.to(torch.bfloat16)


# (40, 36, 44): nz is not a multiple of 8, so the BF16 sweep gathers every
# view; (48, 40, 56): the BF16 slab maps apply and the oblique views go
# through the slab-staged kernel's BF16 boxes
@pytest.mark.parametrize("fp16", [0, 1])
@pytest.mark.parametrize("dims", [(40, 36, 44), (48, 40, 56)])
@pytest.mark.parametrize("bp_mode", [0, 1])
def test_bf16_sart_sweep_equals_rounded_fp32_views(cuda, bp_mode, dims, fp16):
    """stt_sart_sweep_typed(BF16) against the FP32 sweep run one view at a time
    on the widened volume, rounded to BF16 after each view: the same bits with
    voxel BP (the BF16 gather projector, by loads or by tld4 gathers of 16-bit
    textures (fp16), and the slab projector add what the FP32 ones do), within
    a few rounding flips with ray BP (float atomics)."""
    import torch

    import spacetimetomography_b200 as stt

    scan = ob.Scan(dims, (64, 56), off=(0.4, -0.3, 0.2))
    V = 9
    angles = np.linspace(0, 2 * np.pi, V, endpoint=False) + 0.2
    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    from spacetimetomography_b200 import phantom as ph

    truth = ph.ellipsoid_phantom(scan.dims, 5, seed=4, semi=(3.0, 10.0)).to(cuda)
    proj = torch.zeros((V,) + scan.det[::-1], device=cuda)
    ctx.fp(truth, proj)
    proj16 = _bf16(proj)
    start = _bf16(truth * 0.7)
    perm = stt.permutation(3, V)
    gmax = float(proj.max()) / 4
    a = start.clone()
    ctx.set_tuning(0, 0, 0, staged_bins=0x1E0, fp_variant_bf16=fp16)
    if fp16:
        assert ctx.fp_texture_ok(a)  # the texture form really runs
    rl = torch.zeros(scan.det[::-1], device=cuda)
    ctx.sart_sweep(a, proj16, perm, 0.3, gmax, bp_mode, rl)
    b = start.float()
    rl2 = torch.zeros(scan.det[::-1], device=cuda)
    pf = proj16.float()
    for k in perm:
        ctx.sart_sweep(b, pf, [int(k)], 0.3, gmax, bp_mode, rl2)
        b = b.to(torch.bfloat16).float()
    torch.cuda.synchronize()
    if bp_mode == 0:
        np.testing.assert_array_equal(a.float().cpu().numpy(), b.cpu().numpy())
    else:
        assert ob.rel_l2(a.float().cpu().numpy(), b.cpu().numpy()) < 3e-3
    ctx.close()


def test_bf16_voxel_bp_and_warp_entry_points(cuda):
    """stt_bp_voxel_typed(BF16) equals the FP32 backprojection of the widened
    volume rounded to BF16; stt_warp_typed(BF16) equals the FP32 warp of the
    widened source (within an ulp: two compiled instantiations of the sampler
    may contract differently); stt_bp_ray_typed(BF16) is within BF16 rounding
    flips of the rounded FP32 form."""
    import torch

    import spacetimetomography_b200 as stt

    scan = ob.Scan((48, 40, 36), (72, 64))
    angles = np.array([0.3, 1.9])
    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    g = torch.Generator(device=cuda)
    g.manual_seed(2)
    vol16 = _bf16(torch.rand(scan.dims[::-1], device=cuda, generator=g))
    corr = torch.randn(scan.det[::-1], device=cuda, generator=g)
    a = vol16.clone()
    ctx.bp_voxel(corr, a, 0.3, 5.0, 1)
    b = vol16.float()
    ctx.bp_voxel(corr, b, 0.3, 5.0, 1)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.float().cpu().numpy(), _bf16(b).float().cpu().numpy())
    a = vol16.clone()
    ctx.bp_ray(corr, a, 5.0, 0)
    b = vol16.float()
    ctx.bp_ray(corr, b, 5.0, 0)
    torch.cuda.synchronize()
    assert ob.rel_l2(a.float().cpu().numpy(), _bf16(b).float().cpu().numpy()) < 1e-3
    nz, ny, nx = scan.dims[::-1]
    flow = torch.randn((3, nz, ny, nx), device=cuda, generator=g) * 0.7
    w16 = stt.warp(flow, vol16, -1.0)
    w32 = stt.warp(flow, vol16.float(), -1.0)
    torch.cuda.synchronize()
    assert w16.dtype == torch.float32
    assert ob.rel_l2(w16.cpu().numpy(), w32.cpu().numpy()) < 1e-6
    ctx.close()
