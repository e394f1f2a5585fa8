"""The persistent sweep (STT_SOLVE_PERSISTENT): every frame's SART call, ROI
mask and over-relaxation in one cooperative launch (k_persist.cu) gives the
bits of the batched graph form -- multi-frame solves with FP32 and BF16
storage, the two-phase split of a sharded solve, and a batch of uneven
instances in one launch."""
import numpy as np
import pytest

from test_gpu_extras import INSTANCES, _instance
from test_gpu_solver import F, PD_CUT, ROI_CUT, V, make_problem, run_gpu

pytestmark = pytest.mark.gpu

KEYS = ("vol", "xbar", "xprev", "ytv", "ytp", "ybc")


def test_persistent_solver_equals_graph(cuda):
    """Three frames, six views each at random angles (views along x take the
    transpose phase), two iterations: every state array bit for bit."""
    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = make_problem(3)
    ref, nl_graph, _ = run_gpu(scan, angles, st, gmax, stt.SOLVE_GRAPH, 0, 2, cuda)
    out, nl, it = run_gpu(scan, angles, st, gmax, stt.SOLVE_PERSISTENT, 0, 2, cuda)
    assert it == 2
    # make_perm, per frame a warp + dual and (after the first) a warp + primal, one sweep
    assert 0 < nl <= 1 + 4 * F + 1 < nl_graph, (nl, nl_graph)
    for k in KEYS:
        np.testing.assert_array_equal(out[k], ref[k], err_msg=k)


def _solver(ctx, g, gmax, mode, storage="f32"):
    import spacetimetomography_b200 as stt

    pd = stt.PdParams(sigma=0.1125, tau=1.0, tv_w=0.05, tp_w=0.3, bc_w=0.2, huber_factor=0.9, gmax=gmax, cut=PD_CUT)
    return stt.Solver(ctx, g, F, V, pd, alpha=0.3, bp_mode=0, roi_cut=ROI_CUT, seed=5, mode=mode, storage=storage)


def test_persistent_bf16_storage_and_phase_split(cuda):
    """BF16 storage: the persistent solve equals the graph solve bit for bit;
    run as the two phases of a sharded solve (iterate_phase 0 then 1) it
    equals the whole iteration."""
    import torch

    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = make_problem(4)
    outs = {}
    for name, mode, phased in (("graph", stt.SOLVE_GRAPH, False), ("persistent", stt.SOLVE_PERSISTENT, False),
                               ("phased", stt.SOLVE_PERSISTENT, True)):
        ctx = stt.Context(0)
        ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
        g = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in st.items()}
        for k in ("vol", "xbar", "xprev", "proj"):
            g[k] = g[k].to(torch.bfloat16)
        s = _solver(ctx, g, gmax, mode, storage="bf16")
        if mode == stt.SOLVE_PERSISTENT:
            blocks, _ = s.persistent_info()
            assert blocks >= F
        for _ in range(2):
            if phased:
                s.iterate_phase(0)
                s.iterate_phase(1)
            else:
                s.iterate(1)
        torch.cuda.synchronize()
        s.poll_status()
        outs[name] = {k: g[k].float().cpu().numpy() for k in KEYS}
        s.close()
        ctx.close()
    assert np.abs(outs["graph"]["vol"]).max() > 0
    for name in ("persistent", "phased"):
        for k in KEYS:
            np.testing.assert_array_equal(outs[name][k], outs["graph"][k], err_msg=f"{name}: {k}")


def test_persistent_batch_equals_graph_batch(cuda):
    """Three instances of different volume, detector and view counts: their
    SART calls in one persistent launch give the graph batch's volumes."""
    import torch

    import spacetimetomography_b200 as stt

    made = [_instance(k, cuda) for k in range(len(INSTANCES))]
    cut = (2, 2, 2, 2, 2, 2, 3, 3)
    results = {}
    for mode in (stt.SOLVE_GRAPH, stt.SOLVE_PERSISTENT):
        inst = [dict(ctx=ctx, vol=torch.zeros_like(truth), proj=proj, bp_mode=0, alpha=0.3, pd=pd, roi_cut=cut,
                     seed=200 + k) for k, (ctx, proj, pd, truth) in enumerate(made)]
        b = stt.Batch(inst, mode=mode)
        b.iterate(3)
        torch.cuda.synchronize()
        b.poll_status()
        results[mode] = [d["vol"].cpu().numpy() for d in inst]
        b.close()
    for k in range(len(made)):
        assert np.abs(results[stt.SOLVE_GRAPH][k]).max() > 0
        np.testing.assert_array_equal(results[stt.SOLVE_PERSISTENT][k], results[stt.SOLVE_GRAPH][k],
                                      err_msg=f"instance {k}")


def test_persistent_mode_refuses_ray_backprojection(cuda):
    import torch

    import spacetimetomography_b200 as stt

    scan, angles, st, gmax = make_problem(5)
    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    g = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in st.items()}
    pd = stt.PdParams(gmax=gmax, cut=PD_CUT)
    with pytest.raises(stt.STTError):
        stt.Solver(ctx, g, F, V, pd, bp_mode=1, roi_cut=ROI_CUT, mode=stt.SOLVE_PERSISTENT)
    ctx.close()


def test_persistent_larger_frames_equal_graph(cuda):
    """Two frames of 160 x 160 x 164 voxels (4 views each, 128 x 112
    detector; every block runs thousands of tiles per phase): the same bits
    as the graph solve."""
    import math

    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    dims, det, Fr, Vr = (160, 160, 164), (128, 112), 2, 4
    angles = np.arange(Fr * Vr) * (2 * math.pi / (Fr * Vr)) + 0.2
    outs = {}
    for mode in (stt.SOLVE_GRAPH, stt.SOLVE_PERSISTENT):
        ctx = stt.Context(0)
        ctx.set_geometry(dims, (1.0, 1.0, 1.0), det, 1.6, 600.0, 1000.0, angles)
        n = dims[::-1]
        truth = ph.ellipsoid_phantom(dims, 8, seed=7, semi=(8.0, 40.0)).to(cuda)
        proj = torch.zeros((Fr * Vr, det[1], det[0]), device=cuda)
        ctx.fp(truth, proj)
        vol = (0.5 * truth).expand(Fr + 1, *n).contiguous()
        st = dict(vol=vol, xbar=vol.clone(), xprev=torch.zeros((Fr,) + n, device=cuda),
                  ytv=torch.zeros((Fr, 3) + n, device=cuda), ytp=torch.zeros((Fr,) + n, device=cuda),
                  ybc=torch.zeros((Fr,) + n, device=cuda), flow=torch.zeros((Fr, 3) + n, device=cuda),
                  proj=proj.view(Fr, Vr, det[1], det[0]).contiguous())
        pd = stt.PdParams(tv_w=0.01, tp_w=0.1, bc_w=0.05, huber_factor=0.9, gmax=float(proj.max()) / 4,
                          cut=(4, 4, 4, 8, 4, 4, 8, 6))
        s = stt.Solver(ctx, st, Fr, Vr, pd, alpha=0.3, roi_cut=(4, 4, 4, 8, 4, 4, 8, 6), seed=3, mode=mode)
        s.iterate(2)
        torch.cuda.synchronize()
        s.poll_status()
        outs[mode] = {k: st[k].cpu().numpy() for k in KEYS}
        s.close()
        ctx.close()
    assert np.abs(outs[stt.SOLVE_GRAPH]["vol"]).max() > 0
    for k in KEYS:
        np.testing.assert_array_equal(outs[stt.SOLVE_PERSISTENT][k], outs[stt.SOLVE_GRAPH][k], err_msg=k)
