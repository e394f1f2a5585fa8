"""The scatters that add x-neighbour corners with one vector atomic where the
address allows it (scatter_corners; the exact adjoint): accumulators that are
not 16-byte (8-byte) aligned take the scalar atomics.  A two-frame ray-based
solve with an odd voxel count (frame 1's accumulators start 8 bytes off a
16-byte boundary) and an adjoint into a buffer one float off its allocation
give the results of the aligned cases within float-atomic rounding."""
import math

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu


def test_ray_solve_with_odd_voxel_count(cuda):
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    dims, det, F, V = (25, 23, 27), (48, 44), 2, 5  # 15525 voxels: odd
    angles = np.arange(F * V) * (2 * math.pi / (F * V)) + 0.3
    n = dims[::-1]
    outs = {}
    for mode in (stt.SOLVE_PLAIN, stt.SOLVE_GRAPH):
        ctx = stt.Context(0)
        ctx.set_geometry(dims, (1.0, 1.0, 1.0), det, 1.0, 600.0, 1000.0, angles)
        truth = ph.ellipsoid_phantom(dims, 4, seed=3, semi=(2.0, 7.0)).to(cuda)
        proj = torch.zeros((F * V, det[1], det[0]), device=cuda)
        ctx.fp(truth, proj)
        vol = (0.5 * truth).expand(F + 1, *n).contiguous()
        st = dict(vol=vol, xbar=vol.clone(), xprev=torch.zeros((F,) + n, device=cuda),
                  ytv=torch.zeros((F, 3) + n, device=cuda), ytp=torch.zeros((F,) + n, device=cuda),
                  ybc=torch.zeros((F,) + n, device=cuda), flow=torch.zeros((F, 3) + n, device=cuda),
                  proj=proj.view(F, V, det[1], det[0]).contiguous())
        pd = stt.PdParams(tv_w=0.01, tp_w=0.1, bc_w=0.05, huber_factor=0.9, gmax=float(proj.max()) / 4,
                          cut=(2, 2, 2, 3, 2, 2, 3, 3))
        s = stt.Solver(ctx, st, F, V, pd, bp_mode=1, roi_cut=(2, 2, 2, 3, 2, 2, 3, 3), seed=4, mode=mode)
        s.iterate(2)
        torch.cuda.synchronize()
        s.poll_status()
        outs[mode] = st["vol"][:F].cpu().numpy()
        s.close()
        ctx.close()
    assert np.abs(outs[stt.SOLVE_GRAPH]).max() > 0
    assert ob.rel_l2(outs[stt.SOLVE_GRAPH], outs[stt.SOLVE_PLAIN]) < 1e-5


def test_adjoint_into_a_buffer_one_float_off(cuda):
    import torch

    import spacetimetomography_b200 as stt

    scan = ob.Scan((33, 30, 31), (56, 48))
    ctx = stt.Context(0)
    angles = np.arange(4) * (math.pi / 4) + 0.2
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    g = torch.Generator(device=cuda)
    g.manual_seed(6)
    y = torch.rand((4, scan.det[1], scan.det[0]), device=cuda, generator=g)
    nvox = int(np.prod(scan.dims))
    aligned = torch.zeros(nvox, device=cuda)
    backing = torch.zeros(nvox + 1, device=cuda)
    shifted = backing[1:]  # 4 bytes past an aligned allocation
    assert shifted.data_ptr() % 8 == 4
    ctx.fp_vjp(y, aligned.view(scan.dims[::-1]))
    ctx.fp_vjp(y, shifted.view(scan.dims[::-1]))
    torch.cuda.synchronize()
    a, b = aligned.cpu().numpy(), shifted.cpu().numpy()
    assert np.abs(a).max() > 0
    assert ob.rel_l2(b, a) < 1e-6
    ctx.close()
