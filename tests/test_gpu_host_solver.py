"""The solve on host buffers (stt_host_solver_*, include/stt_host.h, through
libstt_facade.so) gives what the device-pointer solver gives from the same
start: each step starts from the submitted volumes with zero duals and the
first view orders, whichever slot it runs on, and steps overlap on two slots
without changing a bit (voxel-driven backprojection)."""
import math

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

F, V, N, DET = 2, 6, 24, (72, 64)
CUT = (3, 3, 3, 5, 3, 3, 6, 5)


def test_host_solver_equals_device_solver(cuda):
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph
    from spacetimetomography_b200.host import HostSolver

    rng = np.random.default_rng(8)
    scan = ob.Scan(N, DET, off=(0.2, 0.1, -0.3))
    angles = rng.uniform(0, 2 * math.pi, F * V)
    params = ph.ellipsoid_params(5, scan.dims, 8, semi=(2.0, 6.0))
    truth = [ph.rasterize(ph.displaced_params(params, f, F, amplitude=1.0, k=2 * math.pi / N), scan.dims).numpy()
             for f in range(F)]
    proj = np.stack([np.stack([ob.fp64(scan, ob.view_angle(angles[f * V + i]), truth[f])[0] for i in range(V)])
                     for f in range(F)]).astype(np.float32)
    vol = np.stack([t * 0.6 for t in truth]).astype(np.float32)
    z, y, x = np.mgrid[0:N, 0:N, 0:N].astype(np.float32)
    flow = np.stack([np.stack([0.5 * np.sin(2 * math.pi * y / N), 0.3 * np.cos(2 * math.pi * x / N),
                               0.4 * np.sin(2 * math.pi * z / N)]) for _ in range(F)]).astype(np.float32)
    pd = stt.PdParams(sigma=0.1125, tau=1.0, tv_w=0.05, tp_w=0.3, bc_w=0.2, huber_factor=0.9,
                      gmax=float(proj[0].max() / 4), cut=CUT)
    iters = 2
    # device-pointer solver from the same start
    ctx = stt.Context(0)
    ctx.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, scan.off)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    full = np.concatenate([vol, vol[-1:]])
    st = dict(vol=T(full), xbar=T(full), xprev=T(np.zeros_like(vol)), ytv=T(np.zeros((F, 3, N, N, N), np.float32)),
              ytp=T(np.zeros_like(vol)), ybc=T(np.zeros_like(vol)), flow=T(flow), proj=T(proj))
    s = stt.Solver(ctx, st, F, V, pd, alpha=0.3, roi_cut=CUT, seed=5)
    s.iterate(iters)
    torch.cuda.synchronize()
    want = st["vol"][:F].cpu().numpy()
    s.close()
    ctx.close()
    # the same on host buffers, three steps on two slots
    hs = HostSolver(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, angles, F, V, pd, alpha=0.3,
                    roi_cut=CUT, seed=5, slots=2, offset=scan.off)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    hv, hf, hp = pin(vol), pin(flow), pin(proj)
    outs = [torch.empty((F, N, N, N)).pin_memory() for _ in range(3)]
    hs.submit(hv, hf, hp, iters, outs[0])
    hs.submit(vol, flow, proj, iters, outs[1])  # pageable numpy arrays work too
    assert hs.pending() == 2
    hs.submit(hv, hf, hp, iters, outs[2])  # slot 0 again: completes the first step first
    assert hs.pending() == 2
    hs.wait()
    hs.wait()
    assert hs.pending() == 0
    hs.close()
    for k, o in enumerate(outs):
        np.testing.assert_array_equal(o.numpy(), want, err_msg=f"step {k}")
