"""Frame sharding on one GPU: a 4-frame space-time solve split into two shards
of two frames each, run phase by phase with the halo exchange of
spacetimetomography_b200.halo between them, equals the unsharded 4-frame solve
bit for bit (voxel-driven backprojection: no atomics anywhere).

The two shards live in one process and take turns; the exchange goes through
an in-process stand-in for the torch.distributed point-to-point calls that
HaloExchange makes (isend/irecv batched by batch_isend_irecv), whose sends
are device-to-device copies into the receiving shard's buffers.  Nothing
waits on another launch, so no kernel of one shard depends on the other's
running at the same time.  Reference: the frame coupling of
ST_Tomography::Render, ST_Tomography.cpp:503-555."""
import math

import numpy as np
import pytest

import oracle_bind as ob

pytestmark = pytest.mark.gpu

F, V, N, DET = 4, 6, 24, (72, 64)
CUT = (3, 3, 3, 5, 3, 3, 6, 5)


class _Mailbox:
    """Messages between the in-process ranks, matched in send order per (src, dst)."""

    def __init__(self):
        self.sent, self.waiting = {}, {}

    def send(self, src, dst, t):
        q = self.waiting.get((src, dst))
        if q:
            q.pop(0).copy_(t)
        else:
            self.sent.setdefault((src, dst), []).append(t.clone())

    def recv(self, src, dst, t):
        q = self.sent.get((src, dst))
        if q:
            t.copy_(q.pop(0))
        else:
            self.waiting.setdefault((src, dst), []).append(t)


class _LocalDist:
    """The part of torch.distributed HaloExchange uses, for one in-process rank."""

    def __init__(self, box, rank):
        self.box, self.rank = box, rank

    @staticmethod
    def P2POp(op, tensor, peer):
        return op, tensor, peer

    def isend(self, tensor, peer):  # only used as an op tag
        raise AssertionError("batched through batch_isend_irecv")

    def irecv(self, tensor, peer):
        raise AssertionError("batched through batch_isend_irecv")

    def batch_isend_irecv(self, ops):
        for op, t, peer in ops:
            if op == self.isend:
                self.box.send(self.rank, peer, t)
        for op, t, peer in ops:
            if op == self.irecv:
                self.box.recv(peer, self.rank, t)
        return []


def _problem(cuda):
    import torch

    from spacetimetomography_b200 import phantom as ph

    rng = np.random.default_rng(3)
    scan = ob.Scan(N, DET, off=(0.3, -0.2, 0.1))
    angles = rng.uniform(0, 2 * math.pi, F * V)
    params = ph.ellipsoid_params(5, scan.dims, 3, semi=(2.0, 6.0))
    truth = [ph.rasterize(ph.displaced_params(params, f, F, amplitude=1.0, k=2 * math.pi / N), scan.dims).numpy()
             for f in range(F)]
    proj = np.stack([np.stack([ob.fp64(scan, ob.view_angle(angles[f * V + i]), truth[f])[0] for i in range(V)])
                     for f in range(F)]).astype(np.float32)
    vol = np.stack([t * 0.7 + 0.05 * rng.random(t.shape) for t in truth]).astype(np.float32)
    z, y, x = np.mgrid[0:N, 0:N, 0:N].astype(np.float32)
    flow = np.stack([np.stack([0.8 * np.sin(2 * math.pi * (y + f) / N), 0.5 * np.cos(2 * math.pi * x / N),
                               0.6 * np.sin(2 * math.pi * z / N)]) for f in range(F)]).astype(np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    return scan, angles, T(vol), T(flow), T(proj), float(proj[0].max() / 4)


def _state(vol, flow, proj, frames, last):
    """Solver state of `frames` frames; `last` fills the X_bar[F] / vol[F] slot."""
    import torch

    full = torch.cat([vol, last[None]]).contiguous()
    shp = vol.shape[1:]
    return dict(vol=full.clone(), xbar=full.clone(), xprev=torch.zeros((frames,) + shp, device=vol.device),
                ytv=torch.zeros((frames, 3) + shp, device=vol.device), ytp=torch.zeros((frames,) + shp, device=vol.device),
                ybc=torch.zeros((frames,) + shp, device=vol.device), flow=flow.contiguous(), proj=proj.contiguous())


@pytest.mark.parametrize("mode", ["graph", "streams"])
def test_sharded_solve_equals_unsharded(cuda, mode):
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200.halo import HaloExchange

    smode = stt.SOLVE_GRAPH if mode == "graph" else stt.SOLVE_STREAMS
    scan, angles, vol, flow, proj, gmax = _problem(cuda)
    pd = stt.PdParams(sigma=0.1125, tau=1.0, tv_w=0.05, tp_w=0.3, bc_w=0.2, huber_factor=0.9, gmax=gmax, cut=CUT)

    def ctx_for(a):
        c = stt.Context(0)
        c.set_geometry(scan.dims, scan.sp, scan.det, scan.ds, scan.sid, scan.sdd, a, scan.off)
        return c

    # unsharded: frames 0..3
    cu = ctx_for(angles)
    su = _state(vol, flow, proj, F, vol[F - 1])
    solver_u = stt.Solver(cu, su, F, V, pd, alpha=0.3, roi_cut=CUT, seed=42, mode=smode)
    # two shards: frames 0..1 and 2..3
    h = F // 2
    box = _Mailbox()
    ca, cb = ctx_for(angles[:h * V]), ctx_for(angles[h * V:])
    sa = _state(vol[:h], flow[:h], proj[:h], h, vol[h])
    sb = _state(vol[h:], flow[h:], proj[h:], h, vol[F - 1])
    xa = HaloExchange(0, 2, sa, _LocalDist(box, 0))
    xb = HaloExchange(1, 2, sb, _LocalDist(box, 1))
    solver_a = stt.Solver(ca, sa, h, V, pd, alpha=0.3, roi_cut=CUT, seed=42, mode=smode, frame_offset=0,
                          total_frames=F)
    solver_b = stt.Solver(cb, sb, h, V, pd, alpha=0.3, roi_cut=CUT, seed=42, mode=smode, halo=True, frame_offset=h,
                          total_frames=F)
    assert torch.equal(sb["flow_halo"], flow[h - 1])
    for _ in range(3):
        solver_u.iterate(1)
        xa.exchange_xbar()
        xb.exchange_xbar()
        solver_a.iterate_phase(0)
        solver_b.iterate_phase(0)
        xa.exchange_duals()
        xb.exchange_duals()
        solver_a.iterate_phase(1)
        solver_b.iterate_phase(1)
    torch.cuda.synchronize()
    for s in (solver_u, solver_a, solver_b):
        s.poll_status()
    for k in ("vol", "xbar", "xprev", "ytv", "ytp", "ybc"):
        got = torch.cat([sa[k][:h], sb[k][:h]])
        assert torch.equal(got, su[k][:F]), (k, float((got - su[k][:F]).abs().max()))
    for s in (solver_u, solver_a, solver_b):
        s.close()
    for c in (cu, ca, cb):
        c.close()


def test_frame_order_follows_the_global_frame():
    """A shard's view orders are those of the frames it holds in the whole sequence."""
    import spacetimetomography_b200 as stt

    for it in range(3):
        for f in range(6):
            a = stt.frame_order(7, it, 6, f, 11)
            assert sorted(a) == list(range(11))
        assert not np.array_equal(stt.frame_order(7, it, 6, 0, 11), stt.frame_order(7, it, 6, 1, 11))
