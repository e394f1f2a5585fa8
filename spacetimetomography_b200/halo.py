"""Frame sharding of the space-time solve across GPUs (one process per GPU).

Rank r owns frames [r*F, (r+1)*F) of the sequence.  One primal-dual iteration
couples neighbouring frames in two places (ST_Tomography.cpp:503-555):

* the dual step of a shard's last frame reads X_bar of the next shard's first
  frame -> before phase 0, rank r receives X_bar[0] of rank r+1 into its
  X_bar[F] slot (the last rank keeps its duplicated last frame there);
* the primal step of a shard's first frame reads Y_tp, Y_bc (after their dual
  step) and the flow of the previous shard's last frame -> between phase 0 and
  phase 1, rank r receives Y_tp[F-1], Y_bc[F-1] of rank r-1 into its halo
  buffers.  Flows change only between primal-dual iterations, so the flow
  halo is exchanged once, at construction.

The exchanges are point-to-point send/recv pairs through torch.distributed
(NCCL over NVLink on GPUs, gloo on CPU in the tests), queued on the caller's
stream so that they order between the solver phases.
"""
from __future__ import annotations

import contextlib


class HaloExchange:
    def __init__(self, rank: int, world: int, st: dict, dist):
        import torch

        self.rank, self.world, self.st, self.dist = rank, world, st, dist
        vol = st["vol"]
        F = st["ytp"].shape[0]
        self.F = F
        shape = tuple(vol.shape[1:])
        st.setdefault("ytp_halo", torch.zeros(shape, dtype=vol.dtype, device=vol.device))
        st.setdefault("ybc_halo", torch.zeros(shape, dtype=vol.dtype, device=vol.device))
        st.setdefault("flow_halo", torch.zeros((3,) + shape, dtype=vol.dtype, device=vol.device))
        self.exchange_flow()

    def _run(self, ops, stream=None):
        if not ops:
            return
        ctx = contextlib.nullcontext()
        if stream is not None:
            import torch

            ctx = torch.cuda.stream(stream)
        with ctx:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()

    def _p2p(self, sends, recvs):
        d = self.dist
        return [d.P2POp(d.isend, t, peer) for t, peer in sends] + [d.P2POp(d.irecv, t, peer) for t, peer in recvs]

    def exchange_flow(self, stream=None):
        """flow[F-1] of rank r-1 -> flow_halo of rank r."""
        st, r, w = self.st, self.rank, self.world
        sends = [(st["flow"][self.F - 1].contiguous(), r + 1)] if r + 1 < w else []
        recvs = [(st["flow_halo"], r - 1)] if r > 0 else []
        self._run(self._p2p(sends, recvs), stream)

    def exchange_xbar(self, stream=None):
        """X_bar[0] of rank r+1 -> X_bar[F] of rank r (before phase 0)."""
        st, r, w = self.st, self.rank, self.world
        sends = [(st["xbar"][0], r - 1)] if r > 0 else []
        recvs = [(st["xbar"][self.F], r + 1)] if r + 1 < w else []
        self._run(self._p2p(sends, recvs), stream)

    def exchange_duals(self, stream=None):
        """Y_tp[F-1], Y_bc[F-1] of rank r-1 -> the halo buffers of rank r (between the phases)."""
        st, r, w = self.st, self.rank, self.world
        sends = ([(st["ytp"][self.F - 1], r + 1), (st["ybc"][self.F - 1], r + 1)] if r + 1 < w else [])
        recvs = [(st["ytp_halo"], r - 1), (st["ybc_halo"], r - 1)] if r > 0 else []
        self._run(self._p2p(sends, recvs), stream)
