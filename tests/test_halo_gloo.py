"""Frame-sharded solve: the halo exchange between neighbouring shards, run as
world-size-2 and -3 gloo process groups on CPU (no GPU)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, F, n, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from spacetimetomography_b200.halo import HaloExchange

    def fill(shape, tag):
        return torch.full(shape, float(tag), dtype=torch.float32)

    st = dict(vol=fill((F + 1, n, n, n), 0), xbar=torch.stack([fill((n, n, n), 100 * rank + f) for f in range(F + 1)]),
              ytp=torch.stack([fill((n, n, n), 1000 + 100 * rank + f) for f in range(F)]),
              ybc=torch.stack([fill((n, n, n), 2000 + 100 * rank + f) for f in range(F)]),
              flow=torch.stack([fill((3, n, n, n), 3000 + 100 * rank + f) for f in range(F)]))
    h = HaloExchange(rank, world, st, dist)
    h.exchange_xbar()
    h.exchange_duals()
    res = dict(rank=rank, xbar_last=float(st["xbar"][F].mean()), ytp_halo=float(st["ytp_halo"].mean()),
               ybc_halo=float(st["ybc_halo"].mean()), flow_halo=float(st["flow_halo"].mean()))
    q.put(res)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_gloo(world):
    F, n = 3, 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, F, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r = q.get(timeout=120)
        out[r["rank"]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        o = out[r]
        # X_bar[F] <- X_bar[0] of the next shard; the last shard keeps its own
        assert o["xbar_last"] == (100 * (r + 1) if r + 1 < world else 100 * r + F)
        if r > 0:  # halos <- the previous shard's last frame
            assert o["ytp_halo"] == 1000 + 100 * (r - 1) + F - 1
            assert o["ybc_halo"] == 2000 + 100 * (r - 1) + F - 1
            assert o["flow_halo"] == 3000 + 100 * (r - 1) + F - 1
        else:
            assert o["ytp_halo"] == 0 and o["ybc_halo"] == 0 and o["flow_halo"] == 0
