"""The multi-rank path of the benchmark on CPU: two gloo ranks, barrier, max-over-ranks time and the
whole-job aggregate (weak scaling: every rank processes its own block, no data exchange)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(ws),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from pmsim_b200 import dist
    ws_, r = dist.init("gloo", timeout_s=60)
    dist.barrier()
    seconds = 0.5 + rank  # rank 1 is the slow one
    rate, tmax = dist.aggregate_rate(1000.0, seconds)
    q.put((r, ws_, rate, tmax))
    dist.finalize()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ws, rate, tmax in out:
        assert ws == 2
        assert tmax == 1.5  # the slowest rank's time
        assert abs(rate - 2 * 1000.0 / 1.5) < 1e-9
