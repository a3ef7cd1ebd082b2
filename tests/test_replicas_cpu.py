"""Replica aggregation across 2 ranks over gloo (the multi-GPU bench path, on CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from dmrg_b200 import replicas
    secs = [0.5, 2.0][rank]                     # rank 1 is the slow one
    rate = replicas.job_rate(100, secs)
    mx = replicas.max_over_ranks(secs)
    q.put((rank, rate, mx))
    dist.destroy_process_group()


def test_two_rank_job_rate_uses_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, mx in out:
        assert mx == 2.0
        assert rate == pytest.approx(2 * 100 / 2.0)
