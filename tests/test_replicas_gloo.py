"""Multi-process replica plumbing on CPU (gloo, world_size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from susy_b200.replicas import rank_seed, seconds_per_solve


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from susy_b200.replicas import max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 + 50.0 * rank
        m = max_over_ranks(local_ms)
        dist.barrier()
        q.put((rank, m, rank_seed(11, rank)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [150.0, 150.0]
    assert res[0][2] != res[1][2]
    assert seconds_per_solve(150.0, 3, 2) == pytest.approx(0.025)
