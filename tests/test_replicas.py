"""The N > 1 path (independent replicas) with two gloo ranks on CPU."""
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


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from fgt2d_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        secs = 1.0 + rank  # rank 1 is the slow one
        pts = 1000.0 * (rank + 1)
        replicas.barrier()
        out[rank] = (replicas.max_over_ranks(secs), replicas.whole_job_rate(pts, secs),
                     replicas.replica_seed(1236, rank))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0
    assert res[0][1] == res[1][1] == pytest.approx(3000.0 / 2.0)
    assert res[0][2] != res[1][2]


def test_single_process_identity():
    from fgt2d_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.whole_job_rate(10.0, 2.0) == 5.0
