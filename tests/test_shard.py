"""The spatial shard of one transform (fgt2d_b200.shard) on CPU ranks.

The host view of a shard builds the same tree and plan as the GPU path and
filters them for (nranks, rank), so the partition and the exchange lists can
be checked without a GPU:

* the ranks' owned points and tasks add up to the one-rank plan, with every
  box owned by exactly one rank;
* rank r's send list to s is rank s's receive list from r;
* the exchange over torch.distributed (gloo, 2 and 3 ranks) delivers, into
  every rank's copy of the expansion pool, exactly the slots its mp -> loc
  tasks read, bit for bit, and leaves every other slot alone.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

CASES = [(2, 1e-3, 1e-6, 60000, 11), (3, 1e-3, 1e-6, 60000, 12), (3, 1e-2, 1e-6, 20000, 13)]


def _points(dim, n, seed):
    rng = np.random.default_rng(seed)
    return rng.random((n, dim)), rng.random((n // 2, dim))


@pytest.mark.parametrize("dim,delta,eps,n,seed", CASES)
@pytest.mark.parametrize("nranks", [2, 3])
def test_partition_covers_the_plan(fgt, dim, delta, eps, n, seed, nranks):
    from fgt2d_b200.shard import HostShard
    src, trg = _points(dim, n, seed)
    full = HostShard(dim, 1, delta, eps, src, trg, 1, 1, 1, 0).stats()
    assert full["m2l_tasks"] > 0
    tot = {k: 0 for k in full}
    for r in range(nranks):
        s = HostShard(dim, 1, delta, eps, src, trg, 1, 1, nranks, r).stats()
        assert s["owned_sources"] > 0
        for k in s:
            tot[k] += s[k]
    for k in ("owned_sources", "owned_targets", "form_tasks", "eval_tasks", "direct_tasks", "m2l_tasks",
              "shift_tasks"):
        assert tot[k] == full[k], k


@pytest.mark.parametrize("dim,delta,eps,n,seed", CASES)
def test_exchange_lists_are_symmetric(fgt, dim, delta, eps, n, seed):
    from fgt2d_b200.shard import HostShard
    src, trg = _points(dim, n, seed)
    R = 3
    H = [HostShard(dim, 1, delta, eps, src, trg, 1, 1, R, r) for r in range(R)]
    moved = 0
    for r in range(R):
        assert H[r].counts(r) == (0, 0)
        for s in range(R):
            if s != r:
                a, b = H[r].slots(s, "send"), H[s].slots(r, "recv")
                assert np.array_equal(a, b)
                moved += a.size
    assert moved > 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


SLOT = 6  # values per slot in the synthetic pool


def _value(slot):
    return np.arange(SLOT, dtype=np.float64) * 0.25 + np.float64(slot) * np.pi


def _worker(rank, world, port, case, out):
    import torch
    import torch.distributed as dist
    from fgt2d_b200.shard import HostShard, exchange
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dim, delta, eps, n, seed = case
        src, trg = _points(dim, n, seed)
        h = HostShard(dim, 1, delta, eps, src, trg, 1, 1, world, rank)
        nmp = h.stats()["mp_slots"]
        pool = np.full((nmp, SLOT), np.nan)
        own = set()
        for peer in range(world):
            for s in h.slots(peer, "send"):  # this rank's own expansions: the values it computed
                pool[s] = _value(s)
                own.add(int(s))

        def pack(peer, buf):
            sl = h.slots(peer, "send")
            buf.copy_(torch.from_numpy(pool[sl].reshape(-1)))

        def unpack(peer, buf):
            sl = h.slots(peer, "recv")
            pool[sl] = buf.numpy().reshape(len(sl), SLOT)

        exchange(world, rank, h.counts, SLOT, pack, unpack, torch.device("cpu"))
        recv = set()
        ok = True
        for peer in range(world):
            for s in h.slots(peer, "recv"):
                recv.add(int(s))
                ok &= bool(np.array_equal(pool[s], _value(s)))
        untouched = [s for s in range(nmp) if s not in own and s not in recv]
        ok &= bool(np.all(np.isnan(pool[untouched]))) if untouched else True
        out[rank] = (ok, len(recv))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", CASES[:2], ids=["2d", "3d"])
def test_gloo_exchange_delivers_the_halo(fgt, world, case):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, case, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    assert all(res[r][0] for r in range(world)), res
    assert sum(res[r][1] for r in range(world)) > 0
