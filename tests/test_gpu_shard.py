"""The spatial shard on the GPU, its ranks run one after the other on one
device (one GPU is available to the tests; no kernel of one rank waits on
another's, so running them in turn is the same computation).

Every rank's shard plan runs phase 1 (formation and merge of its boxes);
the cut-level expansions each rank sends are packed into device buffers and
unpacked into the receiving rank's pool; every rank runs phase 2.  The sum
of the ranks' outputs must equal the unsharded plan's bit for bit, in both
precision forms: an owned point is computed by the same tasks in the same
order, and the other ranks contribute exact zeros.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(2, 1e-3, 1e-6, 60000, 21), (3, 1e-3, 1e-6, 60000, 22), (2, 1e-6, 1e-6, 40000, 23),
         (3, 1e-2, 1e-9, 20000, 24)]


@pytest.mark.parametrize("dim,delta,eps,n,seed", CASES)
@pytest.mark.parametrize("nranks", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_shard_sum_equals_one_gpu(fgt, dim, delta, eps, n, seed, nranks, precision):
    import torch
    from fgt2d_b200.shard import ShardPlan
    if precision == "mixed" and eps < 1e-6:
        pytest.skip("the mixed form applies at eps >= 1e-6")
    rng = np.random.default_rng(seed)
    src, trg = rng.random((n, dim)), rng.random((n // 2, dim))
    q = rng.standard_normal(n)
    dev = torch.device("cuda", 0)
    ctx = fgt.Context(0, precision=precision)
    d_q = torch.from_numpy(q.reshape(-1, 1)).to(dev)
    d_src = torch.from_numpy(src).to(dev)
    d_trg = torch.from_numpy(trg).to(dev)
    one = fgt.Plan(ctx, dim, 1, delta, eps, src, trg, 1, 1)
    ref_pot = torch.zeros((n, 1), dtype=torch.float64, device=dev)
    ref_pt = torch.zeros((n // 2, 1), dtype=torch.float64, device=dev)
    one.execute_device(d_src.data_ptr(), d_q.data_ptr(), d_trg.data_ptr(), ref_pot.data_ptr(), ref_pt.data_ptr())
    plans = [ShardPlan(ctx, dim, 1, delta, eps, src, trg, 1, 1, nranks, r) for r in range(nranks)]
    pots = [torch.full((n, 1), np.nan, dtype=torch.float64, device=dev) for _ in plans]
    pts = [torch.full((n // 2, 1), np.nan, dtype=torch.float64, device=dev) for _ in plans]
    owned = [p.owned() for p in plans]
    assert sum(o[0] for o in owned) == n and sum(o[1] for o in owned) == n // 2
    for r, p in enumerate(plans):
        p.phase(1, d_q.data_ptr(), pots[r].data_ptr(), pts[r].data_ptr())
    torch.cuda.synchronize()
    slot = plans[0].slot_doubles()
    moved = 0
    for r, p in enumerate(plans):
        for s in range(nranks):
            if s == r:
                continue
            ns_, _ = p.counts(s)
            assert plans[s].counts(r)[1] == ns_
            if ns_ == 0:
                continue
            buf = torch.empty(ns_ * slot, dtype=torch.float64, device=dev)
            p.pack(s, buf.data_ptr())
            torch.cuda.synchronize()
            plans[s].unpack(r, buf.data_ptr())
            torch.cuda.synchronize()
            moved += ns_
    for r, p in enumerate(plans):
        p.phase(2, d_q.data_ptr(), pots[r].data_ptr(), pts[r].data_ptr())
    torch.cuda.synchronize()
    tot_pot = sum(pots[1:], pots[0].clone())
    tot_pt = sum(pts[1:], pts[0].clone())
    print(f"{dim}D delta={delta} R={nranks} {precision}: moved {moved} expansions, owned {owned}")
    assert torch.equal(tot_pot, ref_pot)
    assert torch.equal(tot_pt, ref_pt)
    for p in plans:
        p.close()
    one.close()
