"""Intermediate stages against the oracle: the plane-wave expansions that the
GPU plan holds after an execute (fgt_plan_expansion) against the restated
reference's (orc_fgt_expansions), box by box, in the reference's layout and
node order.

  * multipole expansions of the formed leaves (stage (a): Hermite block ->
    plane wave, or the direct exponential sum) and of the merged parents
    (stage (b), merge), at every level from the cut down;
  * local expansions of the cut-level boxes after mp -> loc (stage (b)).

FP64 plan: the same sums in other orders, so each expansion agrees with the
oracle's to rounding relative to its largest coefficient (<= 1e-12)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _cases():
    rng = np.random.default_rng(31)
    th = rng.random(40000) * 2 * np.pi
    r = 0.3 + rng.normal(0, 1e-3, 40000)
    circle = np.c_[0.5 + r * np.cos(th), 0.5 + r * np.sin(th)]
    blobs = (rng.random((8, 3)) * 0.8 + 0.1)[rng.integers(0, 8, 30000)] + rng.normal(0, 0.03, (30000, 3))
    return [("2d_uniform", 2, 1e-3, 1e-6, rng.random((30000, 2))),
            ("2d_circle", 2, 1e-5, 1e-6, circle),
            ("2d_uniform_e1e-9", 2, 1e-3, 1e-9, rng.random((20000, 2))),
            ("3d_uniform", 3, 1e-2, 1e-6, rng.random((20000, 3))),
            ("3d_blobs", 3, 1e-3, 1e-6, blobs)]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_expansions_match_oracle(fgt, oracle, case):
    name, dim, delta, eps, src = case
    rng = np.random.default_rng(7)
    q = rng.standard_normal((src.shape[0], 1))
    ctx = fgt.Context(0, precision="fp64")
    plan = fgt.Plan(ctx, dim, 1, delta, eps, src, None, 1, 0)
    plan.execute_host(src, q)
    inf = plan.info()
    T = fgt.HostTree(dim, delta, eps, src, src)
    lev, nch = T["ilevel"], T["nchild"]
    cut = inf["npwlevel"]
    nbox = T["nboxes"]
    cand = [b for b in range(nbox) if lev[b] >= max(cut, 0)]
    pick = sorted(rng.choice(cand, size=min(300, len(cand)), replace=False).tolist())
    mp, lo, has = oracle.expansions(dim, 1, delta, eps, src, q, None, 1, 0, pick, inf["nexp"])
    n_mp = n_lo = 0
    worst = 0.0
    for i, b in enumerate(pick):
        if not has[i]:
            continue
        d = plan.expansion("mp", b)
        if d is not None:
            ref = mp[i]
            scale = np.abs(ref).max()
            if scale > 0:
                e = np.abs(d - ref).max() / scale
                worst = max(worst, e)
                assert e <= TOL, (b, "mp", e)
                n_mp += 1
        if lev[b] == cut:
            d = plan.expansion("loc", b)
            if d is not None:
                ref = lo[i]
                scale = np.abs(ref).max()
                if scale > 0:
                    e = np.abs(d - ref).max() / scale
                    worst = max(worst, e)
                    assert e <= TOL, (b, "loc", e)
                    n_lo += 1
    print(f"{name}: {n_mp} multipole and {n_lo} cut-level local expansions, worst {worst:.2e}")
    assert n_mp > 0
    if cut >= 0 and any(lev[b] == cut for b in pick):
        assert n_lo > 0
    plan.close()
