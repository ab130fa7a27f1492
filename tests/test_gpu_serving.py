"""The transform server: requests of mixed dimension, size, delta and eps run
concurrently on worker streams, and every result equals the same request run
alone (same kernels, same plan, deterministic reductions: bitwise)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        dim = int(rng.integers(2, 4))
        n = int(10 ** rng.uniform(3, 4.7))
        delta = float(10 ** rng.uniform(-5 if dim == 2 else -3, -1))
        if k % 7 == 3:
            delta = 5.0  # large-delta path
        eps = float(rng.choice([1e-3, 1e-6, 1e-9]))
        src = rng.random((n, dim))
        q = rng.random(n)
        if k % 3 == 0:
            out.append((dim, delta, eps, src, q, src, 1, 0))
        else:
            trg = rng.random((n // 2 + 1, dim))
            out.append((dim, delta, eps, src, q, trg, 1, 1))
    return out


def test_mix_equals_alone(fgt):
    reqs = _requests(5, 24)
    ctx = fgt.Context(0, precision="auto")
    alone = [fgt.transform(d, 1, de, ep, s, q, t, a, b, ctx=ctx) for d, de, ep, s, q, t, a, b in reqs]
    srv = fgt.Server(0, workers=4, precision="auto")
    ids = [srv.submit(d, 1, de, ep, s, q, t, a, b) for d, de, ep, s, q, t, a, b in reqs]
    for (pa, ta), rid in zip(alone, ids):
        pm, tm, lat = srv.wait(rid)
        assert lat > 0
        assert np.array_equal(pa, pm)
        if ta is not None:
            assert np.array_equal(ta, tm)
    st = srv.stats()
    assert st["completed"] == st["submitted"] == len(reqs) and st["failed"] == 0
    assert 0 < st["p50_s"] <= st["p99_s"] <= st["max_s"]
    # every request of this mix has <= 1e5 points: each ran on a worker's
    # highest-priority stream (B200 exposes stream priorities)
    assert st["hi_priority"] == len(reqs), st["hi_priority"]
    srv.close()


def test_admission_under_a_small_budget(fgt):
    reqs = _requests(9, 12)
    srv = fgt.Server(0, max_bytes=96 << 20, workers=6)
    ids = [srv.submit(d, 1, de, ep, s, q, t, a, b) for d, de, ep, s, q, t, a, b in reqs]
    for rid in ids:
        srv.wait(rid)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["budget_bytes"] == 96 << 20
    srv.close()


def test_failed_request_does_not_stop_the_others(fgt):
    rng = np.random.default_rng(2)
    srv = fgt.Server(0, workers=2)
    good = srv.submit(2, 1, 1e-3, 1e-6, rng.random((3000, 2)), rng.random(3000))
    bad = srv.submit(2, 1, 1e-3, 2.0, rng.random((3000, 2)), rng.random(3000))  # eps >= 1
    nan = rng.random((3000, 2))
    nan[5, 0] = np.nan
    bad2 = srv.submit(2, 1, 1e-3, 1e-6, nan, rng.random(3000))
    pot, _, _ = srv.wait(good)
    assert np.all(np.isfinite(pot))
    for rid in (bad, bad2):
        with pytest.raises(fgt.FGTError) as e:
            srv.wait(rid)
        assert e.value.status == 1
    assert srv.stats()["failed"] == 2
    srv.close()


def test_gradient_requests_mixed_in(fgt):
    """Requests with gradients and Hessians among plain ones: each equals the
    same request run alone, bitwise."""
    rng = np.random.default_rng(13)
    reqs = []
    for k in range(10):
        dim = 2 + k % 2
        n = int(10 ** rng.uniform(3, 4.3))
        src, trg, q = rng.random((n, dim)), rng.random((n // 2 + 1, dim)), rng.random(n)
        reqs.append((dim, 1e-3 if dim == 3 else 1e-4, 1e-6, src, q, trg, k % 4, (k + 1) % 4))
    ctx = fgt.Context(0, precision="auto")
    alone = [fgt.transform_pgh(d, 1, de, ep, s, q, t, a, b, ctx=ctx) for d, de, ep, s, q, t, a, b in reqs]
    srv = fgt.Server(0, workers=3, precision="auto")
    ids = [srv.submit(d, 1, de, ep, s, q, t, a, b) for d, de, ep, s, q, t, a, b in reqs]
    for ref, rid in zip(alone, ids):
        got, lat = srv.wait_pgh(rid)
        for k, v in ref.items():
            if v is None:
                assert got[k] is None
            else:
                assert np.array_equal(v, got[k]), k
    assert srv.stats()["failed"] == 0
    srv.close()


def test_dipole_requests(fgt):
    """Dipole requests (with and without charges) through the server equal
    the same transforms run alone, bitwise."""
    rng = np.random.default_rng(29)
    ctx = fgt.Context(0, precision="auto")
    srv = fgt.Server(0, workers=2, precision="auto")
    reqs, ids = [], []
    for k in range(6):
        dim = 2 + k % 2
        n = int(10 ** rng.uniform(3, 4))
        src, trg = rng.random((n, dim)), rng.random((n // 3 + 1, dim))
        q = rng.random(n) if k % 3 else None
        rn, ds = rng.normal(size=(n, dim)), rng.random(n)
        delta = 1e-3 if dim == 3 else 1e-4
        reqs.append(fgt.transform_pgh(dim, 1, delta, 1e-6, src, q, trg, 1 + k % 3, 1, ctx=ctx,
                                      ifcharge=int(q is not None), ifdipole=1, rnormal=rn, dipstr=ds))
        ids.append(srv.submit(dim, 1, delta, 1e-6, src, q, trg, 1 + k % 3, 1, rnormal=rn, dipstr=ds))
    for ref, rid in zip(reqs, ids):
        got, _ = srv.wait_pgh(rid)
        for key, v in ref.items():
            if v is not None:
                assert np.array_equal(v, got[key]), key
    srv.close()
