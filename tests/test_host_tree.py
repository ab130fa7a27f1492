"""The product's host tree (C ABI, no device) against the oracle's literal
restatement of pts_tree_build / pts_tree_fix_lr / pts_tree_sort: integer
outputs and box centres must be identical."""
import numpy as np
import pytest

INT_FIELDS = ["laddr", "ilevel", "iparent", "nchild", "ichild", "nnbors", "nbors", "isrc",
              "isrcse", "itarg", "itargse"]


def _inputs():
    rng = np.random.default_rng(11)
    out = []
    for n in (1000, 30000, 120000):
        out.append((f"2d_uniform_{n}", 2, 1e-4, 1e-6, rng.random((n, 2)), rng.random((n // 2, 2))))
        th = rng.random(n) * 2 * np.pi
        r = 0.3 + rng.normal(0, 1e-3, n)
        c = np.c_[0.5 + r * np.cos(th), 0.5 + r * np.sin(th)]
        out.append((f"2d_circle_{n}", 2, 1e-6, 1e-6, c, c))
        out.append((f"3d_uniform_{n}", 3, 1e-3, 1e-6, rng.random((n, 3)), rng.random((n, 3))))
        cen = rng.random((16, 3)) * 0.8 + 0.1
        b = cen[rng.integers(0, 16, n)] + rng.normal(0, 0.02, (n, 3))
        out.append((f"3d_blobs_{n}", 3, 1e-3, 1e-6, b, rng.random((n // 3, 3))))
    # duplicates and points exactly on box boundaries
    g = np.repeat(np.linspace(0, 1, 33), 40)
    pts = np.c_[g, g[::-1]]
    out.append(("2d_boundaries_dups", 2, 1e-5, 1e-6, pts, pts))
    return out


CASES = _inputs()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_host_tree_matches_oracle(case, fgt, oracle):
    name, dim, delta, eps, src, trg = case
    a = oracle.tree(dim, delta, eps, src, trg)
    b = fgt.HostTree(dim, delta, eps, src, trg)
    assert a["nlevels"] == b["nlevels"] and a["nboxes"] == b["nboxes"]
    assert a["npwlevel"] == b["npwlevel"]
    for f in INT_FIELDS:
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["centers"], b["centers"])
    assert np.array_equal(a["boxsize"], b["boxsize"])


def test_host_tree_thread_count_invariance(fgt):
    rng = np.random.default_rng(5)
    src = rng.random((50000, 2))
    a = fgt.HostTree(2, 1e-5, 1e-6, src, src, nthreads=1)
    b = fgt.HostTree(2, 1e-5, 1e-6, src, src, nthreads=4)
    for f in INT_FIELDS:
        assert np.array_equal(a[f], b[f]), f


def test_host_tree_large_delta_has_no_tree(fgt):
    rng = np.random.default_rng(1)
    t = fgt.HostTree(2, 10.0, 1e-6, rng.random((100, 2)), rng.random((10, 2)))
    assert t["npwlevel"] < -2 and "laddr" not in t
