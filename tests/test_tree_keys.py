"""The exact-key form of the device tree build (fgt_devtree.cu), restated in
numpy on the CPU and checked against the host tree (itself pinned to the
oracle's restatement of pts_tree_build / pts_tree_fix_lr / pts_tree_sort).

Steps restated: every source descends from the root for nlmax levels with
the tree's centre arithmetic, its child digits packed most significant level
first (k_exact_key); one sort of the keys; the range of every box of the
finished tree from its parent's range by the digit of its level
(k_child_bounds); the final order restores the input order inside each leaf
(k_position_rank + the stable sort).  Every box range and the source
permutation must equal the host tree's, including on grids whose points lie
exactly on box boundaries and centres."""
import numpy as np
import pytest


def _keys(x, dim, cen0, bs0, L):
    n = x.shape[0]
    c = np.tile(np.asarray(cen0[:dim], dtype=np.float64), (n, 1))
    k = np.zeros(n, dtype=np.uint64)
    bs = bs0
    for _ in range(L):
        j = np.zeros(n, dtype=np.uint64)
        for d in range(dim):
            j |= (~((x[:, d] - c[:, d]) < 0)).astype(np.uint64) << np.uint64(d)
        k = (k << np.uint64(dim)) | j
        bs = bs / 2
        h = bs / 2
        for d in range(dim):
            c[:, d] = c[:, d] + np.where(((j >> np.uint64(d)) & np.uint64(1)) == 1, h, -h)
    return k


def _cases():
    rng = np.random.default_rng(5)
    out = []
    n = 20000
    out.append(("2d_uniform", 2, 1e-4, 1e-6, rng.random((n, 2))))
    th = rng.random(n) * 2 * np.pi
    r = 0.3 + rng.normal(0, 1e-3, n)
    out.append(("2d_circle", 2, 1e-6, 1e-6, np.c_[0.5 + r * np.cos(th), 0.5 + r * np.sin(th)]))
    out.append(("3d_uniform", 3, 1e-3, 1e-6, rng.random((n, 3))))
    cen = rng.random((8, 3)) * 0.8 + 0.1
    out.append(("3d_blobs", 3, 1e-3, 1e-6, cen[rng.integers(0, 8, n)] + rng.normal(0, 0.02, (n, 3))))
    g = np.array(np.meshgrid(np.linspace(0, 1, 129), np.linspace(0, 1, 129))).reshape(2, -1).T.copy()
    out.append(("2d_grid_exact", 2, 1e-6, 1e-6, g))
    g3 = np.array(np.meshgrid(*[np.linspace(0, 1, 25)] * 3)).reshape(3, -1).T.copy()
    out.append(("3d_grid_exact", 3, 1e-4, 1e-6, g3))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_exact_key_tree_equals_host_tree(fgt, case):
    name, dim, delta, eps, src = case
    T = fgt.HostTree(dim, delta, eps, src, src)
    assert "laddr" in T
    nb, nlev, L = T["nboxes"], T["nlevels"], T["nlmax"]
    assert nlev <= L <= (31 if dim == 2 else 21)
    cen = T["centers"].reshape(-1, dim)
    key = _keys(src, dim, cen[0], T["boxsize"][0], L)
    order = np.argsort(key, kind="stable")
    sk = key[order]
    nch = 1 << dim
    laddr = T["laddr"].reshape(-1, 2) - 1
    ichild = T["ichild"].reshape(-1, nch) - 1
    r0 = np.zeros(nb, np.int64)
    r1 = np.zeros(nb, np.int64)
    r1[0] = src.shape[0]
    for l in range(nlev):
        shift = np.uint64(dim * (L - 1 - l))
        for b in range(laddr[l, 0], laddr[l, 1] + 1):
            if ichild[b, 0] < 0:
                continue
            dg = ((sk[r0[b]:r1[b]] >> shift) & np.uint64(nch - 1)).astype(np.int64)
            assert np.all(np.diff(dg) >= 0)
            for j in range(nch):
                c = ichild[b, j]
                r0[c] = r0[b] + np.searchsorted(dg, j, "left")
                r1[c] = r0[b] + np.searchsorted(dg, j + 1, "left") if j < nch - 1 else r1[b]
    se = T["isrcse"].reshape(-1, 2)
    assert np.array_equal(se[:, 0] - 1, r0)
    assert np.array_equal(se[:, 1], r1)
    perm = order.copy()
    for b in np.where(ichild[:, 0] < 0)[0]:
        perm[r0[b]:r1[b]] = np.sort(perm[r0[b]:r1[b]])
    assert np.array_equal(perm, T["isrc"] - 1)


def _warp_digit_lower_bound(dig, a, b, v):
    """warp_digit_lower_bound (fgt_devtree.cu) lane by lane: each round the 32
    lanes probe a + floor(span * lane / 32), a ballot counts the probes whose
    digit is below v (a prefix of the lanes, the digits being sorted), and the
    range narrows to the gap after the last of them; <= 32 keys are probed
    one per lane."""
    for _ in range(8):
        if b - a <= 32:
            break
        span = b - a
        p = [a + span * lane // 32 for lane in range(32)]
        below = [dig[q] < v for q in p]
        c = sum(below)
        assert below == [True] * c + [False] * (32 - c)
        if c == 0:
            return a
        a, b = p[c - 1] + 1, (p[c] if c < 32 else b)
    assert b - a <= 32
    return a + sum(1 for lane in range(32) if a + lane < b and dig[a + lane] < v)


def test_warp_digit_search_matches_lower_bound():
    rng = np.random.default_rng(17)
    for n in [1, 2, 31, 32, 33, 64, 65, 1000, 4097, 100_000]:
        for nch in (4, 8):
            for _ in range(3):
                dig = np.sort(rng.integers(0, nch, n))
                if rng.random() < 0.3:  # runs of one digit, empty digits
                    dig = np.sort(rng.choice([0, nch - 1], n))
                for v in range(1, nch):
                    assert _warp_digit_lower_bound(dig, 0, n, v) == np.searchsorted(dig, v, "left")
