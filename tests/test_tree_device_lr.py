"""The device form of the tree build's refinement, colleagues and level
restriction (fgt_devtree.cu: k_ref_*, k_lr_*), restated in Python on the CPU
and checked against the host tree (itself pinned to the oracle's restatement
of pts_tree_build / pts_tree_fix_lr).

What is restated is the order of the device steps: boxes keep creation ids
(original boxes, the first restriction pass's, the second pass's), every
level is the concatenation of at most three id ranges, flags and
refinements follow the host build's passes, and one renumbering and one
colleague pass finish the tree.  Every integer field, the centres and the
colleague lists must equal the host tree's, on inputs whose level
restriction adds boxes in both passes."""
import numpy as np
import pytest

from test_tree_keys import _keys

F105 = float(np.float32(1.05))


def _device_tree(src, dim, T):
    ndiv0, ndiv = (10, 80) if dim == 2 else (40, 100)
    levcut, L, nch = T["npwlevel"], T["nlmax"], 1 << dim
    cen0 = T["centers"].reshape(-1, dim)[0].copy()
    bs0 = T["boxsize"][0]
    key = np.sort(_keys(src, dim, cen0, bs0, L))
    bsz = [bs0]
    for _ in range(L + 3):
        bsz.append(bsz[-1] / 2)
    level, par, nchild, child, cen = [0], [-1], [0], [[-1] * nch], [cen0.copy()]
    r0, r1, lfirst, llast = [0], [src.shape[0]], [0], [0]

    def new_child(box, j, h, lev):
        level.append(lev); par.append(box); nchild.append(0); child.append([-1] * nch)
        cen.append(np.array([cen[box][d] + (h if (j >> d) & 1 else -h) for d in range(dim)]))

    for l in range(L):  # k_ref_count / k_scan_top / k_ref_rank, k_ref_children
        thr = ndiv0 if l < levcut else ndiv
        shift, h, first = np.uint64(dim * (L - 1 - l)), bsz[l + 1] / 2, len(level)
        for box in range(lfirst[l], llast[l] + 1):
            if r1[box] - r0[box] <= thr:
                continue
            dg = ((key[r0[box]:r1[box]] >> shift) & np.uint64(nch - 1)).astype(np.int64)
            nchild[box] = nch
            for j in range(nch):
                child[box][j] = len(level)
                new_child(box, j, h, l + 1)
                r0.append(r0[box] + np.searchsorted(dg, j))
                r1.append(r0[box] + np.searchsorted(dg, j + 1) if j < nch - 1 else r1[box])
        if len(level) == first:
            break
        lfirst.append(first)
        llast.append(len(level) - 1)
    lev = len(lfirst) - 1

    def touch(x, y, lim):
        return all(abs(cen[x][d] - cen[y][d]) <= lim for d in range(dim))

    coll = {0: [0]}

    def colleagues(b, lim):
        return [kb for jb in coll[par[b]] for kb in child[jb] if kb >= 0 and touch(kb, b, lim)]

    for l in range(1, lev + 1):  # k_ref_colleagues
        for b in range(lfirst[l], llast[l] + 1):
            coll[b] = colleagues(b, F105 * bsz[l])
    flag = [0] * len(level)
    RL = [[(lfirst[l], llast[l]) if l <= lev else None, None, None] for l in range(lev + 2)]

    def boxes(l):
        return [b for r in RL[l] if r is not None for b in range(r[0], r[1] + 1)]

    def refine(box):
        h, ids = bsz[level[box] + 1] / 2, []
        nchild[box] = nch
        for j in range(nch):
            child[box][j] = len(level)
            ids.append(len(level))
            new_child(box, j, h, level[box] + 1)
            flag.append(3 if flag[box] == 1 else 0)
        return ids

    passes = [0, 0]
    if lev >= 2:
        for b in range(lfirst[2], llast[lev] + 1):  # k_lr_flag1
            l, dad = level[b], par[b]
            for jb in coll[par[dad]]:
                if nchild[jb] == 0 and flag[jb] == 0 and touch(jb, dad, 1.05 * (bsz[l - 1] + bsz[l - 2]) / 2.0):
                    flag[jb] = 1
        for l in range(lev, 0, -1):  # k_lr_flag2
            for b in range(lfirst[l], llast[l] + 1):
                if flag[b] in (1, 2):
                    for jb in coll[par[b]]:
                        if nchild[jb] == 0 and flag[jb] == 0 and touch(jb, b, 1.05 * (bsz[l] + bsz[l - 1]) / 2.0):
                            flag[jb] = 2
        for l in range(1, lev - 1):  # first pass, original boxes in id order
            ids = [c for b in range(lfirst[l], llast[l] + 1) if flag[b] > 0 for c in refine(b)]
            if ids:
                RL[l + 1][1] = (ids[0], ids[-1])
                passes[0] += len(ids)
        for l in range(1, lev + 1):
            for b in boxes(l):
                coll[b] = colleagues(b, F105 * bsz[l])
        flag = [f if f == 3 else 0 for f in flag]
        for l in range(2, lev - 1):  # second pass, level by level
            for box in boxes(l):  # k_lr_update
                if flag[box] != 3:
                    continue
                flag[box] = int(any(kb >= 0 and nchild[kb] > 0 and touch(kb, box, 1.05 * (bsz[l] + bsz[l + 1]) / 2.0)
                                    for jb in coll[box] for kb in child[jb]))
            ids = [c for b in boxes(l) if flag[b] > 0 for c in refine(b)]
            if ids:
                RL[l + 1][2] = (ids[0], ids[-1])
                passes[1] += len(ids)
                for b in ids:
                    coll[b] = colleagues(b, F105 * bsz[l + 1])
    order = [b for l in range(lev + 1) for b in boxes(l)]
    mp = {b: i for i, b in enumerate(order)}
    out = {"ilevel": np.array([level[b] for b in order]),
           "iparent": np.array([mp[par[b]] if par[b] >= 0 else -1 for b in order]),
           "nchild": np.array([nchild[b] for b in order]),
           "ichild": np.array([[mp[c] if c >= 0 else -1 for c in child[b]] for b in order]),
           "centers": np.array([cen[b] for b in order])}
    fcoll, start = [[0]], 1
    for l in range(1, lev + 1):  # colleagues of the finished tree
        for b in range(start, start + len(boxes(l))):
            fcoll.append([kb for jb in fcoll[out["iparent"][b]] for kb in out["ichild"][jb]
                          if kb >= 0 and all(abs(out["centers"][kb][d] - out["centers"][b][d]) <= F105 * bsz[l]
                                             for d in range(dim))])
        start += len(boxes(l))
    out["coll"] = fcoll
    return out, passes


def _cases():
    rng = np.random.default_rng(9)
    th = rng.random(20000) * 2 * np.pi
    r = 0.3 + rng.normal(0, 1e-4, 20000)
    c2 = np.concatenate([rng.random((2000, 2)), 0.5 + 1e-3 * rng.standard_normal((14000, 2))])
    c3 = np.concatenate([rng.random((3000, 3)), 0.3 + 1e-3 * rng.standard_normal((12000, 3))])
    return [("2d_thin_circle", 2, 1e-7, 1e-6, np.c_[0.5 + r * np.cos(th), 0.5 + r * np.sin(th)]),
            ("2d_point_cluster", 2, 1e-8, 1e-6, c2),
            ("3d_point_cluster", 3, 1e-7, 1e-6, c3),
            ("3d_uniform", 3, 1e-3, 1e-6, rng.random((15000, 3)))]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_device_level_restriction_equals_host_tree(fgt, case):
    name, dim, delta, eps, src = case
    T = fgt.HostTree(dim, delta, eps, src, src)
    got, passes = _device_tree(src, dim, T)
    nb, nch, nco = T["nboxes"], 1 << dim, 9 if dim == 2 else 27
    assert got["ilevel"].size == nb
    assert np.array_equal(got["ilevel"], T["ilevel"])
    assert np.array_equal(np.where(got["iparent"] >= 0, got["iparent"] + 1, -1), T["iparent"])
    assert np.array_equal(got["nchild"], T["nchild"])
    ch = got["ichild"].reshape(-1)
    assert np.array_equal(ch[ch >= 0] + 1, T["ichild"][ch >= 0])
    assert np.array_equal(got["centers"].reshape(-1), T["centers"])
    nn, nbr = T["nnbors"], T["nbors"].reshape(-1, nco) - 1
    assert all(list(nbr[b][:nn[b]]) == got["coll"][b] for b in range(nb))
    if name.endswith("cluster") or name.startswith("2d_thin"):
        assert passes[0] > 0 and passes[1] > 0  # both restriction passes add boxes
