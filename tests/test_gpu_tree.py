"""The tree built with its point work on the GPU (the build plans use by
default) against the host build, which the CPU tests pin to the oracle's
restatement of pts_tree_build / pts_tree_fix_lr / pts_tree_sort: every
integer field, the centres and the box sizes must be identical, and
transforms planned on either tree must give identical results.

The device build has two forms: the exact-key form (one sort of each
source's child digits, every level a search of each box's key range; the default for
trees of at most 31 levels in 2D, 21 in 3D) and the level-by-level
refinement over all points (deeper trees; FGT_TREE_LEVELWISE=1 selects it
for any tree).  Both are checked."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

INT_FIELDS = ["laddr", "ilevel", "iparent", "nchild", "ichild", "nnbors", "nbors", "isrc",
              "isrcse", "itarg", "itargse"]


def _cases():
    rng = np.random.default_rng(21)
    out = []
    for n in (1000, 50000, 300000):
        out.append((f"2d_uniform_{n}", 2, 1e-4, 1e-6, rng.random((n, 2)), rng.random((n // 2, 2))))
        th = rng.random(n) * 2 * np.pi
        r = 0.3 + rng.normal(0, 1e-3, n)
        c = np.c_[0.5 + r * np.cos(th), 0.5 + r * np.sin(th)]
        out.append((f"2d_circle_{n}", 2, 1e-6, 1e-6, c, c))
        out.append((f"3d_uniform_{n}", 3, 1e-3, 1e-6, rng.random((n, 3)), rng.random((n, 3))))
        cen = rng.random((16, 3)) * 0.8 + 0.1
        b = cen[rng.integers(0, 16, n)] + rng.normal(0, 0.02, (n, 3))
        out.append((f"3d_blobs_{n}", 3, 1e-3, 1e-6, b, rng.random((n // 3, 3))))
    g = np.repeat(np.linspace(0, 1, 33), 40)
    pts = np.c_[g, g[::-1]]
    out.append(("2d_boundaries_dups", 2, 1e-5, 1e-6, pts, pts))
    out.append(("2d_single_point", 2, 1e-4, 1e-6, np.array([[0.3, 0.7]]), np.array([[0.1, 0.2]])))
    # points exactly on box boundaries and centres at every level
    grid = np.array(np.meshgrid(np.linspace(0, 1, 257), np.linspace(0, 1, 257))).reshape(2, -1).T.copy()
    out.append(("2d_grid_exact", 2, 1e-6, 1e-6, grid, grid))
    g3 = np.array(np.meshgrid(*[np.linspace(0, 1, 33)] * 3)).reshape(3, -1).T.copy()
    out.append(("3d_grid_exact", 3, 1e-4, 1e-6, g3, g3[::7]))
    return out


CASES = _cases()


@pytest.fixture(scope="module")
def ctx(fgt):
    return fgt.Context(0, precision="fp64")


@pytest.mark.parametrize("form", ["keys", "levelwise"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_device_tree_equals_host_tree(case, form, fgt, ctx, monkeypatch):
    name, dim, delta, eps, src, trg = case
    if form == "levelwise":
        monkeypatch.setenv("FGT_TREE_LEVELWISE", "1")
    trg_arg = src if trg is src else trg
    a = fgt.HostTree(dim, delta, eps, src, trg_arg)
    b = fgt.DeviceTree(ctx, dim, delta, eps, src, trg_arg)
    for k in ("nlevels", "nboxes", "npwlevel", "nlmax"):
        assert a[k] == b[k], k
    if "laddr" not in a:
        assert "laddr" not in b
        return
    for f in INT_FIELDS:
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["centers"], b["centers"])
    assert np.array_equal(a["boxsize"], b["boxsize"])


@pytest.mark.parametrize("dim,n,delta,eps", [(2, 200000, 1e-6, 1e-6), (2, 60000, 1e-4, 1e-9),
                                             (3, 100000, 1e-3, 1e-6), (2, 500, 10.0, 1e-6)])
@pytest.mark.parametrize("form", ["keys", "levelwise"])
@pytest.mark.parametrize("targets", ["separate", "sources"])
def test_plans_on_either_tree_agree(fgt, dim, n, delta, eps, form, targets, monkeypatch):
    """Transforms planned on the device tree (either form; the level-by-level
    form leaves no tree arrays on the device, so the near-field build uploads
    them) and on the host tree, bitwise; targets apart from the sources, or
    the sources themselves (one permutation serves both)."""
    if form == "levelwise":
        monkeypatch.setenv("FGT_TREE_LEVELWISE", "1")
    rng = np.random.default_rng(n + dim)
    src, trg, q = rng.random((n, dim)), rng.random((n // 2, dim)), rng.standard_normal(n)
    if targets == "sources":
        trg = src
    cd = fgt.Context(0, precision="fp64", tree="device")
    ch = fgt.Context(0, precision="fp64", tree="host")
    pd, ptd = fgt.transform(dim, 1, delta, eps, src, q, trg, 1, 1, ctx=cd)
    ph, pth = fgt.transform(dim, 1, delta, eps, src, q, trg, 1, 1, ctx=ch)
    assert np.array_equal(pd, ph)
    assert np.array_equal(ptd, pth)
