"""The NUFFT scheme (FGT_SCHEME_NUFFT: 2d/nufft, 3d/nufft) on the GPU against
the oracle's restatement of the same scheme and against the FP64 direct sum.

Both sides compute the scheme's plane-wave expansions as the exact sums that
the reference's type-1 / type-2 NUFFTs approximate, so the GPU agrees with
the oracle to rounding (relative l2 <= 1e-12) and with the direct sum as the
plane-wave scheme does (<= 10 eps).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _cases():
    rng = np.random.default_rng(77)
    out = []

    def circle(n):
        th = rng.random(n) * 2 * np.pi
        r = 0.3 + rng.normal(0, 1e-3, n)
        p = np.c_[0.5 + r * np.cos(th), 0.5 + r * np.sin(th)]
        p[: n // 10] = rng.random((n // 10, 2))
        return p

    # name, dim, nd, delta, eps, sources, targets, ifpgh, ifpghtarg
    out.append(("2d_unif_d1e-3_e1e-6", 2, 1, 1e-3, 1e-6, rng.random((40000, 2)), rng.random((20000, 2)), 1, 1))
    out.append(("2d_unif_d1e-2_e1e-3", 2, 1, 1e-2, 1e-3, rng.random((20000, 2)), rng.random((10000, 2)), 1, 1))
    out.append(("2d_circle_d1e-5_e1e-6", 2, 1, 1e-5, 1e-6, circle(60000), circle(20000), 1, 1))
    out.append(("2d_unif_nd2_e1e-9", 2, 2, 1e-3, 1e-9, rng.random((20000, 2)), rng.random((10000, 2)), 1, 1))
    out.append(("2d_grad_hess", 2, 1, 1e-3, 1e-6, rng.random((20000, 2)), rng.random((10000, 2)), 3, 3))
    out.append(("3d_unif_d1e-2_e1e-6", 3, 1, 1e-2, 1e-6, rng.random((30000, 3)), rng.random((10000, 3)), 1, 1))
    out.append(("3d_unif_d1e-3_e1e-6", 3, 1, 1e-3, 1e-6, rng.random((40000, 3)), rng.random((20000, 3)), 1, 1))
    out.append(("3d_grad", 3, 1, 1e-2, 1e-6, rng.random((20000, 3)), rng.random((10000, 3)), 2, 2))
    out.append(("3d_large_delta", 3, 1, 10.0, 1e-6, rng.random((3000, 3)), rng.random((2000, 3)), 1, 1))
    return out


CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_nufft_scheme_parity(case, fgt, oracle):
    name, dim, nd, delta, eps, src, trg, ifpgh, ifpghtarg = case
    rng = np.random.default_rng(len(name))
    q = rng.standard_normal((src.shape[0], nd))
    ctx = fgt.Context(0, precision="fp64", scheme="nufft")
    got = fgt.transform_pgh(dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg, ctx=ctx)
    ref = oracle.fgt_full(dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg, scheme="nufft")
    keys = [k for k, f in (("pot", ifpgh >= 1), ("grad", ifpgh >= 2), ("hess", ifpgh >= 3),
                           ("pottarg", ifpghtarg >= 1), ("gradtarg", ifpghtarg >= 2),
                           ("hesstarg", ifpghtarg >= 3)) if f]
    for k in keys:
        a, b = np.asarray(got[k]).reshape(-1), np.asarray(ref[k]).reshape(-1)
        e = oracle.derr(b, a)
        print(f"{name} {k}: vs oracle {e:.3e}")
        assert e <= FP64_TOL, (k, e)
    # potentials at sampled targets against the direct sum
    if ifpghtarg >= 1:
        idx = np.arange(0, trg.shape[0], max(1, trg.shape[0] // 400))
        ex = oracle.direct_cut(dim, nd, delta, src, q, trg[idx])
        e = oracle.derr(ex, np.asarray(got["pottarg"])[idx])
        print(f"{name} pottarg: vs direct {e:.3e}")
        assert e <= 10 * eps


def test_nufft_scheme_differs_from_planewave_only_by_its_truncations(fgt, oracle):
    """The two schemes share the tree above the cut, the near field and the
    shifts; at eps their results agree to about eps."""
    rng = np.random.default_rng(5)
    src, trg, q = rng.random((30000, 2)), rng.random((10000, 2)), rng.standard_normal((30000, 1))
    a = fgt.transform_pgh(2, 1, 1e-3, 1e-6, src, q, trg, 0, 1, ctx=fgt.Context(0, precision="fp64", scheme="nufft"))
    b = fgt.transform_pgh(2, 1, 1e-3, 1e-6, src, q, trg, 0, 1, ctx=fgt.Context(0, precision="fp64"))
    assert oracle.derr(b["pottarg"], a["pottarg"]) <= 1e-5


def test_nufft_scheme_2d_dipoles_unsupported(fgt):
    rng = np.random.default_rng(6)
    src = rng.random((2000, 2))
    ctx = fgt.Context(0, precision="fp64", scheme="nufft")
    with pytest.raises(fgt.FGTError):
        fgt.transform_pgh(2, 1, 1e-3, 1e-6, src, None, None, 1, 0, ctx=ctx, ifcharge=0, ifdipole=1,
                          rnormal=rng.standard_normal((2000, 2)), dipstr=rng.standard_normal((2000, 1)))
