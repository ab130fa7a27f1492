"""GPU parity of dipole sources (ifdipole = 1, with and without charges)
against the oracle's restatement of g2dformhd/hcd_vec, g3dformhd/hcd_vec,
g3dformpwd/pwcd_vec, g2dformld/lcd_vec, g3dformld/lcd_vec and
g2d_directd*/cd*_vec, g3d_directd*/cd*_vec (2d/planewave/src/g2drouts.f:173-338,
685-840; g2ddirect.f:217-658; 3d/planewave/src/g3drouts.f:197-405, 857-1040,
2042-2262; g3ddirect.f:207-708), through the C ABI.

Bars as the gradient tests: FP64 vs oracle <= 1e-12 (pot), 1e-11 (grad) and
1e-10 (Hessian); vs the exact sums no worse than twice the oracle's own
error (or 20 eps).  Dipole plans run the FP64 near field in either precision
mode, so both modes meet the FP64 bar.
"""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSAMPLE = 200


def _cases():
    rng = np.random.default_rng(17)

    def unif(n, d, s=1.0):
        return rng.random((n, d)) * s

    out = []
    # name, dim, nd, delta, eps, sources, targets, ifcharge, ifpgh, ifpghtarg
    out.append(("2d_dip", 2, 1, 1e-4, 1e-6, unif(30000, 2), unif(20000, 2), 0, 1, 1))
    out.append(("2d_cd_h", 2, 1, 1e-4, 1e-6, unif(30000, 2), unif(20000, 2), 1, 3, 3))
    out.append(("2d_dip_g_nd2", 2, 2, 1e-3, 1e-3, unif(20000, 2), unif(10000, 2), 0, 2, 2))
    # orders above 32 below the cut: the FMA form kernel
    out.append(("2d_cd_e9_h", 2, 1, 1e-4, 1e-9, unif(20000, 2), unif(10000, 2), 1, 3, 3))
    out.append(("3d_dip", 3, 1, 1e-2, 1e-3, unif(20000, 3), unif(10000, 3), 0, 1, 1))
    out.append(("3d_cd_h", 3, 1, 3e-3, 1e-4, unif(20000, 3), unif(10000, 3), 1, 3, 3))
    out.append(("3d_dip_g_nd2", 3, 2, 1e-2, 1e-6, unif(20000, 3), unif(5000, 3), 0, 2, 2))
    # root box a leaf below the cut: the direct plane-wave form (g3dformpwd_vec)
    out.append(("3d_pw_form", 3, 1, 1e-2, 1e-3, unif(50, 3, 0.08), unif(50, 3, 0.08), 1, 1, 1))
    out.append(("3d_pw_form_dip", 3, 1, 1e-2, 1e-3, unif(50, 3, 0.08), unif(50, 3, 0.08), 0, 2, 2))
    out.append(("2d_alldirect", 2, 1, 1e-6, 1e-6, unif(3000, 2), unif(2000, 2), 1, 3, 3))
    out.append(("3d_alldirect", 3, 1, 1e-4, 1e-6, unif(3000, 3), unif(2000, 3), 0, 3, 3))
    out.append(("2d_large_delta", 2, 1, 10.0, 1e-6, unif(3000, 2), unif(2000, 2), 1, 3, 3))
    out.append(("3d_large_delta", 3, 1, 10.0, 1e-6, unif(3000, 3), unif(2000, 3), 0, 2, 2))
    return out


CASES = _cases()
KEYS = (("pot", "grad", "hess"), ("pottarg", "gradtarg", "hesstarg"))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("precision", ["fp64", "auto"])
def test_dipoles(case, precision, fgt, oracle):
    name, dim, nd, delta, eps, src, trg, ifcharge, ifpgh, ifpghtarg = case
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    ns = src.shape[0]
    q = 2 * rng.random((ns, nd)) - 1 if ifcharge else None
    rn = rng.normal(size=(ns, dim))
    rn /= np.linalg.norm(rn, axis=1)[:, None]
    ds = rng.random((ns, nd))
    ctx = fgt.Context(0, precision=precision)
    got = fgt.transform_pgh(dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg, ctx=ctx,
                            ifcharge=ifcharge, ifdipole=1, rnormal=rn, dipstr=ds)
    ref = oracle.fgt_full(dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg, rn, ds)
    for flag, pts, keys in ((ifpgh, src, KEYS[0]), (ifpghtarg, trg, KEYS[1])):
        idx = rng.choice(pts.shape[0], min(NSAMPLE, pts.shape[0]), replace=False)
        exact = oracle.direct_full(dim, nd, delta, src, pts[idx], q, rn, ds, pgh=flag)
        for order, k in enumerate(keys[:flag]):
            e_ref = oracle.derr(ref[k], got[k])
            e_dir = oracle.derr(exact[order], got[k][idx])
            e_orc = oracle.derr(exact[order], ref[k][idx])
            tol = (1e-12, 1e-11, 1e-10)[order]
            print(f"{name} {precision} {k}: vs oracle {e_ref:.2e} (tol {tol:.0e}) vs direct "
                  f"{e_dir:.2e} (oracle {e_orc:.2e}) {ref['info']}")
            assert e_ref <= tol, (k, e_ref, tol)
            assert e_dir <= max(20 * eps, 2 * e_orc), (k, e_dir, e_orc)


def test_dipole_plan_api(fgt, oracle):
    """A dipole plan applied twice with new strengths and directions equals
    the one-shot transform, bitwise; a charges-only request on the same
    points is unchanged by the dipole support."""
    rng = np.random.default_rng(23)
    dim, nd, delta, eps = 3, 1, 1e-2, 1e-6
    src, trg = rng.random((20000, 3)), rng.random((10000, 3))
    ctx = fgt.Context(0, precision="fp64")
    plan = fgt.Plan(ctx, dim, nd, delta, eps, src, trg, 2, 1, ifcharge=1, ifdipole=1)
    for _ in range(2):
        q, ds = rng.random((20000, 1)), rng.random((20000, 1))
        rn = rng.normal(size=(20000, 3))
        o = plan.execute_host_full(q, rn, ds)
        one = fgt.transform_pgh(dim, nd, delta, eps, src, q, trg, 2, 1, ctx=ctx, ifdipole=1,
                                rnormal=rn, dipstr=ds)
        for k in ("pot", "grad", "pottarg"):
            assert np.array_equal(o[k], one[k]), k
    plan.close()
    # no sources of either kind: zero fields
    z = fgt.transform_pgh(2, 1, 1e-4, 1e-6, rng.random((500, 2)), None, rng.random((50, 2)), 2, 2,
                          ctx=ctx, ifcharge=0, ifdipole=0)
    assert not np.any(z["pot"]) and not np.any(z["gradtarg"])


def test_dipole_bad_arguments(fgt):
    rng = np.random.default_rng(1)
    src = rng.random((100, 2))
    rn = rng.normal(size=(100, 2))
    ds = rng.random(100)
    rn[3, 1] = np.nan
    with pytest.raises(fgt.FGTError) as e:
        fgt.transform_pgh(2, 1, 1e-4, 1e-6, src, None, None, 1, 0, ctx=fgt.Context(0),
                          ifcharge=0, ifdipole=1, rnormal=rn, dipstr=ds)
    assert e.value.status == 1
    with pytest.raises(fgt.FGTError) as e:
        fgt.transform_pgh(2, 1, 1e-4, 1e-6, src, None, None, 1, 0, ctx=fgt.Context(0),
                          ifcharge=0, ifdipole=2, rnormal=rn, dipstr=ds)
    assert e.value.status == 2
