"""GPU parity of the 3D evaluation routes that bypass the Taylor conversion
kernels: the plane-wave route (g3dpwevalp_vec, g3drouts.f:2268-2362; chosen
when ((p+1)/npw)^3 >= 3, fgt3d.f:1302-1311) and Taylor-route leaves whose
order exceeds the conversion kernels (g3dpw2local_real_vec + g3dlevalp_vec,
g3drouts.f:1774-1938, 1045-1107), both evaluated by k_eval3d_sep for
potentials, and by the derivative kernels when gradients are asked for.
eps = 1e-9 at small delta puts cut-level leaves at order 31 and some on the
plane-wave route.  Bars as the parity tests: FP64 vs the oracle <= 1e-12 (1e-11 for gradients),
vs the exact sum no worse than twice the oracle's own error."""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(3)
    box = lambda n, s, o=0.0: o + rng.random((n, 3)) * s
    return [
        ("clusters_d1.4e-4", 1.41e-4, 1e-9, np.r_[box(6000, 0.2), box(3000, 0.05, 0.05)]),
        ("uniform_d1e-3", 1e-3, 1e-9, rng.random((30000, 3))),
        ("uniform_d1e-2", 1e-2, 1e-9, rng.random((20000, 3))),
        ("clusters_wide", 1.41e-4, 1e-9, np.r_[box(20000, 0.3), box(10000, 0.05, 0.1)]),
    ]


CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("pgh", [1, 2])
def test_eval3d_routes(case, pgh, fgt, oracle):
    name, delta, eps, src = case
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    q = rng.random(src.shape[0])
    trg = rng.random((3000, 3)) * src.max(axis=0)
    ctx = fgt.Context(0, precision="fp64")
    got = fgt.transform_pgh(3, 1, delta, eps, src, q, trg, pgh, pgh, ctx=ctx)
    ref = oracle.fgt_pgh(3, 1, delta, eps, src, q, trg, pgh, pgh)
    for pts, keys in ((src, ("pot", "grad")), (trg, ("pottarg", "gradtarg"))):
        idx = rng.choice(pts.shape[0], 200, replace=False)
        exact = oracle.direct_pgh(3, 1, delta, src, q, pts[idx], pgh=pgh)
        for order, k in enumerate(keys[:pgh]):
            e_ref = oracle.derr(ref[k], got[k])
            e_dir = oracle.derr(exact[order], got[k][idx])
            e_orc = oracle.derr(exact[order], ref[k][idx])
            print(f"{name} pgh={pgh} {k}: vs oracle {e_ref:.2e} vs direct {e_dir:.2e} (oracle {e_orc:.2e})")
            assert e_ref <= (1e-12 if k.startswith("pot") else 1e-11), (k, e_ref)
            assert e_dir <= max(10 * eps, 2 * e_orc), (k, e_dir, e_orc)


def test_eval3d_routes_two_densities(fgt, oracle):
    """Two densities through the same routes (the kernels' density index)."""
    rng = np.random.default_rng(41)
    box = lambda n, s, o=0.0: o + rng.random((n, 3)) * s
    src = np.r_[box(6000, 0.2), box(3000, 0.05, 0.05)]
    q = rng.random((src.shape[0], 2)) - 0.5
    trg = rng.random((2000, 3)) * 0.2
    got = fgt.transform_pgh(3, 2, 1.41e-4, 1e-9, src, q, trg, 1, 1, ctx=fgt.Context(0, precision="fp64"))
    ref = oracle.fgt_pgh(3, 2, 1.41e-4, 1e-9, src, q, trg, 1, 1)
    for k in ("pot", "pottarg"):
        e = oracle.derr(ref[k], got[k])
        print(k, e)
        assert e <= 1e-11, (k, e)
