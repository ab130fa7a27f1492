"""CPU checks of the oracle: the reference's own known-answer test (FGT vs FP64
direct sum, relative l2 ``derr``), independent restatements of the generator
and the expansion-length formulas, and the golden fixtures."""
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "oracle_golden.npz")


def test_dlaran_known_answer(oracle):
    """DLARAN is x_{k+1} = a x_k mod 2^48, a = 33952834046453 (dlaran.f:36-40),
    seed (0,0,0,1) -> x_0 = 1; checked with exact integers."""
    vals = oracle.hkrand(20, reset=True)
    a, m, x = 33952834046453, 2 ** 48, 1
    for v in vals:
        x = (a * x) % m
        assert v == x / m


def _hlterms(ndim, bsize, delta, eps):
    # g2dterms.f:19-64, written independently (1.09 is a single-precision literal)
    e1 = math.exp(1.0)
    r = bsize / math.sqrt(2.0 * delta)
    p0 = int(e1 * r * r) + 1
    rk = float(np.float32(1.09)) * (8 * math.atan(1.0)) ** -0.25
    for p in range(p0, 301):
        rp = r * math.sqrt(e1 / p)
        err = ndim * rk * p ** -0.25 * rp ** p / (1 - rp)
        if err < eps:
            return p
    return -1


def _pwterms(bsize, delta, eps):
    rmax = bsize / math.sqrt(delta)
    d = math.sqrt(math.log(1.0 / eps))
    pmax = 2.0 * d
    h = 2 * math.pi / (rmax + d)
    return pmax, 2 * int(pmax / h)


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-9, 1e-12])
def test_term_counts(oracle, ndim, eps):
    for delta in (1e-6, 1e-4, 1e-2):
        for bs in (0.1, 0.01, 1e-3, 5e-4):
            assert oracle.hlterms(ndim, bs, delta, eps) == _hlterms(ndim, bs, delta, eps)
        pm, n = oracle.pwterms(0.2, delta, eps)
        pm2, n2 = _pwterms(0.2, delta, eps)
        assert n == n2 and abs(pm - pm2) < 1e-12


def test_cut_level_and_npw_of_configs(oracle):
    """npwlevel / npw of the benchmark configurations as derived from the
    reference formulas (2D uniform N=1e5: npwlevel 5, npw 38; 2D circle
    delta=eps=1e-6: npwlevel 9, npw 26)."""
    rng = np.random.default_rng(0)
    pts = rng.random((1000, 2))
    pts[0] = (0, 0)
    pts[1] = (1, 1)
    lc, bs0, _ = oracle.boxsize0(2, 1e-4, 1e-9, pts, pts)
    assert lc == 5
    _, npw = oracle.pwterms(2 * bs0 / 2 ** 5, 1e-4, 1e-9)
    assert npw == 38
    lc, bs0, _ = oracle.boxsize0(2, 1e-6, 1e-6, pts, pts)
    assert lc == 9
    _, npw = oracle.pwterms(2 * bs0 / 2 ** 9, 1e-6, 1e-6)
    assert npw == 26


def test_reference_driver_2d_known_answer(oracle):
    """test_fgt2d.f: FGT vs direct sum on the first 20 sources (reduced N)."""
    src, q, trg, delta, eps = oracle.reference_test_inputs_2d(5000)
    pot, _, _ = oracle.fgt(2, 1, delta, eps, src, q, trg, 1, 0)
    ex = oracle.direct(2, 1, delta, src, q, src[:20])
    assert oracle.derr(ex, pot[:20]) <= 10 * eps


def test_reference_driver_3d_known_answer(oracle):
    src, q, trg, delta, eps = oracle.reference_test_inputs_3d(5000)
    pot, _, _ = oracle.fgt(3, 1, delta, eps, src, q, trg, 1, 0)
    ex = oracle.direct(3, 1, delta, src, q, src[:20])
    assert oracle.derr(ex, pot[:20]) <= 10 * eps


@pytest.mark.parametrize("dim,n,delta,eps", [(2, 20000, 1e-4, 1e-9), (2, 20000, 1e-4, 1e-6),
                                             (3, 15000, 1e-2, 1e-6), (3, 8000, 1e-3, 1e-3),
                                             (2, 3000, 10.0, 1e-6), (3, 3000, 10.0, 1e-6)])
def test_plane_wave_path_vs_direct(oracle, dim, n, delta, eps):
    rng = np.random.default_rng(n + dim)
    src, trg, q = rng.random((n, dim)), rng.random((n // 2, dim)), rng.random(n)
    pot, pt, info = oracle.fgt(dim, 1, delta, eps, src, q, trg, 1, 1)
    idx = rng.choice(n, 200, replace=False)
    assert oracle.derr(oracle.direct(dim, 1, delta, src, q, src[idx]), pot[idx]) <= 10 * eps
    jdx = rng.choice(n // 2, 200, replace=False)
    assert oracle.derr(oracle.direct(dim, 1, delta, src, q, trg[jdx]), pt[jdx]) <= 10 * eps


def test_golden_fixtures(oracle):
    g = np.load(GOLDEN)
    assert np.array_equal(oracle.hkrand(64, reset=True), g["hkrand_first64"])
    src, q, trg, delta, eps = oracle.reference_test_inputs_2d(3000)
    pot, _, info = oracle.fgt(2, 1, delta, eps, src, q, trg, 1, 0)
    assert np.allclose(pot[:20, 0], g["ref2d_pot_first20"], rtol=1e-13, atol=1e-16)
    assert oracle.derr(g["ref2d_direct_first20"], pot[:20, 0]) <= 10 * eps
    src, q, trg, delta, eps = oracle.reference_test_inputs_3d(3000)
    pot, _, _ = oracle.fgt(3, 1, delta, eps, src, q, trg, 1, 0)
    assert np.allclose(pot[:20, 0], g["ref3d_pot_first20"], rtol=1e-13, atol=1e-16)
    rng = np.random.default_rng(1235)
    s2, t2, c2 = rng.random((20000, 2)), rng.random((20000, 2)), rng.random(20000)
    p2, pt2, _ = oracle.fgt(2, 1, 1e-4, 1e-9, s2, c2, t2, 1, 1)
    assert np.allclose(p2[:50, 0], g["pw2d_pot_first50"], rtol=1e-12)
    assert np.allclose(pt2[:50, 0], g["pw2d_pottarg_first50"], rtol=1e-12)


def test_derr_switches_to_absolute(oracle):
    """derr uses an absolute norm when the exact vector is tiny (test_fgt2d.f:216-221)."""
    ex = np.full(10, 1e-12)
    ap = ex + 1e-13
    assert abs(oracle.derr(ex, ap) - np.sqrt(10 * 1e-26) / 10) < 1e-20


def test_direct_derivatives_by_finite_differences(oracle):
    """The exact-sum gradient and Hessian (the checker of the gradient tests)
    against central differences of the exact potential."""
    rng = np.random.default_rng(3)
    for dim in (2, 3):
        delta = 1e-2
        src, q = rng.random((200, dim)), rng.random((200, 1))
        x = rng.random((5, dim))
        p, g, h = oracle.direct_pgh(dim, 1, delta, src, q, x)
        assert np.allclose(p, oracle.direct(dim, 1, delta, src, q, x), rtol=1e-14)
        step = 1e-5
        pairs = [(0, 0), (0, 1), (1, 1)] if dim == 2 else \
            [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
        for d in range(dim):
            e = np.zeros(dim)
            e[d] = step
            fd = (oracle.direct(dim, 1, delta, src, q, x + e) - oracle.direct(dim, 1, delta, src, q, x - e)) / (2 * step)
            assert np.allclose(g[:, d], fd, rtol=1e-6, atol=1e-8)
        for c, (a, b) in enumerate(pairs):
            ea, eb = np.zeros(dim), np.zeros(dim)
            ea[a] = step
            eb[b] = step
            fd = (oracle.direct_pgh(dim, 1, delta, src, q, x + eb)[1][:, a] -
                  oracle.direct_pgh(dim, 1, delta, src, q, x - eb)[1][:, a]) / (2 * step)
            assert np.allclose(h[:, c], fd, rtol=1e-5, atol=1e-6), (dim, c)


@pytest.mark.parametrize("dim,n,delta,eps", [(2, 20000, 1e-4, 1e-6), (2, 10000, 1e-4, 1e-9),
                                             (3, 10000, 1e-3, 1e-6), (3, 8000, 1e-2, 1e-3),
                                             (2, 3000, 10.0, 1e-6), (3, 3000, 10.0, 1e-6)])
def test_oracle_derivatives_vs_direct(oracle, dim, n, delta, eps):
    """Gradients and Hessians of the restated transform (g2dlevalg/h_vec,
    g2dpwevalg/h_vec, g2d_directcg/ch_vec and the 3D twins) against the exact
    derivatives.  The reference raises the orders by the derivative order
    and divides the plane-wave eps by 100 for Hessians (fgt2d.f:340-356);
    its derivative error grows with the derivative order, so the bars are
    10, 100 and 1000 eps."""
    rng = np.random.default_rng(n + 7 * dim)
    src, trg, q = rng.random((n, dim)), rng.random((n // 2, dim)), rng.random(n)
    r = oracle.fgt_pgh(dim, 1, delta, eps, src, q, trg, 3, 3)
    for pts, keys in ((src, ("pot", "grad", "hess")), (trg, ("pottarg", "gradtarg", "hesstarg"))):
        idx = rng.choice(pts.shape[0], 150, replace=False)
        exact = oracle.direct_pgh(dim, 1, delta, src, q, pts[idx])
        for order, k in enumerate(keys):
            assert oracle.derr(exact[order], r[k][idx]) <= 10 ** (order + 1) * eps, (k, order)
    # pot-only requests through the gradient entry are the plain transform
    # (up to the order of the near field's threaded accumulation)
    r1 = oracle.fgt_pgh(dim, 1, delta, eps, src, q, trg, 1, 1)
    pot, pt, _ = oracle.fgt(dim, 1, delta, eps, src, q, trg, 1, 1)
    assert oracle.derr(pot, r1["pot"]) <= 1e-14 and oracle.derr(pt, r1["pottarg"]) <= 1e-14


def test_direct_dipoles_are_source_derivatives(oracle):
    """The exact dipole field (the checker of the dipole tests) is the
    derivative of the charge field along n at the source, times dipstr
    (g2d_directdp_vec: grad_s exp(-r^2/delta) . n)."""
    rng = np.random.default_rng(4)
    for dim in (2, 3):
        delta, step = 1e-2, 1e-6
        src, x = rng.random((50, dim)), rng.random((6, dim))
        n = rng.normal(size=(50, dim))
        n /= np.linalg.norm(n, axis=1)[:, None]
        ds = rng.random((50, 1))
        p, g, h = oracle.direct_full(dim, 1, delta, src, x, None, n, ds, pgh=3)
        fd = (oracle.direct_full(dim, 1, delta, src + step * n, x, ds, pgh=3)[0] -
              oracle.direct_full(dim, 1, delta, src - step * n, x, ds, pgh=3)[0]) / (2 * step)
        assert np.allclose(p, fd, rtol=1e-6, atol=1e-8)
        fdg = (oracle.direct_full(dim, 1, delta, src + step * n, x, ds, pgh=3)[1] -
               oracle.direct_full(dim, 1, delta, src - step * n, x, ds, pgh=3)[1]) / (2 * step)
        assert np.allclose(g, fdg, rtol=1e-5, atol=1e-6)
        fdh = (oracle.direct_full(dim, 1, delta, src + step * n, x, ds, pgh=3)[2] -
               oracle.direct_full(dim, 1, delta, src - step * n, x, ds, pgh=3)[2]) / (2 * step)
        assert np.allclose(h, fdh, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("dim,n,delta,eps", [(2, 20000, 1e-4, 1e-6), (3, 10000, 1e-3, 1e-6),
                                             (3, 8000, 1e-2, 1e-3), (2, 3000, 10.0, 1e-6),
                                             (3, 3000, 10.0, 1e-6)])
def test_oracle_dipoles_vs_direct(oracle, dim, n, delta, eps):
    """Dipoles (g2dformhd/hcd_vec, g3dformpwd_vec, g2dformld_vec,
    g2d_directd*/cd*_vec and the 3D twins) with and without charges.  The
    dipole field is one derivative rougher than the charge field, so the
    bars are twice the charge ones (20, 200, 2000 eps)."""
    rng = np.random.default_rng(n + 11 * dim)
    src, trg = rng.random((n, dim)), rng.random((n // 2, dim))
    q, ds = rng.random(n), rng.random(n)
    rn = rng.normal(size=(n, dim))
    rn /= np.linalg.norm(rn, axis=1)[:, None]
    for charge in (None, q):
        r = oracle.fgt_full(dim, 1, delta, eps, src, charge, trg, 3, 3, rn, ds)
        idx = rng.choice(n // 2, 150, replace=False)
        exact = oracle.direct_full(dim, 1, delta, src, trg[idx], charge, rn, ds, pgh=3)
        for order, k in enumerate(("pottarg", "gradtarg", "hesstarg")):
            assert oracle.derr(exact[order], r[k][idx]) <= 2 * 10 ** (order + 1) * eps, (k, order)
