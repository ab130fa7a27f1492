"""The gfortran-ABI drop-ins ``fgt2d_`` / ``fgt3d_`` / ``fgt2d_st_`` / ``fgt3d_st_``
called the way a Fortran caller calls ``fgt2d``: every argument by reference,
arrays in the reference's column-major layouts (fgt2d.f:19-22 and docs
:23-61; fgt3d.f:19-64).  Outputs are compared with the oracle (the restated
reference driver) at the FP64 bar, and the status variants must set ``ier`` on
bad input and write no partial result (outputs untouched, or zeroed when the
check that failed ran after the plan started)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_dp = ctypes.POINTER(ctypes.c_double)


def _i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _d(v):
    return ctypes.byref(ctypes.c_double(float(v)))


def _a(x):
    return x.ctypes.data_as(_dp)


def _call(L, dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg, status=False, ifdipole=0,
          rnormal=None, dipstr=None):
    ns, nt = src.shape[0], trg.shape[0]
    H = 3 if dim == 2 else 6
    pot = np.full((ns, nd), np.nan)
    grad = np.full((ns, dim, nd), np.nan)
    hess = np.full((ns, H, nd), np.nan)
    pt = np.full((nt, nd), np.nan)
    gt = np.full((nt, dim, nd), np.nan)
    ht = np.full((nt, H, nd), np.nan)
    rn = rnormal if rnormal is not None else np.zeros((ns, dim))
    ds = dipstr if dipstr is not None else np.zeros((ns, nd))
    args = [_i(nd), _d(delta), _d(eps), _i(ns), _a(src), _i(1), _a(q), _i(ifdipole), _a(rn), _a(ds),
            _i(0), _i(ifpgh), _a(pot), _a(grad), _a(hess), _i(nt), _a(trg), _i(ifpghtarg), _a(pt),
            _a(gt), _a(ht)]
    ier = ctypes.c_int(-1)
    fn = {(2, False): L.fgt2d_, (3, False): L.fgt3d_, (2, True): L.fgt2d_st_,
          (3, True): L.fgt3d_st_}[(dim, status)]
    if status:
        args.append(ctypes.byref(ier))
    fn.restype = None
    fn(*args)
    return pot, grad, hess, pt, gt, ht, ier.value


@pytest.mark.parametrize("dim,delta,eps,ifpgh,ifpghtarg,status", [
    (2, 1e-4, 1e-6, 1, 1, False), (2, 1e-3, 1e-9, 2, 1, True), (3, 1e-2, 1e-6, 1, 3, False),
    (3, 1e-3, 1e-6, 3, 2, True)])
def test_dropin_matches_oracle(fgt, oracle, dim, delta, eps, ifpgh, ifpghtarg, status):
    rng = np.random.default_rng(1000 + 10 * dim + ifpgh + ifpghtarg)
    nd, ns, nt = 2, 12000 if dim == 2 else 6000, 5000
    src, trg = rng.random((ns, dim)), rng.random((nt, dim))
    q = rng.random((ns, nd))
    pot, grad, hess, pt, gt, ht, ier = _call(fgt.lib(), dim, nd, delta, eps, src, q, trg, ifpgh,
                                             ifpghtarg, status=status)
    if status:
        assert ier == 0
    o = oracle.fgt_pgh(dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg)
    opot, ograd, ohess = o["pot"], o["grad"], o["hess"]
    opt, ogt, oht = o["pottarg"], o["gradtarg"], o["hesstarg"]
    # the drop-ins run the default context: the mixed form at eps >= 1e-6
    # (parity bar eps, 10 eps for derivatives), the FP64 form below it
    tol = (eps, 10 * eps, 10 * eps) if eps >= 1e-6 else (1e-12, 1e-11, 1e-10)
    if ifpgh >= 1:
        assert oracle.derr(opot, pot) <= tol[0]
    if ifpgh >= 2:
        assert oracle.derr(ograd, grad.reshape(ograd.shape)) <= tol[1]
    if ifpgh >= 3:
        assert oracle.derr(ohess, hess.reshape(ohess.shape)) <= tol[2]
    if ifpghtarg >= 1:
        assert oracle.derr(opt, pt) <= tol[0]
    if ifpghtarg >= 2:
        assert oracle.derr(ogt, gt.reshape(ogt.shape)) <= tol[1]
    if ifpghtarg >= 3:
        assert oracle.derr(oht, ht.reshape(oht.shape)) <= tol[2]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("bad", ["eps", "nd", "nan", "ifpgh"])
def test_dropin_status_on_bad_input(fgt, dim, bad):
    rng = np.random.default_rng(5)
    src, trg, q = rng.random((500, dim)), rng.random((300, dim)), rng.random((500, 1))
    eps, nd, ifpgh = 1e-6, 1, 1
    if bad == "eps":
        eps = 2.0
    elif bad == "nd":
        nd = 0
    elif bad == "nan":
        src[17, 0] = np.nan
    else:
        ifpgh = 7
    pot, _, _, pt, _, _, ier = _call(fgt.lib(), dim, max(nd, 1), 1e-3, eps, src, q, trg, ifpgh, 1,
                                     status=True) if bad != "nd" else _call_nd0(fgt.lib(), dim, src, q, trg)
    assert ier in (1, 2), ier
    assert np.all(np.isnan(pt)) or np.all(pt == 0.0)


def _call_nd0(L, dim, src, q, trg):
    """nd = 0 passed through the status variant (the arrays are sized for 1)."""
    ns, nt = src.shape[0], trg.shape[0]
    pot = np.full((ns, 1), np.nan)
    pt = np.full((nt, 1), np.nan)
    z = np.zeros(1)
    ier = ctypes.c_int(-1)
    fn = L.fgt2d_st_ if dim == 2 else L.fgt3d_st_
    fn.restype = None
    fn(_i(0), _d(1e-3), _d(1e-6), _i(ns), _a(src), _i(1), _a(q), _i(0), _a(z), _a(z), _i(0), _i(1),
       _a(pot), _a(z), _a(z), _i(nt), _a(trg), _i(1), _a(pt), _a(z), _a(z), ctypes.byref(ier))
    return pot, None, None, pt, None, None, ier.value
