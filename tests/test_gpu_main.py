"""The reference's host/device cut: fgt2dmain_gpu_ / fgt3dmain_gpu_ called with
the reference-layout tree (itree/iptr from the oracle's restated
pts_tree_build) and tree-sorted arrays, as a Fortran caller that keeps its own
tree would call it (fgt2d.f:410-421).  Outputs are incremented."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)
_dp = ctypes.POINTER(ctypes.c_double)


def _ref(v, t):
    return ctypes.byref(t(v))


def _assemble(oracle, dim, delta, eps, src, trg, ifpgh, ifpghtarg):
    T = oracle.tree(dim, delta, eps, src, trg)
    nb, nlev, npwl = T["nboxes"], T["nlevels"], T["npwlevel"]
    nadd = max(ifpgh, ifpghtarg)
    nch, nco = (4, 9) if dim == 2 else (8, 27)
    parts = [T["laddr"], T["ilevel"], T["iparent"], T["nchild"], T["ichild"], T["nnbors"], T["nbors"]]
    iptr = [1]
    for a in parts:
        iptr.append(iptr[-1] + a.size)
    itree = np.concatenate(parts).astype(np.int32)
    nlocal = np.zeros(nlev + 1, dtype=np.int32)
    # fgt2d.f:339-355: orders raised by the derivative order, plane-wave eps / 100 for Hessians
    for lev in range(max(npwl, 0), nlev + 1):
        nlocal[lev] = oracle.hlterms(dim, T["boxsize"][lev], delta, eps) + (nadd if nadd >= 2 else 0)
    bs0 = T["boxsize"][0]
    pmax, npw = oracle.pwterms(2 * bs0 / 2.0 ** max(npwl, 0), delta, eps / 100 if nadd > 2 else eps)
    return T, itree, np.array(iptr[:8], dtype=np.int64), nlocal, pmax, npw


@pytest.mark.parametrize("dim,n,delta,eps", [(2, 30000, 1e-4, 1e-6), (2, 20000, 1e-4, 1e-9),
                                             (3, 20000, 1e-2, 1e-6)])
def test_main_gpu_cut(fgt, oracle, dim, n, delta, eps):
    rng = np.random.default_rng(3 * n + dim)
    src, trg, q = rng.random((n, dim)), rng.random((n // 2, dim)), rng.random(n)
    T, itree, iptr, nlocal, pmax, npw = _assemble(oracle, dim, delta, eps, src, trg, 1, 1)
    isrc, itarg = T["isrc"] - 1, T["itarg"] - 1
    ss = np.ascontiguousarray(src[isrc])
    qs = np.ascontiguousarray(q[isrc])
    ts = np.ascontiguousarray(trg[itarg])
    pot = np.full(n, 0.5)        # outputs are incremented: start from a known value
    pt = np.full(n // 2, -0.25)
    L = fgt.lib()
    dummy = np.zeros(2)
    iaddr = np.zeros(2, dtype=np.int32)
    P = lambda a: a.ctypes.data_as(_dp)
    I = lambda a: a.ctypes.data_as(_ip)
    common = [_ref(1, ctypes.c_int), _ref(delta, ctypes.c_double), _ref(eps, ctypes.c_double),
              _ref(n, ctypes.c_int), P(ss), _ref(1, ctypes.c_int), P(qs), _ref(0, ctypes.c_int),
              P(dummy), P(dummy), _ref(n // 2, ctypes.c_int), P(ts), I(iaddr), P(dummy), I(itree)]
    tail = [_ref(T["nboxes"], ctypes.c_int), _ref(0, ctypes.c_int), P(T["boxsize"]),
            P(T["centers"]), I(T["laddr"]), I(T["isrcse"]), I(T["itargse"]), I(nlocal), I(nlocal),
            _ref(int(nlocal.max()), ctypes.c_int), _ref(pmax, ctypes.c_double),
            _ref(npw, ctypes.c_int), _ref(1, ctypes.c_int), P(pot), P(dummy), P(dummy),
            _ref(1, ctypes.c_int), P(pt), P(dummy), P(dummy)]
    if dim == 2:
        iptr32 = iptr.astype(np.int32)
        st = L.fgt2dmain_gpu_(*common, _ref(itree.size, ctypes.c_int), I(iptr32),
                              _ref(T["nlevels"], ctypes.c_int), _ref(T["npwlevel"], ctypes.c_int),
                              *tail)
    else:
        st = L.fgt3dmain_gpu_(*common, _ref(itree.size, ctypes.c_longlong),
                              iptr.ctypes.data_as(_lp), _ref(T["nlevels"], ctypes.c_int),
                              _ref(T["npwlevel"], ctypes.c_int), _ref(100, ctypes.c_int), *tail)
    assert st == 0
    opot, opt, _ = oracle.fgt(dim, 1, delta, eps, src, q, trg, 1, 1)
    # the default context runs the mixed form at eps >= 1e-6 (FP32 near-field
    # exponentials), the plain FP64 form below
    tol = eps if eps >= 1e-6 else 1e-12
    assert oracle.derr(opot[isrc, 0], pot - 0.5) <= tol
    assert oracle.derr(opt[itarg, 0], pt + 0.25) <= tol


@pytest.mark.parametrize("dim,n,delta,eps,pgh", [(2, 20000, 1e-4, 1e-6, 3), (3, 10000, 1e-3, 1e-6, 2)])
def test_main_gpu_cut_gradients(fgt, oracle, dim, n, delta, eps, pgh):
    """The cut with gradients / Hessians: incremented grad and hess arrays."""
    rng = np.random.default_rng(5 * n + dim)
    src, trg, q = rng.random((n, dim)), rng.random((n // 2, dim)), rng.random(n)
    T, itree, iptr, nlocal, pmax, npw = _assemble(oracle, dim, delta, eps, src, trg, pgh, pgh)
    isrc, itarg = T["isrc"] - 1, T["itarg"] - 1
    ss, qs, ts = (np.ascontiguousarray(a) for a in (src[isrc], q[isrc], trg[itarg]))
    H = 3 if dim == 2 else 6
    nt = n // 2
    pot, pt = np.full(n, 0.5), np.full(nt, -0.25)
    grad, gt = np.full((n, dim), 1.0), np.full((nt, dim), 2.0)
    hess, ht = np.zeros((n, H)), np.zeros((nt, H))
    L = fgt.lib()
    dummy = np.zeros(2)
    iaddr = np.zeros(2, dtype=np.int32)
    P = lambda a: a.ctypes.data_as(_dp)
    I = lambda a: a.ctypes.data_as(_ip)
    common = [_ref(1, ctypes.c_int), _ref(delta, ctypes.c_double), _ref(eps, ctypes.c_double),
              _ref(n, ctypes.c_int), P(ss), _ref(1, ctypes.c_int), P(qs), _ref(0, ctypes.c_int),
              P(dummy), P(dummy), _ref(nt, ctypes.c_int), P(ts), I(iaddr), P(dummy), I(itree)]
    tail = [_ref(T["nboxes"], ctypes.c_int), _ref(0, ctypes.c_int), P(T["boxsize"]),
            P(T["centers"]), I(T["laddr"]), I(T["isrcse"]), I(T["itargse"]), I(nlocal), I(nlocal),
            _ref(int(nlocal.max()), ctypes.c_int), _ref(pmax, ctypes.c_double),
            _ref(npw, ctypes.c_int), _ref(pgh, ctypes.c_int), P(pot), P(grad), P(hess),
            _ref(pgh, ctypes.c_int), P(pt), P(gt), P(ht)]
    if dim == 2:
        st = L.fgt2dmain_gpu_(*common, _ref(itree.size, ctypes.c_int), I(iptr.astype(np.int32)),
                              _ref(T["nlevels"], ctypes.c_int), _ref(T["npwlevel"], ctypes.c_int),
                              *tail)
    else:
        st = L.fgt3dmain_gpu_(*common, _ref(itree.size, ctypes.c_longlong),
                              iptr.ctypes.data_as(_lp), _ref(T["nlevels"], ctypes.c_int),
                              _ref(T["npwlevel"], ctypes.c_int), _ref(100, ctypes.c_int), *tail)
    assert st == 0
    ref = oracle.fgt_pgh(dim, 1, delta, eps, src, q, trg, pgh, pgh)
    tol = eps  # the default context runs the mixed form at eps >= 1e-6
    assert oracle.derr(ref["pot"][isrc, 0], pot - 0.5) <= tol
    assert oracle.derr(ref["grad"][isrc, :, 0], grad - 1.0) <= 10 * tol
    assert oracle.derr(ref["gradtarg"][itarg, :, 0], gt - 2.0) <= 10 * tol
    if pgh == 3:
        assert oracle.derr(ref["hess"][isrc, :, 0], hess) <= 10 * tol
        assert oracle.derr(ref["hesstarg"][itarg, :, 0], ht) <= 10 * tol
