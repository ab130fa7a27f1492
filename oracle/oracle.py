"""ORACLE -- test infrastructure only.

ctypes front end for ``oracle/fgt_oracle.cpp``, a CPU restatement of the
reference plane-wave FGT (flatironinstitute/fgt2d, 2d/planewave and
3d/planewave).  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` import this module; the product package never does.

Parity pin: the reference's only known-answer test is the FGT against an FP64
direct sum at sampled targets, scored with ``derr`` (relative l2, switching to
absolute below 1e-10; 2d/planewave/test/test_fgt2d.f:204-225).  ``derr`` and
the hkrand/DLARAN input generator (hkrand.f:3-19, dlaran.f:1-89) are restated
here so the reference test cases can be regenerated exactly.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libfgt_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile the oracle shared library with its Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_SO) or (
        os.path.getmtime(_SO) < os.path.getmtime(os.path.join(_HERE, "fgt_oracle.cpp"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        L.orc_fgt.restype = ctypes.c_int
        L.orc_fgt.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                              ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                              _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _ip, ctypes.c_int]
        L.orc_fgt_pgh.restype = ctypes.c_int
        L.orc_fgt_pgh.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                  _dp, _dp, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp,
                                  _ip, ctypes.c_int]
        L.orc_fgt_full.restype = ctypes.c_int
        L.orc_fgt_full.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp,
                                   ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _dp, ctypes.c_int,
                                   _dp, _dp, _dp, _ip, ctypes.c_int]
        L.orc_fgt_expansions.restype = ctypes.c_int
        L.orc_fgt_expansions.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, _ip, ctypes.c_int]
        L.orc_fgt_nufft.restype = ctypes.c_int
        L.orc_fgt_nufft.argtypes = L.orc_fgt_full.argtypes
        L.orc_direct_cut.restype = None
        L.orc_direct_cut.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.orc_direct_full.restype = None
        L.orc_direct_full.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                      _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp,
                                      ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]
        L.orc_direct_pgh.restype = None
        L.orc_direct_pgh.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                     _dp, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp,
                                     ctypes.c_int]
        L.orc_direct.restype = None
        L.orc_direct.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp,
                                 _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.orc_hkrand.argtypes = [ctypes.c_longlong, _dp]
        L.orc_hkrand_reset.argtypes = []
        L.orc_hlterms.restype = ctypes.c_int
        L.orc_hlterms.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_pwterms.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _ip]
        L.orc_boxsize0.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   _dp, ctypes.c_int, _dp, _ip, _dp, _dp]
        L.orc_tree_build.restype = ctypes.c_void_p
        L.orc_tree_build.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                     _dp, ctypes.c_int, _dp]
        L.orc_tree_dims.argtypes = [ctypes.c_void_p, _ip]
        L.orc_tree_int.restype = ctypes.c_longlong
        L.orc_tree_int.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip]
        L.orc_tree_dbl.restype = ctypes.c_longlong
        L.orc_tree_dbl.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_tree_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def fgt(dim, nd, delta, eps, sources, charge, targ=None, ifpgh=1, ifpghtarg=0, nthreads=0):
    """Run the restated reference transform.

    ``sources`` is (ns, dim) (the reference's ``sources(dim, ns)`` in
    row-major), ``charge`` is (ns, nd) or (ns,), ``targ`` is (nt, dim).
    Returns (pot (ns, nd), pottarg (nt, nd), info dict).
    """
    src = _f64(sources)
    ns = src.shape[0]
    q = _f64(charge).reshape(ns, nd) if ns else np.zeros((0, nd))
    trg = _f64(targ) if targ is not None else np.zeros((0, dim))
    nt = trg.shape[0]
    pot = np.zeros((max(ns, 1), nd))
    pt = np.zeros((max(nt, 1), nd))
    info = np.zeros(8, dtype=np.int32)
    rc = lib().orc_fgt(dim, nd, float(delta), float(eps), ns, _d(src), 1, _d(q), 0, ifpgh,
                       _d(pot), nt, _d(trg), ifpghtarg, _d(pt), info.ctypes.data_as(_ip), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle fgt returned status {rc}")
    keys = ["npwlevel", "nlevels", "nboxes", "npw", "nlmax", "ndirect_leaves"]
    return pot[:ns], pt[:nt], {k: int(info[i]) for i, k in enumerate(keys)}


def nhess(dim):
    return 3 if dim == 2 else 6


def fgt_pgh(dim, nd, delta, eps, sources, charge, targ=None, ifpgh=1, ifpghtarg=0, nthreads=0):
    """The restated transform with gradients (ifpgh = 2) and Hessians (3).

    Returns a dict of pot (ns, nd), grad (ns, dim, nd), hess (ns, H, nd) and
    the same for the targets (H = 3 in 2D: xx, xy, yy; 6 in 3D: xx, yy, zz,
    xy, xz, yz), each None when not requested, plus ``info``.
    """
    src = _f64(sources)
    ns = src.shape[0]
    q = _f64(charge).reshape(ns, nd) if ns else np.zeros((0, nd))
    trg = _f64(targ) if targ is not None else np.zeros((0, dim))
    nt = trg.shape[0]
    H = nhess(dim)
    pot, grad, hess = np.zeros((max(ns, 1), nd)), np.zeros((max(ns, 1), dim, nd)), np.zeros((max(ns, 1), H, nd))
    pt, gt, ht = np.zeros((max(nt, 1), nd)), np.zeros((max(nt, 1), dim, nd)), np.zeros((max(nt, 1), H, nd))
    info = np.zeros(8, dtype=np.int32)
    rc = lib().orc_fgt_pgh(dim, nd, float(delta), float(eps), ns, _d(src), 1, _d(q), 0, ifpgh,
                           _d(pot), _d(grad), _d(hess), nt, _d(trg), ifpghtarg, _d(pt), _d(gt),
                           _d(ht), info.ctypes.data_as(_ip), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle fgt returned status {rc}")
    keys = ["npwlevel", "nlevels", "nboxes", "npw", "nlmax", "ndirect_leaves"]
    return {"pot": pot[:ns] if ifpgh >= 1 else None, "grad": grad[:ns] if ifpgh >= 2 else None,
            "hess": hess[:ns] if ifpgh >= 3 else None,
            "pottarg": pt[:nt] if ifpghtarg >= 1 else None,
            "gradtarg": gt[:nt] if ifpghtarg >= 2 else None,
            "hesstarg": ht[:nt] if ifpghtarg >= 3 else None,
            "info": {k: int(info[i]) for i, k in enumerate(keys)}}


def fgt_full(dim, nd, delta, eps, sources, charge=None, targ=None, ifpgh=1, ifpghtarg=0,
             rnormal=None, dipstr=None, nthreads=0, scheme="planewave"):
    """The restated transform with charges and/or dipoles (``charge`` or
    ``dipstr`` None switches that source kind off): rnormal (ns, dim),
    dipstr (ns, nd).  scheme "nufft" restates the NUFFT scheme of 2d/nufft,
    3d/nufft (its NUFFTs as the exact sums they approximate).  Returns the
    dict of fgt_pgh."""
    src = _f64(sources)
    ns = src.shape[0]
    ifc, ifd = int(charge is not None), int(dipstr is not None)
    q = _f64(charge).reshape(ns, nd) if ifc else np.zeros((1, nd))
    rn = _f64(rnormal).reshape(ns, dim) if ifd else np.zeros((1, dim))
    ds = _f64(dipstr).reshape(ns, nd) if ifd else np.zeros((1, nd))
    trg = _f64(targ) if targ is not None else np.zeros((0, dim))
    nt = trg.shape[0]
    H = nhess(dim)
    pot, grad, hess = np.zeros((max(ns, 1), nd)), np.zeros((max(ns, 1), dim, nd)), np.zeros((max(ns, 1), H, nd))
    pt, gt, ht = np.zeros((max(nt, 1), nd)), np.zeros((max(nt, 1), dim, nd)), np.zeros((max(nt, 1), H, nd))
    info = np.zeros(8, dtype=np.int32)
    fn = lib().orc_fgt_nufft if scheme == "nufft" else lib().orc_fgt_full
    rc = fn(dim, nd, float(delta), float(eps), ns, _d(src), ifc, _d(q), ifd, _d(rn),
            _d(ds), ifpgh, _d(pot), _d(grad), _d(hess), nt, _d(trg), ifpghtarg,
            _d(pt), _d(gt), _d(ht), info.ctypes.data_as(_ip), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle fgt returned status {rc}")
    keys = ["npwlevel", "nlevels", "nboxes", "npw", "nlmax", "ndirect_leaves"]
    return {"pot": pot[:ns] if ifpgh >= 1 else None, "grad": grad[:ns] if ifpgh >= 2 else None,
            "hess": hess[:ns] if ifpgh >= 3 else None,
            "pottarg": pt[:nt] if ifpghtarg >= 1 else None,
            "gradtarg": gt[:nt] if ifpghtarg >= 2 else None,
            "hesstarg": ht[:nt] if ifpghtarg >= 3 else None,
            "info": {k: int(info[i]) for i, k in enumerate(keys)}}


def expansions(dim, nd, delta, eps, sources, charge, targ, ifpgh, ifpghtarg, boxes, nexp, nthreads=0):
    """The restated transform's plane-wave expansions of ``boxes`` (0-based)
    after the shifts: (mp, loc, has) with mp/loc complex (nbox, nd, nexp)."""
    src = _f64(sources)
    ns = src.shape[0]
    q = _f64(charge).reshape(ns, nd)
    trg = _f64(targ) if targ is not None else np.zeros((0, dim))
    bx = np.ascontiguousarray(boxes, dtype=np.int32)
    mp = np.zeros(2 * len(bx) * nd * nexp)
    lo = np.zeros(2 * len(bx) * nd * nexp)
    has = np.zeros(len(bx), dtype=np.int32)
    rc = lib().orc_fgt_expansions(dim, nd, float(delta), float(eps), ns, _d(src), _d(q), trg.shape[0], _d(trg),
                                  ifpgh, ifpghtarg, len(bx), bx.ctypes.data_as(_ip), _d(mp), _d(lo),
                                  has.ctypes.data_as(_ip), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle expansions returned status {rc}")
    c = lambda a: (a[0::2] + 1j * a[1::2]).reshape(len(bx), nd, nexp)
    return c(mp), c(lo), has.astype(bool)


def direct_full(dim, nd, delta, sources, targ, charge=None, rnormal=None, dipstr=None, pgh=3,
                nthreads=0):
    """Exact sums with charges and/or dipoles: (pot, grad, hess) at targ."""
    src = _f64(sources)
    ns = src.shape[0]
    trg = _f64(targ)
    nt = trg.shape[0]
    ifc, ifd = int(charge is not None), int(dipstr is not None)
    q = _f64(charge).reshape(ns, nd) if ifc else np.zeros((1, nd))
    rn = _f64(rnormal).reshape(ns, dim) if ifd else np.zeros((1, dim))
    ds = _f64(dipstr).reshape(ns, nd) if ifd else np.zeros((1, nd))
    pot, grad, hess = np.zeros((nt, nd)), np.zeros((nt, dim, nd)), np.zeros((nt, nhess(dim), nd))
    lib().orc_direct_full(dim, nd, float(delta), ns, _d(src), ifc, _d(q), ifd, _d(rn), _d(ds), nt,
                          _d(trg), pgh, _d(pot), _d(grad), _d(hess), nthreads)
    return pot, grad, hess


def direct_pgh(dim, nd, delta, sources, charge, targ, pgh=3, nthreads=0):
    """FP64 direct sum without cutoff with gradients and Hessians:
    (pot (nt, nd), grad (nt, dim, nd), hess (nt, H, nd))."""
    src = _f64(sources)
    trg = _f64(targ)
    q = _f64(charge).reshape(src.shape[0], nd)
    nt = trg.shape[0]
    pot, grad, hess = np.zeros((nt, nd)), np.zeros((nt, dim, nd)), np.zeros((nt, nhess(dim), nd))
    lib().orc_direct_pgh(dim, nd, float(delta), src.shape[0], _d(src), _d(q), nt, _d(trg), pgh,
                         _d(pot), _d(grad), _d(hess), nthreads)
    return pot, grad, hess


def direct(dim, nd, delta, sources, charge, targ, nthreads=0):
    """FP64 direct Gaussian sum without cutoff at every target."""
    src = _f64(sources)
    trg = _f64(targ)
    q = _f64(charge).reshape(src.shape[0], nd)
    out = np.zeros((trg.shape[0], nd))
    lib().orc_direct(dim, nd, float(delta), src.shape[0], _d(src), _d(q), trg.shape[0], _d(trg),
                     _d(out), nthreads)
    return out


def direct_cut(dim, nd, delta, sources, charge, targ, nthreads=0):
    """FP64 direct sum at ``targ`` over sources binned on a grid, dropping
    pairs farther apart than sqrt(delta ln 1e30) (terms below 1e-30 of their
    charge): the plain direct sum to rounding, at a cost that does not grow
    with N for a fixed density.  Used for sampled-target errors at full size."""
    src = _f64(sources)
    trg = _f64(targ)
    q = _f64(charge).reshape(src.shape[0], nd)
    out = np.zeros((trg.shape[0], nd))
    rcut = float(np.sqrt(delta * np.log(1e30)))
    lib().orc_direct_cut(dim, nd, float(delta), rcut, src.shape[0], _d(src), _d(q), trg.shape[0],
                         _d(trg), _d(out), nthreads)
    return out


def derr(exact, approx):
    """Relative l2 error of the reference test driver (test_fgt2d.f:204-225)."""
    e = np.asarray(exact, dtype=np.float64).ravel()
    a = np.asarray(approx, dtype=np.float64).ravel()
    n = e.size
    ra = float(np.sum(e * e))
    err = float(np.sum((e - a) ** 2))
    if np.sqrt(ra) / n < 1e-10:
        return np.sqrt(err) / n
    return float(np.sqrt(err / ra))


def hkrand(n, reset=False):
    """``n`` successive values of hkrand(0) (hkrand.f, DLARAN, seed 0,0,0,1)."""
    if reset:
        lib().orc_hkrand_reset()
    out = np.zeros(int(n))
    lib().orc_hkrand(int(n), _d(out))
    return out


def hlterms(ndim, bsize, delta, eps):
    return int(lib().orc_hlterms(ndim, bsize, delta, eps))


def pwterms(bsize, delta, eps):
    pm = ctypes.c_double()
    n = ctypes.c_int()
    lib().orc_pwterms(bsize, delta, eps, ctypes.byref(pm), ctypes.byref(n))
    return pm.value, n.value


def boxsize0(dim, delta, eps, sources, targ):
    src = _f64(sources)
    trg = _f64(targ)
    lc = ctypes.c_int()
    bs = ctypes.c_double()
    cen = np.zeros(3)
    lib().orc_boxsize0(dim, delta, eps, src.shape[0], _d(src), trg.shape[0], _d(trg),
                       ctypes.byref(lc), ctypes.byref(bs), _d(cen))
    return lc.value, bs.value, cen[:dim].copy()


_TREE_INT = ["laddr", "ilevel", "iparent", "nchild", "ichild", "nnbors", "nbors", "isrc",
             "isrcse", "itarg", "itargse"]


def tree(dim, delta, eps, sources, targ):
    """The restated reference tree (1-based ids) as a dict of numpy arrays."""
    src = _f64(sources)
    trg = _f64(targ)
    L = lib()
    h = L.orc_tree_build(dim, delta, eps, src.shape[0], _d(src), trg.shape[0], _d(trg))
    if not h:
        return None
    try:
        dims = np.zeros(4, dtype=np.int32)
        L.orc_tree_dims(h, dims.ctypes.data_as(_ip))
        out = {"dim": int(dims[0]), "nlevels": int(dims[1]), "nboxes": int(dims[2]),
               "npwlevel": int(dims[3])}
        for i, k in enumerate(_TREE_INT):
            n = L.orc_tree_int(h, i, None)
            a = np.zeros(n, dtype=np.int32)
            L.orc_tree_int(h, i, a.ctypes.data_as(_ip))
            out[k] = a
        for i, k in enumerate(["centers", "boxsize"]):
            n = L.orc_tree_dbl(h, i, None)
            a = np.zeros(n)
            L.orc_tree_dbl(h, i, _d(a))
            out[k] = a
        return out
    finally:
        L.orc_tree_free(h)


def reference_test_inputs_2d(nsrc, ntarg=None):
    """Inputs of 2d/planewave/test/test_fgt2d.f:66-114 (hkrand stream order kept)."""
    ntarg = nsrc if ntarg is None else ntarg
    r = hkrand(7 * nsrc, reset=True).reshape(nsrc, 7)  # thet, x, y, rn1, rn2, charge, dipstr
    src = r[:, 1:3].copy()
    chg = r[:, 5].copy()
    chg[0] = 0.0
    chg[1] = 0.0
    chg[2] = 1.0
    src[0] = (0.0, 0.0)
    src[1] = (1.0, 1.0)
    src[2] = (0.05, 0.05)
    trg = hkrand(2 * ntarg).reshape(ntarg, 2)
    bb = 1.0 / 2.0 ** 6
    delta = bb * bb / (1.5 * 1.5) * 2.0 ** -4
    return src, chg, trg, delta, 0.5e-10


def reference_test_inputs_3d(nsrc, ntarg=None):
    """Inputs of 3d/planewave/test/test_fgt3d.f:44-105 (hkrand stream order kept)."""
    ntarg = nsrc if ntarg is None else ntarg
    r = hkrand(10 * nsrc, reset=True).reshape(nsrc, 10)  # th, phi, x, y, z, rn*3, chg, dip
    src = r[:, 2:5].copy()
    chg = r[:, 8].copy()
    chg[0] = 0.0
    chg[1] = 0.0
    chg[2] = 1.0
    src[0] = (0.0, 0.0, 0.0)
    src[1] = (1.0, 1.0, 1.0)
    src[2] = (0.05, 0.05, 0.05)
    trg = hkrand(3 * ntarg).reshape(ntarg, 3)
    return src, chg, trg, 0.3e-3 * 4, 1e-6
