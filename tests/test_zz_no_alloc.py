"""The allocation-free large-delta call (fgt_large_delta_noalloc).

It serves callers that must not have the library allocate device memory --
codes that pass device arrays from their own pool under a fixed budget, and
latency-critical loops that cannot afford cudaMalloc, which can synchronise
the device.  Its scratch is one fixed device array shared by all calls.  The
test drives it through the C ABI with device arrays the test owns and checks
two calls in a row against the oracle (the restated reference, whose driver
takes the same large-delta path for these inputs) and against the allocating
drop-in (fgt_transform), at the FP64 parity tolerance of the other GPU tests.
The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # FP64 relative l2 against the oracle and the allocating path


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _run(fgt, oracle, dim, nd, ns, nt, ifpgh, ifpghtarg, stream, seed):
    import torch
    rng = np.random.default_rng(seed)
    delta, eps = 10.0, 1e-6
    src = rng.random((max(ns, 1), dim))[:ns]
    trg = rng.random((nt, dim))
    q = rng.random((ns, nd))
    # the driver's large-delta parameters (fgt2d.f:125-135): box centre and
    # nlocal = hlterms(dim, bs0) + max(ifpgh, ifpghtarg) - 1
    lev, bs0, cen = oracle.boxsize0(dim, delta, eps, src if ns else trg, trg)
    assert lev < -2
    nlocal = oracle.hlterms(dim, bs0, delta, eps) + max(ifpgh, ifpghtarg) - 1
    center = np.ascontiguousarray(cen, dtype=np.float64)
    dev = torch.device("cuda", 0)
    d_src = torch.from_numpy(src).to(dev) if ns else None
    d_q = torch.from_numpy(q).to(dev) if ns else None
    d_trg = torch.from_numpy(trg).to(dev) if nt else None
    L = fgt.lib()
    outs = []
    for call in range(2):
        d_pot = torch.full((max(ns, 1), nd), float("nan"), dtype=torch.float64, device=dev)
        d_pt = torch.full((max(nt, 1), nd), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        st = L.fgt_large_delta_noalloc(dim, nd, delta, ns, _ptr(d_src), _ptr(d_q), nlocal,
                                       center.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       ifpgh, _ptr(d_pot), nt, _ptr(d_trg), ifpghtarg, _ptr(d_pt), sp)
        assert st == 0, st
        if stream is not None:
            stream.synchronize()
        else:
            torch.cuda.synchronize()
        outs.append((d_pot.cpu().numpy()[:ns], d_pt.cpu().numpy()[:nt]))
    return src, q, trg, delta, eps, outs


@pytest.mark.parametrize("dim,nd,ifpgh,ifpghtarg,on_stream", [
    (2, 1, 1, 1, False), (2, 2, 1, 1, False), (3, 1, 1, 1, False),
    (2, 1, 1, 0, False), (3, 1, 0, 1, False), (2, 1, 1, 1, True), (3, 2, 1, 1, True)])
def test_noalloc_matches_oracle(fgt, oracle, dim, nd, ifpgh, ifpghtarg, on_stream):
    import torch
    stream = torch.cuda.Stream() if on_stream else None
    ns, nt = 3000, 2000
    src, q, trg, delta, eps, outs = _run(fgt, oracle, dim, nd, ns, nt, ifpgh, ifpghtarg, stream,
                                         40 + dim + nd + 2 * ifpgh + ifpghtarg)
    opot, opt, info = oracle.fgt(dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg)
    ctx = fgt.Context(0, precision="fp64")
    rpot, rpt = fgt.transform(dim, nd, delta, eps, src, q, trg, ifpgh, ifpghtarg, ctx=ctx)
    for call, (pot, pt) in enumerate(outs):
        if ifpgh:
            assert oracle.derr(opot, pot) <= TOL, (call, oracle.derr(opot, pot))
            assert oracle.derr(rpot, pot) <= TOL, call
        else:  # the untouched output keeps the sentinel
            assert np.all(np.isnan(pot)), call
        if ifpghtarg:
            assert oracle.derr(opt, pt) <= TOL, (call, oracle.derr(opt, pt))
            assert oracle.derr(rpt, pt) <= TOL, call
        else:
            assert np.all(np.isnan(pt)), call


def test_noalloc_no_sources_gives_zero(fgt, oracle):
    """ns = 0: the shared array is cleared by each call, so the targets'
    potentials are exactly zero even after an earlier call left a local
    expansion in it."""
    _run(fgt, oracle, 2, 1, 3000, 100, 1, 1, None, 7)  # leaves a non-zero local behind
    _, _, _, _, _, outs = _run(fgt, oracle, 2, 1, 0, 500, 0, 1, None, 8)
    for _, pt in outs:
        assert np.all(pt == 0.0)


def test_noalloc_rejects_oversized_expansions(fgt):
    import torch
    dev = torch.device("cuda", 0)
    x = torch.zeros((10, 3), dtype=torch.float64, device=dev)
    q = torch.ones((10, 1), dtype=torch.float64, device=dev)
    out = torch.full((10, 1), 7.0, dtype=torch.float64, device=dev)
    center = np.zeros(3)
    st = fgt.lib().fgt_large_delta_noalloc(3, 1, 10.0, 10, _ptr(x), _ptr(q), 60,
                                           center.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           1, _ptr(out), 0, None, 0, None, None)
    assert st == 6
    assert torch.all(out == 7.0)
