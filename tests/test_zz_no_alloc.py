"""The allocation-free large-delta call (fgt_large_delta_noalloc).

It serves callers that must not have the library allocate device memory --
codes that pass device arrays from their own pool under a fixed budget, and
latency-critical loops that cannot afford cudaMalloc, which can synchronise
the device.  Its scratch is one fixed device array shared by all calls.  The
test drives it through the C ABI with device arrays the test owns and checks
two calls in a row against the allocating drop-in (fgt_transform), which takes
the same large-delta path for these inputs, at the FP64 parity tolerance of
the other GPU tests.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("dim,nd", [(2, 1), (2, 2), (3, 1)])
def test_noalloc_matches_allocating_path(fgt, oracle, dim, nd):
    import torch
    rng = np.random.default_rng(40 + dim + nd)
    delta, eps, ns, nt = 10.0, 1e-6, 3000, 2000
    src = rng.random((ns, dim))
    trg = rng.random((nt, dim))
    q = rng.random((ns, nd))
    ctx = fgt.Context(0, precision="fp64")
    pot_ref, pt_ref = fgt.transform(dim, nd, delta, eps, src, q, trg, 1, 1, ctx=ctx)
    # the driver's large-delta parameters (fgt2d.f:125-135): box centre and
    # nlocal = hlterms(dim, bs0) + max(ifpgh, ifpghtarg) - 1
    lev, bs0, cen = oracle.boxsize0(dim, delta, eps, src, trg)
    assert lev < -2
    nlocal = oracle.hlterms(dim, bs0, delta, eps)
    center = np.ascontiguousarray(cen, dtype=np.float64)
    dev = torch.device("cuda", 0)
    d_src = torch.from_numpy(src).to(dev)
    d_q = torch.from_numpy(q).to(dev)
    d_trg = torch.from_numpy(trg).to(dev)
    L = fgt.lib()
    for call in range(2):
        d_pot = torch.full((ns, nd), float("nan"), dtype=torch.float64, device=dev)
        d_pt = torch.full((nt, nd), float("nan"), dtype=torch.float64, device=dev)
        st = L.fgt_large_delta_noalloc(dim, nd, delta, ns, _ptr(d_src), _ptr(d_q), nlocal,
                                       center.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       1, _ptr(d_pot), nt, _ptr(d_trg), 1, _ptr(d_pt), None)
        assert st == 0, st
        torch.cuda.synchronize()
        pot, pt = d_pot.cpu().numpy(), d_pt.cpu().numpy()
        assert oracle.derr(pot_ref, pot) <= 1e-2 * eps, call
        assert oracle.derr(pt_ref, pt) <= 1e-2 * eps, call


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
