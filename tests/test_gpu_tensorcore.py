"""The tcgen05 tensor-core path of the mixed form.

* The BF16 x 3 compensated tile (three exact BF16 pieces per operand, the six
  piece products of order <= 2 accumulated in FP32 in TMEM) against an FP64
  product: FP32-level agreement for every N the kernels use.
* The mixed 3D form (tcgen05 Taylor evaluation, FP32 near field; the
  tcgen05 Hermite blocks too with FGT_FORM3D_TC set, else the FP64 blocks)
  against the FP64 form on the same inputs: the difference is rounding of
  FP32 size (~1e-7), well below eps, and no bounded wait of a tensor-core
  kernel gave up.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [16, 32, 112, 176, 256])
def test_bf16x3_tile_matches_fp64(fgt, n):
    err = ctypes.c_double()
    st = fgt.lib().fgt_tc_selftest(0, n, ctypes.byref(err))
    assert st == 0, st
    print(f"N={n}: max error / max entry {err.value:.3e}")
    assert err.value <= 2e-7, err.value


@pytest.mark.parametrize("delta,n", [(1e-3, 60000), (1e-2, 30000)])
@pytest.mark.parametrize("tc_form", [False, True])
def test_mixed_3d_eval_matches_fp64(fgt, oracle, delta, n, tc_form, monkeypatch):
    if tc_form:
        monkeypatch.setenv("FGT_FORM3D_TC", "1")
    rng = np.random.default_rng(77)
    src = rng.random((n, 3))
    trg = rng.random((n // 2, 3))
    q = 2 * rng.random(n) - 1
    eps = 1e-6
    out = {}
    for prec in ("fp64", "mixed"):
        ctx = fgt.Context(0, precision=prec)
        out[prec] = fgt.transform(3, 1, delta, eps, src, q, trg, 1, 1, ctx=ctx)
    flag = ctypes.c_int()
    assert fgt.lib().fgt_tc_error(0, 1, ctypes.byref(flag)) == 0
    assert flag.value == 0
    for k in range(2):
        d = oracle.derr(out["fp64"][k], out["mixed"][k])
        print(f"delta={delta} {'pot' if k == 0 else 'pottarg'}: mixed vs fp64 {d:.3e}")
        assert d <= 0.3 * eps, d
    idx = rng.choice(trg.shape[0], 300, replace=False)
    ex = oracle.direct(3, 1, delta, src, q, trg[idx])
    e_mixed = oracle.derr(ex, out["mixed"][1][idx])
    e_fp64 = oracle.derr(ex, out["fp64"][1][idx])
    print(f"vs direct: fp64 {e_fp64:.3e} mixed {e_mixed:.3e}")
    assert e_mixed <= max(eps, e_fp64 + 0.1 * eps)
