"""Generates the small golden fixtures under tests/golden/ from the oracle.

The reference (Fortran) cannot be built in this environment, so the fixtures
pin the oracle to itself across changes, on the reference test driver's own
inputs (hkrand stream, test_fgt2d.f:66-114 / test_fgt3d.f:44-105) scaled down,
together with the FP64 direct sum that the driver uses as its known answer.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def main():
    O.build()
    out = {}
    hk = O.hkrand(64, reset=True)
    out["hkrand_first64"] = hk
    src, q, trg, delta, eps = O.reference_test_inputs_2d(3000)
    pot, _, info = O.fgt(2, 1, delta, eps, src, q, trg, 1, 0)
    out["ref2d_pot_first20"] = pot[:20, 0]
    out["ref2d_direct_first20"] = O.direct(2, 1, delta, src, q, src[:20])[:, 0]
    out["ref2d_info"] = np.array([info["npwlevel"], info["nlevels"], info["nboxes"], info["npw"]])
    src, q, trg, delta, eps = O.reference_test_inputs_3d(3000)
    pot, _, info = O.fgt(3, 1, delta, eps, src, q, trg, 1, 0)
    out["ref3d_pot_first20"] = pot[:20, 0]
    out["ref3d_direct_first20"] = O.direct(3, 1, delta, src, q, src[:20])[:, 0]
    out["ref3d_info"] = np.array([info["npwlevel"], info["nlevels"], info["nboxes"], info["npw"]])
    # a plane-wave-path case: 2D uniform, delta 1e-4, eps 1e-9 (the 2D CPU config), 20000 points
    rng = np.random.default_rng(1235)
    s2, t2, c2 = rng.random((20000, 2)), rng.random((20000, 2)), rng.random(20000)
    p2, pt2, info = O.fgt(2, 1, 1e-4, 1e-9, s2, c2, t2, 1, 1)
    out["pw2d_pot_first50"] = p2[:50, 0]
    out["pw2d_pottarg_first50"] = pt2[:50, 0]
    out["pw2d_info"] = np.array([info["npwlevel"], info["nlevels"], info["nboxes"], info["npw"]])
    np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "oracle_golden.npz"))


if __name__ == "__main__":
    main()
