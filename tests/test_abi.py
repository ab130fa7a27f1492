"""The C-ABI library loads without a GPU and exports every function that
include/fgt_b200.h declares; host-only entry points validate arguments."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "fgt_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*[\s\*]+([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                       txt, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "return")))


def test_header_declares_the_drop_ins():
    names = declared_functions()
    for n in ("fgt2d_", "fgt3d_", "fgt2dmain_gpu_", "fgt3dmain_gpu_", "fgt_transform",
              "fgt_plan_create", "fgt_plan_execute_device"):
        assert n in names


def test_library_exports_every_declared_symbol(fgt):
    lib = ctypes.CDLL(fgt.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(fgt):
    L = fgt.lib()
    assert L.fgt_status_string(0) == b"ok"
    assert L.fgt_status_string(2) == b"unsupported option"


def test_host_tree_rejects_bad_arguments(fgt):
    with pytest.raises(fgt.FGTError) as e:
        fgt.HostTree(2, -1.0, 1e-6, np.random.rand(10, 2), np.random.rand(5, 2))
    assert e.value.status == 1
    with pytest.raises(fgt.FGTError) as e:
        fgt.HostTree(2, 1e-3, 1.5, np.random.rand(10, 2), np.random.rand(5, 2))
    assert e.value.status == 1
    bad = np.random.rand(10, 2)
    bad[3, 1] = np.inf
    with pytest.raises(fgt.FGTError) as e:
        fgt.HostTree(2, 1e-3, 1e-6, bad, bad)
    assert e.value.status == 1


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_is_reported(fgt):
    with pytest.raises(fgt.FGTError) as e:
        fgt.Context(0)
    assert e.value.status == 5


def test_oracle_library_loads(oracle):
    assert oracle.hlterms(2, 0.01, 1e-4, 1e-6) > 0
