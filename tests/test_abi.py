"""CPU tests of the C ABI: the library loads, exports every function that
include/coresg_b200.h declares, and reports "no device" cleanly without a GPU."""
import ctypes as C
import os

import pytest

import coresg_b200 as cs
from coresg_b200 import _abi


def test_library_builds_and_loads():
    assert os.path.exists(cs.LIB_PATH), "run __graft_entry__.build() first"
    cs.lib()


def test_every_header_symbol_is_exported():
    syms = cs.header_symbols()
    assert len(syms) >= 25
    L = C.CDLL(cs.LIB_PATH)
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, f"declared but not exported: {missing}"
    # and the binding covers every declared function
    assert set(syms) == set(_abi._SIGS), set(syms) ^ set(_abi._SIGS)


def test_no_gpu_is_reported_not_crashed():
    n = cs.device_count()
    if n > 0:
        pytest.skip("a device is visible")
    with pytest.raises(cs.CsError):
        cs.Context(0)
    assert cs.lib().cs_last_error(None)


def test_null_context_is_invalid():
    st = cs.lib().cs_graph_create(None, 8, 8, 0, C.byref(C.c_void_p()))
    assert st == cs.CS_ERR_INVALID
