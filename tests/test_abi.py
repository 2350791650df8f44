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


def test_server_structs_match_the_header_layout():
    """ctypes mirrors of the serving structs have the C layout of coresg_b200.h
    (natural alignment on x86-64)."""
    import ctypes as C

    from coresg_b200.serving import Request, Result, ServerConfig, Stats

    assert C.sizeof(Request) == 72 and Request.eps.offset == 8 and Request.out_labels_cap.offset == 64
    assert C.sizeof(Result) == 216 and Result.weight.offset == 24 and Result.error.offset == 56
    assert C.sizeof(ServerConfig) == 104 and ServerConfig.insert.offset == 24
    assert C.sizeof(Stats) == 112 and Stats.sweep_ms.offset == 88 and Stats.reused_batches.offset == 104


def test_request_stream_is_seeded_and_shaped():
    from coresg_b200.serving import CS_REQ_EPS_LABELS, CS_REQ_INSERT, request_stream

    a = request_stream(20.0, 200.0, 32, seed=9)
    b = request_stream(20.0, 200.0, 32, seed=9)
    assert a == b
    assert 3600 < len(a) < 4400  # Poisson(4000)
    ins = [x for x in a if x.kind == CS_REQ_INSERT]
    cuts = [x for x in a if x.kind == CS_REQ_EPS_LABELS]
    assert 0.07 < len(ins) / len(a) < 0.13
    assert all(1_000 <= x.size <= 100_000 for x in ins)
    assert all(1 <= x.mpts <= 32 for x in a if x.kind != CS_REQ_INSERT)
    assert 0.18 < len(cuts) / (len(a) - len(ins)) < 0.32
    assert all(a[i].t < a[i + 1].t for i in range(len(a) - 1))
