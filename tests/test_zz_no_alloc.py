"""cs_mst_noalloc: the MST entry point that allocates nothing.

Some callers cannot allocate device memory -- plugins whose host application owns
every device allocation, code that must not touch the allocation API -- so this
entry point takes the edge list and output buffers as the caller's device pointers
and keeps every intermediate in a fixed scratch array inside the library.  This test
checks, through the C ABI, that two calls in a row give exactly the tree, labels,
component count and weight of the allocating entry point (cs_extract), and that
sizes beyond the stated limits are rejected.  It runs last (file name) so a failure
here never hides another test; it passes alone and after the others.
"""
import ctypes as C

import numpy as np
import pytest

import coresg_b200 as cs
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _call(torch, edges, n, labels=True, stream=None):
    """Call cs_mst_noalloc on device copies of `edges` (numpy, cs_edge layout) on
    `stream` (a torch.cuda.Stream, or None for the default stream).  Returns the
    status and the device outputs."""
    d_u = _dev(torch, edges["u"].astype(np.int32))
    d_v = _dev(torch, edges["v"].astype(np.int32))
    d_w = _dev(torch, edges["w"].astype(np.float32))
    d_out = torch.zeros(max(n - 1, 1) * 3, dtype=torch.int32, device="cuda")
    d_lab = torch.zeros(n, dtype=torch.int32, device="cuda") if labels else None
    ne, nc, w = C.c_uint64(), C.c_uint32(), C.c_double()
    torch.cuda.synchronize()
    st = cs.lib().cs_mst_noalloc(C.c_void_p(d_u.data_ptr()), C.c_void_p(d_v.data_ptr()),
                                 C.c_void_p(d_w.data_ptr()), len(edges), n, C.c_void_p(d_out.data_ptr()),
                                 C.c_void_p(d_lab.data_ptr()) if labels else None, C.byref(ne), C.byref(nc),
                                 C.byref(w), C.c_void_p(stream.cuda_stream) if stream is not None else None)
    torch.cuda.synchronize()
    return st, d_out, d_lab, ne, nc, w


def _run_noalloc(torch, edges, n, labels=True, stream=None):
    st, d_out, d_lab, ne, nc, w = _call(torch, edges, n, labels, stream)
    assert st == cs.CS_OK, cs.lib().cs_last_error(None).decode()
    tree = d_out.cpu().numpy().view(cs.EDGE_DTYPE)[:ne.value]
    lab = d_lab.cpu().numpy().view(np.uint32) if labels else None
    return tree, lab, int(nc.value), float(w.value)


def test_noalloc_matches_allocating_entry_twice():
    torch = pytest.importorskip("torch")
    z = load_golden("coresg_n6000_d16_k32")
    ctx = cs.Context(0)
    g = cs.CoreSG(ctx, int(z["dim"]), int(z["k"]))
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    n = len(z["counts"])
    for m in (8, 2):  # two calls in a row on the shared scratch
        edges = g.edges(m)
        ref = g.mst(m)  # the allocating entry point (cs_extract)
        tree, lab, ncomp, w = _run_noalloc(torch, edges, n)
        assert tree.tobytes() == ref.edges.tobytes()  # bit-exact, as all extraction tests
        assert np.array_equal(lab, ref.component)
        assert ncomp == ref.num_components
        assert w == ref.weight


def test_noalloc_rejects_oversize_and_handles_forests():
    torch = pytest.importorskip("torch")
    st = cs.lib().cs_mst_noalloc(None, None, None, 0, 131073, None, None, None, None, None, None)
    assert st == cs.CS_ERR_INVALID
    assert "131072" in cs.lib().cs_last_error(None).decode()
    st = cs.lib().cs_mst_noalloc(None, None, None, 1048577, 100, None, None, None, None, None, None)
    assert st == cs.CS_ERR_INVALID
    # a forest: two disjoint paths plus isolated nodes, then a tiny graph reusing the scratch
    e = np.array([(0, 1, 1.0), (1, 2, 2.0), (0, 2, 2.0), (5, 6, 0.5)], cs.EDGE_DTYPE)
    tree, lab, ncomp, w = _run_noalloc(torch, e, 8)
    assert len(tree) == 3 and ncomp == 5 and w == 3.5
    assert list(lab) == [0, 0, 0, 1, 2, 3, 3, 4]
    tree, lab, ncomp, w = _run_noalloc(torch, e[:1], 2)
    assert len(tree) == 1 and ncomp == 1 and w == 1.0


def test_noalloc_without_labels_on_a_caller_stream():
    """No labels buffer, a stream the caller created: the tree, the component count
    and the weight still equal cs_extract's, twice in a row."""
    torch = pytest.importorskip("torch")
    z = load_golden("coresg_n3000_d24_k16")
    ctx = cs.Context(0)
    g = cs.CoreSG(ctx, int(z["dim"]), int(z["k"]))
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    n = len(z["counts"])
    stream = torch.cuda.Stream()
    for m in (4, 16):
        edges = g.edges(m)
        ref = g.mst(m)
        tree, lab, ncomp, w = _run_noalloc(torch, edges, n, labels=False, stream=stream)
        assert lab is None
        assert tree.tobytes() == ref.edges.tobytes()
        assert ncomp == ref.num_components and w == ref.weight


def test_noalloc_rejects_bad_edges():
    """An endpoint >= n, a negative weight and a NaN weight are each rejected with
    CS_ERR_INVALID and a message; a valid call afterwards still gives the right tree."""
    torch = pytest.importorskip("torch")
    good = np.array([(0, 1, 1.0), (1, 2, 2.0), (0, 2, 3.0)], cs.EDGE_DTYPE)
    cases = [(np.array([(0, 1, 1.0), (1, 3, 2.0)], cs.EDGE_DTYPE), "endpoint"),
             (np.array([(0, 1, 1.0), (1, 2, -2.0)], cs.EDGE_DTYPE), "negative"),
             (np.array([(0, 1, np.nan), (1, 2, 2.0)], cs.EDGE_DTYPE), "NaN")]
    for e, word in cases:
        st = _call(torch, e, 3)[0]
        assert st == cs.CS_ERR_INVALID
        assert word in cs.lib().cs_last_error(None).decode()
    tree, lab, ncomp, w = _run_noalloc(torch, good, 3)
    assert len(tree) == 2 and ncomp == 1 and w == 3.0 and list(lab) == [0, 0, 0]
    # +inf weights (an empty neighbourhood's core distance) are valid
    inf = np.array([(0, 1, np.inf), (1, 2, 2.0)], cs.EDGE_DTYPE)
    tree, lab, ncomp, w = _run_noalloc(torch, inf, 3)
    assert len(tree) == 2 and ncomp == 1 and w == np.inf
