"""Failure paths, made on the host or by a bounded wait, never by a GPU fault:

* a grid-barrier wait of the persistent sweep kernel runs out (block 0 holds back
  before its first barrier for longer than the other blocks may wait): the sweep
  returns CS_ERR_TIMEOUT, and the same graph and context then sweep normally with
  the same trees as before;
* device allocations fail by injection (cs_test_fail_device_allocs) at several
  points of a build: each call returns CS_ERR_OOM, nothing crashes, and builds
  afterwards on the same context equal the oracle's;
* the serving loop refuses queries and inserts whose memory does not fit under its
  reserve (admission by free HBM) with CS_ERR_OOM per request, and a server with a
  normal reserve on the same graph then serves them.
The reference records OOM as a job result (src/cuda_backend.cpp:88-103)."""
import numpy as np
import pytest

import coresg_b200 as cs
from conftest import load_golden
from coresg_b200.serving import Pinned, Server

pytestmark = pytest.mark.gpu

NO_INJECTION = 2 ** 64 - 1


def resident(ctx, z):
    g = cs.CoreSG(ctx, int(z["dim"]), int(z["k"]))
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    return g


def same_results(a, b):
    for x, y in zip(a, b):
        assert x.edges.tobytes() == y.edges.tobytes()
        assert np.array_equal(x.component, y.component)
        assert x.num_components == y.num_components and x.weight == y.weight


def test_sweep_barrier_timeout_leaves_graph_and_context_usable(gpu_ctx):
    z = load_golden("coresg_n6000_d16_k32")
    g = resident(gpu_ctx, z)
    mp = [1, 8, 16, 32]
    before = g.all_msts(mp)
    # barrier waits limited to 0.2 ms while block 0 arrives 20 ms late
    gpu_ctx.check(cs.lib().cs_test_sweep_barrier(g.h, 200_000, 20_000_000))
    with pytest.raises(cs.CsError) as e:
        g.all_msts(mp)
    assert e.value.status == cs.CS_ERR_TIMEOUT
    assert "barrier" in str(e.value)
    # the default limit again: the same graph sweeps to the same trees
    gpu_ctx.check(cs.lib().cs_test_sweep_barrier(g.h, 0, 0))
    same_results(g.all_msts(mp), before)
    same_results([g.mst(m) for m in mp], before)
    # a hold below the limit is only a delay
    gpu_ctx.check(cs.lib().cs_test_sweep_barrier(g.h, 0, 1_000_000))
    same_results(g.all_msts(mp), before)
    gpu_ctx.check(cs.lib().cs_test_sweep_barrier(g.h, 0, 0))


def test_injected_allocation_failures_return_oom(gpu_ctx, oracle):
    z = load_golden("coresg_n3000_d24_k16")
    d, k = int(z["dim"]), int(z["k"])
    # the first allocation of a fresh graph fails; a retry on the same graph builds
    g = cs.CoreSG(gpu_ctx, d, k)
    cs.lib().cs_test_fail_device_allocs(0)
    try:
        with pytest.raises(cs.CsError) as e:
            g.set_points(z["points"])
        assert e.value.status == cs.CS_ERR_OOM and "injected" in str(e.value)
    finally:
        cs.lib().cs_test_fail_device_allocs(NO_INJECTION)
    st = g.build(z["points"])
    ids, dists, flags, counts = g.knn()
    br, nsel, _ = oracle.bridges(z["padded"], d, ids, dists, counts)
    assert st["selected"] == nsel and g.missing_edges().tobytes() == br.tobytes()
    g.close()
    # failures later in a build (the descent's, the selection's, the sweep's scratch):
    # each build stops with CS_ERR_OOM; a fresh graph on the same context then builds
    # and sweeps normally
    failed = 0
    for after in (3, 8, 14, 20, 26):
        h = cs.CoreSG(gpu_ctx, d, k)
        cs.lib().cs_test_fail_device_allocs(after)
        try:
            h.build(z["points"])
            h.all_msts([2, 16])
        except cs.CsError as ex:
            assert ex.status == cs.CS_ERR_OOM, str(ex)
            failed += 1
        finally:
            cs.lib().cs_test_fail_device_allocs(NO_INJECTION)
        h.close()
    assert failed >= 3
    h = cs.CoreSG(gpu_ctx, d, k)
    h.build(z["points"])
    ids, dists, flags, counts = h.knn()
    br, _, _ = oracle.bridges(z["padded"], d, ids, dists, counts)
    assert h.missing_edges().tobytes() == br.tobytes()
    for m, r in zip((2, 16), h.all_msts([2, 16])):
        e = oracle.edges(m, ids, dists, counts, br)
        o = oracle.mst(e, len(counts))
        assert r.edges.tobytes() == e[o["in_tree"]].tobytes()


def test_server_admission_rejects_what_does_not_fit(gpu_ctx):
    z = load_golden("coresg_n3000_d24_k16")
    g = cs.CoreSG(gpu_ctx, int(z["dim"]), int(z["k"]))
    g.build(z["points"])
    n = g.n
    out = Pinned((n,), cs.EDGE_DTYPE)
    rows = z["points"][:50] + np.float32(0.01)
    # a reserve larger than any GPU's memory: nothing is admitted
    srv = Server(g, reserve_bytes=1 << 60)
    try:
        r = srv.wait(srv.extract(4, out.array))
        assert r["status"] == cs.CS_ERR_OOM and "not admitted" in r["error"]
        r = srv.wait(srv.insert(rows))
        assert r["status"] == cs.CS_ERR_OOM and "not admitted" in r["error"]
        st = srv.stats()
        assert st["failed"] == 2 and st["inserted_rows"] == 0
    finally:
        srv.close()
    assert g.n == n
    # the default reserve on the same graph serves both
    srv = Server(g)
    try:
        r = srv.wait(srv.extract(4, out.array))
        assert r["status"] == 0
        want = g.mst(4)
        assert out.array[:r["nedges"]].tobytes() == want.edges.tobytes() and r["weight"] == want.weight
        r = srv.wait(srv.insert(rows))
        assert r["status"] == 0
    finally:
        srv.close()
        out.free()
    assert g.n == n + len(rows)
