"""The reference-side binding of the engine, compiled: tests/binding/b200_backend.cpp
(the B200Backend and the extraction hook that INTEGRATION.md shows) built against the
reference's own headers and objects by oracle/Makefile (target `binding`).

CPU: the binding library exists, loads (resolving libcoresg_b200.so) and exports its
entry points.  GPU: one KnnJob through the reference's JobScheduler onto
B200Backend::run_knn_job reaches the reference NN-Descent's recall with the
reference's distances; JobScheduler::mrd_matrix through B200Backend::mrd_block equals
the oracle's dense MRD; and MSTs of a CORE-SG read by the reference's CoreSG::load,
extracted through the hook, equal the C-ABI path (cs_extract) and CoreSG::mst."""
import ctypes as C
import os

import numpy as np
import pytest

import coresg_b200 as cs
from checkers import EDGE_DTYPE, Reference
from conftest import edge_keys, load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINDING = os.path.join(ROOT, "oracle", "_ref", "libb200_binding.so")
needs_binding = pytest.mark.skipif(not os.path.exists(BINDING), reason="binding not built (oracle/Makefile binding)")


def binding():
    lib = C.CDLL(BINDING)
    p, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
    lib.bb_last_error.restype = C.c_char_p
    lib.bb_knn_job.argtypes = [p, u64, u32, u32, u32, u32, u64, C.c_int, C.c_int, p, p, p, p, p]
    lib.bb_mrd_matrix.argtypes = [p, u64, u32, u32, p, C.c_int, p]
    lib.bb_extract.argtypes = [C.c_char_p, p, u32, C.c_int, C.c_int, p, p, p, p, p]
    return lib


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


@needs_binding
def test_binding_library_loads_and_exports():
    lib = binding()
    for name in ("bb_knn_job", "bb_mrd_matrix", "bb_extract", "bb_last_error"):
        assert hasattr(lib, name)
    # the binding resolved the engine's library, whose C ABI it calls
    maps = open("/proc/self/maps").read()
    assert "libcoresg_b200.so" in maps


@needs_binding
@pytest.mark.gpu
def test_knn_job_through_job_scheduler(oracle):
    from coresg_b200.datagen import gaussian_mixture, pad_rows

    lib = binding()
    pts = gaussian_mixture(12000, 16, 8, (0.2, 1.0), 0.05, seed=71)
    n, k = len(pts), 16
    ids = np.empty((n, k), np.uint32)
    dists = np.empty((n, k), np.float32)
    counts = np.empty(n, np.uint32)
    oom, cuda = C.c_int(), C.c_int()
    rc = lib.bb_knn_job(ptr(pts), n, 16, k, 8, 10, 42, 0, 0, ptr(ids), ptr(dists), ptr(counts), C.byref(oom),
                        C.byref(cuda))
    assert rc == 0, lib.bb_last_error().decode()
    assert oom.value == 0 and cuda.value == 1  # KnnJob::ran_on says the device ran it
    padded = pad_rows(pts)
    q = np.random.default_rng(9).choice(n, 1000, replace=False).astype(np.uint32)
    truth, _ = oracle.brute_knn(padded, k, q)
    rec = np.mean([len(np.intersect1d(truth[t], ids[v])) / k for t, v in enumerate(q)])
    rids = Reference().nndescent(pts, k=k, sample=8, iters=10, seed=42)[0] if Reference.available() else None
    if rids is not None:
        ref = np.mean([len(np.intersect1d(truth[t], rids[v])) / k for t, v in enumerate(q)])
        assert rec >= ref - 0.005
    assert rec > 0.95
    for v in range(0, n, 101):
        for j in range(int(counts[v])):
            assert oracle.dist(padded[v], padded[ids[v, j]]).view(np.uint32) == dists[v, j].view(np.uint32)


@needs_binding
@pytest.mark.gpu
def test_mrd_matrix_through_job_scheduler(oracle):
    lib = binding()
    z = load_golden("coresg_n2000_d40_k10")
    sel = z["selected"][:150]
    pts = np.ascontiguousarray(z["padded"][sel])
    core = np.ascontiguousarray(oracle.core(z["dists"], z["counts"], int(z["k"]))[sel])
    m = len(sel)
    out = np.empty((m, m), np.float32)
    rc = lib.bb_mrd_matrix(ptr(pts), m, 40, pts.shape[1], ptr(core), 0, ptr(out))
    assert rc == 0, lib.bb_last_error().decode()
    assert np.array_equal(out.view(np.uint32), oracle.mrd_block(pts, core).view(np.uint32))


@needs_binding
@pytest.mark.gpu
def test_extraction_hook_on_a_loaded_coresg(gpu_ctx, tmp_path):
    lib = binding()
    z = load_golden("coresg_n6000_d16_k32")
    g = cs.CoreSG(gpu_ctx, int(z["dim"]), int(z["k"]))
    g.set_points(z["points"])
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    path = str(tmp_path / "g.coresg")
    g.save(path)  # CORESG01, read back by the reference's CoreSG::load inside the binding
    n = len(z["counts"])
    mp = np.array([1, 4, 16, 32], np.uint32)
    K = len(mp)
    sg = Reference().from_state(z["padded"], int(z["dim"]), z["ids"], z["dists"], z["flags"], z["counts"],
                                z["bridges"]) if Reference.available() else None
    for all_ in (0, 1):
        edges = np.zeros((K, n - 1), EDGE_DTYPE)
        labels = np.zeros((K, n), np.uint32)
        ne, nc, w = np.zeros(K, np.uint64), np.zeros(K, np.uint32), np.zeros(K, np.float64)
        rc = lib.bb_extract(path.encode(), ptr(mp), K, all_, 0, ptr(edges), ptr(labels), ptr(ne), ptr(nc), ptr(w))
        assert rc == 0, lib.bb_last_error().decode()
        for j, m in enumerate(mp):
            mine = g.mst(int(m))  # the C-ABI path
            assert edges[j, :ne[j]].tobytes() == mine.edges.tobytes()
            assert np.array_equal(labels[j], mine.component)
            assert nc[j] == mine.num_components and w[j] == mine.weight
            if sg is not None:
                r = sg.mst(int(m))
                assert np.array_equal(edge_keys(edges[j, :ne[j]]), edge_keys(r["edges"]))
                assert np.array_equal(labels[j], r["labels"])
