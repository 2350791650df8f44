"""Incremental insertion on the device (cs_insert) against the reference's own
CoreSG::insert on the same base set and batches (half from existing clusters, half from
new ones, as the insertion workload): new-point and overall recall at least the
reference's (minus the sampling tolerance), KnnGraph invariants, and bridges bit-exact
against the oracle's bridge computation on the resulting graph."""
import numpy as np
import pytest

import coresg_b200 as cs
from checkers import Reference
from coresg_b200.datagen import gaussian_mixture, pad_rows
from test_knn_gpu import validate

pytestmark = pytest.mark.gpu


def workload(seed=31, n=16000, d=16, clusters=12, batch=2500):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, 10, size=(clusters, d))
    base = gaussian_mixture(n, d, clusters, (0.2, 1.0), 0.03, seed=seed + 1, centres=centres)
    old = gaussian_mixture(batch, d, clusters, (0.2, 1.0), 0.0, seed=seed + 2, centres=centres)
    fresh = gaussian_mixture(batch, d, 3, (0.2, 1.0), 0.0, seed=seed + 3)
    return base, [old, fresh]


def recall(oracle, padded, ids, k, queries):
    truth, _ = oracle.brute_knn(padded, k, queries)
    return float(np.mean([len(np.intersect1d(truth[t], ids[q])) / k for t, q in enumerate(queries)]))


@pytest.mark.skipif(not Reference.available(), reason="reference not built (oracle/_ref)")
def test_insert_recall_at_least_reference(gpu_ctx, oracle):
    k = 24
    base, batches = workload()
    allpts = np.concatenate([base] + batches)
    padded = pad_rows(allpts)
    n0 = len(base)
    # engine
    g = cs.CoreSG(gpu_ctx, base.shape[1], k)
    g.build(base)
    for b in batches:
        st = g.insert(b)
        assert st["active"] >= len(b)
    ids, dists, flags, counts = g.knn()
    validate(ids, dists, counts, len(allpts), k)
    # reference, same data
    ref = Reference()
    sg = ref.build(base, k_max=k, instances=1, iters=10, sample=16, seed=42, threads=8)
    for b in batches:
        sg.insert(b)
    rids = sg.knn()[0]
    rng = np.random.default_rng(3)
    q_new = rng.choice(np.arange(n0, len(allpts)), 800, replace=False).astype(np.uint32)
    q_all = rng.choice(len(allpts), 800, replace=False).astype(np.uint32)
    mine_new, ref_new = recall(oracle, padded, ids, k, q_new), recall(oracle, padded, rids, k, q_new)
    mine_all, ref_all = recall(oracle, padded, ids, k, q_all), recall(oracle, padded, rids, k, q_all)
    print(f"new-point recall {mine_new:.4f} (reference {ref_new:.4f}); overall {mine_all:.4f} (reference {ref_all:.4f})")
    assert mine_new >= ref_new - 0.01
    assert mine_all >= ref_all - 0.01
    # stored distances are the reference arithmetic
    for p in range(0, len(allpts), 211):
        for j in range(int(counts[p])):
            assert oracle.dist(padded[p], padded[ids[p, j]]).view(np.uint32) == dists[p, j].view(np.uint32)
    # the bridges re-selected after the last batch are the oracle's for this graph
    br, nsel, nrep = oracle.bridges(padded, base.shape[1], ids, dists, counts)
    assert g.missing_edges().tobytes() == br.tobytes()


def test_insert_requires_a_built_graph(gpu_ctx):
    g = cs.CoreSG(gpu_ctx, 8, 8)
    with pytest.raises(cs.CsError):
        g.insert(np.zeros((10, 8), np.float32))


def test_inserts_within_a_reserve_allocate_nothing(gpu_ctx, oracle):
    """cs_graph_reserve for every row to come, then inserts of four sizes (the largest
    last): the library makes no device allocation during them (cs_device_allocs), and
    the graph they leave keeps the KnnGraph invariants and carries the oracle's
    bridges for it."""
    k = 24
    base, (old, fresh) = workload(seed=47, n=12000, batch=1500)
    d = base.shape[1]
    big = gaussian_mixture(4000, d, 4, (0.2, 1.0), 0.0, seed=101)
    batches = [old[:200], old[200:], fresh, big]
    g = cs.CoreSG(gpu_ctx, d, k)
    g.build(base)
    g.reserve(len(base) + sum(len(b) for b in batches))
    before = cs.device_allocs()
    for b in batches:
        g.insert(b)
    after = cs.device_allocs()
    assert after == before, f"{after[0] - before[0]} device allocations ({after[1] - before[1]} bytes) in the inserts"
    allpts = np.concatenate([base] + batches)
    ids, dists, flags, counts = g.knn()
    validate(ids, dists, counts, len(allpts), k)
    br, _, _ = oracle.bridges(pad_rows(allpts), d, ids, dists, counts)
    assert g.missing_edges().tobytes() == br.tobytes()


def test_incremental_hubness_matches_full_after_every_batch(gpu_ctx, oracle):
    """The bridge re-selection after an insert refreshes the hubness incrementally
    (HubnessIndex::refresh, src/hubness.cpp:523-544) when few lists changed: the
    reverse-degree deltas of the changed lists, and only the nodes whose score inputs
    moved rescored; after a large insert a full pass.  After every batch -- small ones
    that take the refresh, a large one that takes the full pass -- the selection (order
    included) and the bridges equal a full pass on the same k-NN graph (a fresh graph
    given the same arrays) and the oracle's bridge computation."""
    k = 16
    base, (old, fresh) = workload(seed=53, n=20000, batch=3000)
    d = base.shape[1]
    batches = [old[:40], fresh[:60], old[40:70], fresh[60:110], old[100:3100], fresh[200:250]]
    g = cs.CoreSG(gpu_ctx, d, k)
    g.build(base)
    st = g.bridge_stats()
    assert st["hub_refreshed"] == 0 and st["rescored"] == len(base)
    pts = base
    refreshed = 0
    for b in batches:
        g.insert(b)
        pts = np.concatenate([pts, b])
        n = len(pts)
        st = g.bridge_stats()
        # the rule: the refresh when at most n / 16 lists changed
        assert st["hub_refreshed"] == int(st["changed"] * 16 <= n)
        if st["hub_refreshed"]:
            refreshed += 1
            assert 0 < st["rescored"] < n
        else:
            assert st["rescored"] == n
        ids, dists, flags, counts = g.knn()
        h = cs.CoreSG(gpu_ctx, d, k)
        h.set_points(pts)
        h.set_knn(ids, dists, flags, counts)
        h.select_bridges()
        assert h.bridge_stats()["hub_refreshed"] == 0
        assert np.array_equal(g.selected(), h.selected())
        assert g.missing_edges().tobytes() == h.missing_edges().tobytes()
        br, _, _ = oracle.bridges(pad_rows(pts), d, ids, dists, counts)
        assert g.missing_edges().tobytes() == br.tobytes()
        h.close()
    assert refreshed >= 3, "the small batches should have taken the refresh"
    # replacing the k-NN arrays starts over with a full pass
    g.set_knn(*g.knn())
    g.select_bridges()
    assert g.bridge_stats()["hub_refreshed"] == 0
