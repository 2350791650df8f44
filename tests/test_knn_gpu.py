"""GPU NN-Descent: recall at or above the reference NN-Descent's at equal iterations
(the reference's exhaustive recall is stored in tests/golden/recall_*.npz), the
KnnGraph invariants (src/knn_graph.cpp:237-273), and stored distances equal to the
reference's metric_distance bit for bit."""
import numpy as np
import pytest

import coresg_b200 as cs
from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu


def validate(ids, dists, counts, n, k):
    """KnnGraph::validate: sorted, no self loop, no duplicate, valid ids in range."""
    for p in range(n):
        c = int(counts[p])
        assert c <= k
        row = ids[p, :c]
        assert not np.any(row == p), f"self loop at {p}"
        assert not np.any(row == 0xFFFFFFFF)
        assert len(np.unique(row)) == c, f"duplicate at {p}"
        assert np.all(np.diff(dists[p, :c]) >= 0), f"unsorted at {p}"
        assert np.all(ids[p, c:] == 0xFFFFFFFF) and np.all(np.isinf(dists[p, c:]))


def sampled_recall(oracle, padded, ids, k, queries):
    truth, _ = oracle.brute_knn(padded, k, queries)
    hits = 0
    for t, q in enumerate(queries):
        hits += len(np.intersect1d(truth[t], ids[q]))
    return hits / (len(queries) * k)


@pytest.mark.parametrize("name", golden_names("recall_"))
def test_recall_at_least_reference(gpu_ctx, oracle, name):
    z = load_golden(name)
    pts, padded = z["points"], z["padded"]
    n, k = len(pts), int(z["k"])
    g = cs.CoreSG(gpu_ctx, pts.shape[1], k)
    g.set_points(pts)
    st = g.build_knn(sample=int(z["sample"]), iters=int(z["iters"]), delta=0.001, seed=42)
    assert 1 <= st["rounds"] <= int(z["iters"])
    ids, dists, flags, counts = g.knn()
    validate(ids, dists, counts, n, k)
    q = np.random.default_rng(5).choice(n, 2000, replace=False).astype(np.uint32)
    rec = sampled_recall(oracle, padded, ids, k, q)
    ref = float(np.min(z["ref_recall"]))
    # 2000 sampled queries: standard error ~0.0005 at this recall
    assert rec >= ref - 0.003, f"recall {rec:.4f} below the reference's {ref:.4f}"
    # stored distances are the reference arithmetic, bit for bit
    for p in range(0, n, 97):
        for j in range(int(counts[p])):
            assert oracle.dist(padded[p], padded[ids[p, j]]).view(np.uint32) == dists[p, j].view(np.uint32)


def test_nndescent_host_entry_and_warm_start(gpu_ctx, oracle):
    """cs_nndescent (the nndescent_gpu drop-in) on host buffers, then a warm restart."""
    from coresg_b200.datagen import gaussian_mixture, pad_rows

    pts = pad_rows(gaussian_mixture(5000, 12, 6, (0.2, 1.0), 0.05, seed=8))
    ids, dists, flags, counts, upd = gpu_ctx.nndescent(pts, k=16, sample=8, iters=6, seed=3)
    assert upd > 0
    validate(ids, dists, counts, len(pts), 16)
    q = np.arange(0, 5000, 10, dtype=np.uint32)
    r1 = sampled_recall(oracle, pts, ids, 16, q)
    assert r1 > 0.9
    ids2, dists2, flags2, counts2, upd2 = gpu_ctx.nndescent(pts, k=16, sample=8, iters=6, seed=4, ids=ids,
                                                            dists=dists, flags=flags, counts=counts)
    validate(ids2, dists2, counts2, len(pts), 16)
    assert sampled_recall(oracle, pts, ids2, 16, q) >= r1 - 1e-9


def test_build_then_extract_matches_oracle(gpu_ctx, oracle):
    """GPU k-NN graph -> engine extraction == oracle extraction on the same graph."""
    z = load_golden("coresg_n3000_d24_k16")
    g = cs.CoreSG(gpu_ctx, 24, 16)
    g.set_points(z["points"])
    g.build_knn()
    ids, dists, flags, counts = g.knn()
    g.set_bridges(z["bridges"][:0])
    for m in (2, 16):
        e = oracle.edges(m, ids, dists, counts, z["bridges"][:0])
        assert g.edges(m).tobytes() == e.tobytes()
        o = oracle.mst(e, len(counts))
        assert g.mst(m).edges.tobytes() == e[o["in_tree"]].tobytes()
