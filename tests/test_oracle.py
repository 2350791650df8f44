"""CPU tests: the oracle (my C restatement of the reference) pinned against the
golden fixtures that the reference itself produced, plus the reference's own
known-answer MST / k-NN graph cases (tests/test_mst.cpp, tests/test_knn_graph.cpp)."""
import hashlib

import numpy as np
import pytest

from conftest import edge_keys, golden_names, load_golden
from checkers import EDGE_DTYPE, Reference


def E(rows):
    out = np.empty(len(rows), EDGE_DTYPE)
    for i, (u, v, w) in enumerate(rows):
        out[i] = (min(u, v), max(u, v), w)
    return out


# ---- known answers from the reference's own tests -----------------------------------

def test_small_known_tree(oracle):  # tests/test_mst.cpp:14-25
    r = oracle.mst(E([(0, 1, 1.0), (1, 2, 2.0), (0, 2, 5.0)]), 3)
    assert r["nedges"] == 2 and r["ncomp"] == 1 and abs(r["weight"] - 3.0) < 1e-12


def test_forest(oracle):  # tests/test_mst.cpp:27-38
    r = oracle.mst(E([(0, 1, 1.0), (2, 3, 1.0)]), 5)
    assert r["nedges"] == 2 and r["ncomp"] == 3
    lab = r["labels"]
    assert lab[0] == lab[1] and lab[2] == lab[3] and lab[0] != lab[2]
    assert list(lab) == [0, 0, 1, 1, 2]  # numbered by smallest node


def test_kruskal_and_boruvka_order_agree_on_weight(oracle):  # tests/test_mst.cpp:40-63
    rng = np.random.default_rng(42)
    n = 3000
    rows = [(i, int(rng.integers(0, i)), float(rng.uniform(0.01, 10))) for i in range(1, n)]
    for _ in range(n * 10):
        a, b = (int(x) for x in rng.integers(0, n, 2))
        if a != b:
            rows.append((a, b, float(rng.uniform(0.01, 10))))
    e = E(rows)
    b = oracle.mst(e, n)
    k = oracle.mst_kruskal(e, n)
    assert b["ncomp"] == 1 and k["ncomp"] == 1 and b["nedges"] == k["nedges"] == n - 1
    wb = np.sort(e["w"][b["in_tree"]])
    wk = np.sort(e["w"][k["in_tree"]])
    assert np.array_equal(wb.view(np.uint32), wk.view(np.uint32))


def test_dense_prim_matches_kruskal(oracle):  # tests/test_mst.cpp:65-84
    rng = np.random.default_rng(7)
    m = 120
    mat = np.zeros((m, m), np.float32)
    rows = []
    for i in range(m):
        for j in range(i + 1, m):
            v = np.float32(rng.uniform(0.5, 4.0))
            mat[i, j] = mat[j, i] = v
            rows.append((i, j, v))
    prim = oracle.prim_dense(mat)
    kru = oracle.mst(E(rows), m)
    assert len(prim) == m - 1
    assert abs(oracle.exact_sum(prim["w"]) - kru["weight"]) < 1e-9


def test_prim_disconnected(oracle):  # tests/test_mst.cpp:86-98
    n = 8
    mat = np.full((n, n), np.inf, np.float32)
    mat[:4, :4] = 1.0
    mat[4:, 4:] = 1.0
    assert len(oracle.prim_dense(mat)) == 6


def test_core_distance_rules(oracle):  # tests/test_knn_graph.cpp:50-58
    dists = np.full((2, 4), np.inf, np.float32)
    dists[0, 0] = 1.0
    counts = np.array([1, 0], np.uint32)
    assert oracle.core(dists, counts, 1)[0] == 1.0
    assert oracle.core(dists, counts, 4)[0] == 1.0  # clamp to the filled range
    assert np.isinf(oracle.core(dists, counts, 1)[1])  # empty neighbourhood
    assert oracle.core(dists, counts, 0)[0] == 1.0  # mpts 0 behaves as 1


def test_undirected_dedup(oracle):  # tests/test_knn_graph.cpp:60-74
    ids = np.full((3, 2), 0xFFFFFFFF, np.uint32)
    dists = np.full((3, 2), np.inf, np.float32)
    ids[0, 0], dists[0, 0] = 1, 1.0
    ids[1, 0], dists[1, 0] = 0, 1.0
    ids[2, 0], dists[2, 0] = 0, 4.0
    counts = np.array([1, 1, 1], np.uint32)
    e = oracle.undirected(ids, dists, counts)
    assert len(e) == 2
    assert set(zip(e["u"].tolist(), e["v"].tolist())) == {(0, 1), (0, 2)}


def test_exact_sum_is_exact(oracle):
    rng = np.random.default_rng(3)
    w = rng.uniform(1e-3, 1e3, 100000).astype(np.float32)
    from fractions import Fraction

    exact = sum((Fraction(float(x)) for x in w), Fraction(0))
    assert oracle.exact_sum(w) == float(exact)
    assert oracle.exact_sum(np.array([], np.float32)) == 0.0
    assert np.isinf(oracle.exact_sum(np.array([1.0, np.inf], np.float32)))
    tiny = np.array([1e-45, 1e-45, 3e-38], np.float32)  # subnormals
    assert oracle.exact_sum(tiny) == float(sum(Fraction(float(x)) for x in tiny))


def test_l2_association_order(oracle):
    """orc_l2sqr restates the AVX2 lane order; a plain left-to-right sum differs
    in the last bits on some inputs, and the fixtures pin which one is right."""
    z = load_golden("coresg_n2000_d40_k10")
    P, ids, dists, counts = z["padded"], z["ids"], z["dists"], z["counts"]
    for p in range(0, len(P), 13):
        for j in range(int(counts[p])):
            assert oracle.dist(P[p], P[ids[p, j]]).view(np.uint32) == dists[p, j].view(np.uint32)


# ---- the oracle against every golden fixture -----------------------------------------

@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_fixture(oracle, name):
    z = load_golden(name)
    ids, dists, counts, bridges = z["ids"], z["dists"], z["counts"], z["bridges"]
    n = len(counts)
    # stored k-NN distances are the reference arithmetic on these points
    P = z["padded"]
    for p in range(0, n, 17):
        for j in range(int(counts[p])):
            assert oracle.dist(P[p], P[ids[p, j]]).view(np.uint32) == dists[p, j].view(np.uint32)
    assert len(oracle.undirected(ids, dists, counts)) == int(z["undirected"])
    for m in z["mpts"]:
        m = int(m)
        core = oracle.core(dists, counts, m)
        assert np.array_equal(core.view(np.uint32), z[f"core_{m}"].view(np.uint32))
        e = oracle.edges(m, ids, dists, counts, bridges)
        assert len(e) == int(z[f"edges_len_{m}"])
        assert hashlib.sha256(e.tobytes()).digest() == z[f"edges_sha_{m}"].tobytes()
        r = oracle.mst(e, n)
        tree = e[r["in_tree"]]
        assert np.array_equal(edge_keys(tree), z[f"mst_keys_{m}"])
        assert np.array_equal(np.sort(tree["w"]).view(np.uint32), z[f"mst_wbits_{m}"])
        assert np.array_equal(r["labels"], z[f"mst_labels_{m}"])
        assert r["ncomp"] == int(z[f"mst_ncomp_{m}"])
        ref_w = float(z[f"mst_weight_{m}"])
        assert abs(r["weight"] - ref_w) <= 1e-12 * max(1.0, abs(ref_w)) * n
    if "edges_full" in z:
        m = int(z["edges_full_mpts"])
        assert oracle.edges(m, ids, dists, counts, bridges).tobytes() == z["edges_full"].tobytes()
    # hubness, connectivity, bridges
    rd = oracle.rdeg(ids, counts)
    assert np.array_equal(rd, z["rdeg"])
    sc = oracle.scores(ids, counts, rd)
    assert np.array_equal(sc.view(np.uint64), z["score"].view(np.uint64))
    lab, nc = oracle.conn(ids, counts)
    assert nc == int(z["ncomp_knn"]) and np.array_equal(lab, z["conn"])
    br, nsel, nrep = oracle.bridges(P, int(z["dim"]), ids, dists, counts)
    assert nsel == len(z["selected"])
    assert nrep == int(z["repair"])
    assert br.tobytes() == bridges.tobytes()
    budget = oracle.budget(int(z["dim"]), int(z["undirected"]), n)
    sel = oracle.select(sc, rd, budget, lab, nc, 2)
    assert np.array_equal(sel, z["selected"])


@pytest.mark.skipif(not Reference.available(), reason="reference not built (oracle/_ref)")
def test_oracle_against_live_reference(oracle):
    """A fresh case not in the fixtures, against the reference compiled here."""
    from coresg_b200.datagen import gaussian_mixture

    ref = Reference()
    pts = gaussian_mixture(3500, 12, 7, (0.1, 0.8), 0.04, seed=99)
    sg = ref.build(pts, k_max=12, threads=4)
    ids, dists, flags, counts = sg.knn()
    br = sg.bridges()
    assert br.tobytes() == oracle.bridges(sg.points(), 12, ids, dists, counts)[0].tobytes()
    for m in (1, 6, 12):
        e = sg.edges(m)
        assert e.tobytes() == oracle.edges(m, ids, dists, counts, br).tobytes()
        r = sg.mst(m, algo=1, threads=4)
        o = oracle.mst(e, sg.n)
        assert np.array_equal(edge_keys(r["edges"]), edge_keys(e[o["in_tree"]]))
        assert np.array_equal(r["labels"], o["labels"])
