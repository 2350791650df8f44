"""Serving loop (cs_server_*): every result served in a mixed, batched request stream
equals the same request served alone -- trees, labels, exact weights and component
counts bit for bit -- on the graph state the request saw (before or after an insert
barrier); epsilon-cut labels equal dbscan_labels_from_mst (src/eval.cpp:230-239)
restated on the host."""
import threading

import numpy as np
import pytest

import coresg_b200 as cs
from conftest import load_golden

pytestmark = pytest.mark.gpu


def resident(ctx, z):
    g = cs.CoreSG(ctx, int(z["dim"]), int(z["k"]))
    g.set_points(z["points"])
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    return g


def cut_labels(tree, n, eps):
    """dbscan_labels_from_mst: union of the tree edges with double(w) <= eps, labels
    dense in order of each component's smallest node."""
    parent = np.arange(n)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for u, v, w in tree:
        if float(w) <= eps:
            a, b = find(int(u)), find(int(v))
            if a != b:
                parent[max(a, b)] = min(a, b)
    roots = np.array([find(i) for i in range(n)])
    _, first = np.unique(roots, return_index=True)
    order = np.argsort(first)
    remap = np.empty(n, np.int64)
    remap[np.unique(roots)[order]] = np.arange(len(order))
    return remap[roots].astype(np.uint32), len(order)


def bufs(n):
    return np.zeros(n, cs.EDGE_DTYPE), np.zeros(n, np.uint32)


def test_mix_equals_alone_across_an_insert(gpu_ctx):
    z = load_golden("coresg_n6000_d16_k32")
    g = resident(gpu_ctx, z)
    n0 = len(z["counts"])
    pre = [4, 8, 16, 4, 32, 1, 8]
    alone = {m: g.mst(m) for m in set(pre)}
    eps8 = float(np.quantile(alone[8].edges["w"], 0.5))
    eps1 = float(np.quantile(alone[1].edges["w"], 0.9))
    rows = np.random.default_rng(5).normal(5.0, 1.0, size=(400, int(z["dim"]))).astype(np.float32)
    srv = cs.Server(g, max_batch=32)
    cap = n0 + len(rows)
    t_pre, t_cut = [], []
    for m in pre:
        e, lab = bufs(cap)
        t_pre.append((srv.extract(m, e, lab), m, e, lab))
    lab8, lab1 = np.zeros(cap, np.uint32), np.zeros(cap, np.uint32)
    t_cut.append((srv.cut(8, eps8, lab8), 8, eps8, lab8))
    t_cut.append((srv.cut(1, eps1, lab1), 1, eps1, lab1))
    t_ins = srv.insert(rows)
    post = [8, 4, 16, 32]
    t_post = []
    for m in post:
        e, lab = bufs(cap)
        t_post.append((srv.extract(m, e, lab), m, e, lab))
    res_pre = [(srv.wait(t), m, e, lab) for t, m, e, lab in t_pre]
    res_cut = [(srv.wait(t), m, eps, lab) for t, m, eps, lab in t_cut]
    ins = srv.wait(t_ins)
    res_post = [(srv.wait(t), m, e, lab) for t, m, e, lab in t_post]
    st = srv.stats()
    srv.close()
    assert ins["status"] == 0 and ins["n"] == cap
    for r, m, e, lab in res_pre:
        a = alone[m]
        assert r["status"] == 0 and r["n"] == n0
        assert e[: r["nedges"]].tobytes() == a.edges.tobytes()
        assert np.array_equal(lab[:n0], a.component)
        assert r["weight"] == a.weight and r["ncomp"] == a.num_components
    for r, m, eps, lab in res_cut:
        want, k = cut_labels(alone[m].edges, n0, eps)
        assert r["status"] == 0 and r["ncomp"] == k
        assert np.array_equal(lab[:n0], want)
    # after the barrier: the same requests alone on the grown graph
    for r, m, e, lab in res_post:
        a = g.mst(m)
        assert r["status"] == 0 and r["n"] == cap
        assert e[: r["nedges"]].tobytes() == a.edges.tobytes()
        assert np.array_equal(lab, a.component)
        assert r["weight"] == a.weight
    assert st["inserts"] == 1 and st["queries"] == len(pre) + 2 + len(post)
    # queries that arrived while the first sweep ran (it also captures the plan)
    # were served together by a later one
    assert st["max_batch_seen"] >= 2 and st["batches"] < st["queries"]
    assert st["failed"] == 0


def test_concurrent_submitters(gpu_ctx):
    """Four host threads submit at once; every result equals its alone twin."""
    z = load_golden("coresg_n3000_d24_k16")
    g = resident(gpu_ctx, z)
    n = len(z["counts"])
    mp = [1, 2, 3, 5, 8, 13, 16]
    alone = {m: g.mst(m) for m in mp}
    srv = cs.Server(g, max_batch=4, max_slots=8)  # forces several batches and slot reuse
    errors = []

    def worker(seed):
        rng = np.random.default_rng(seed)
        try:
            for _ in range(12):
                m = int(rng.choice(mp))
                e, lab = bufs(n)
                r = srv.wait(srv.extract(m, e, lab))
                a = alone[m]
                if not (r["status"] == 0 and e[: r["nedges"]].tobytes() == a.edges.tobytes()
                        and np.array_equal(lab, a.component) and r["weight"] == a.weight):
                    errors.append((seed, m, r))
        except Exception as ex:  # surfaced below
            errors.append((seed, repr(ex)))

    th = [threading.Thread(target=worker, args=(s,)) for s in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    st = srv.stats()
    srv.close()
    assert not errors, errors[:3]
    assert st["queries"] == 48 and st["slots"] <= 8


def test_request_errors(gpu_ctx):
    z = load_golden("coresg_n3000_d24_k16")
    g = resident(gpu_ctx, z)
    n = len(z["counts"])
    srv = cs.Server(g)
    with pytest.raises(cs.CsError):
        srv.extract(17)  # k_max = 16
    small = np.zeros(10, cs.EDGE_DTYPE)
    r = srv.wait(srv.extract(4, small))
    assert r["status"] == cs.CS_ERR_INVALID and "out_edges_cap" in r["error"]
    # the server keeps serving after a failed request
    e, lab = bufs(n)
    r = srv.wait(srv.extract(4, e, lab))
    assert r["status"] == 0 and e[: r["nedges"]].tobytes() == g.mst(4).edges.tobytes()
    # weight and counts only, no buffers
    r = srv.wait(srv.extract(8))
    assert r["status"] == 0 and r["weight"] == g.mst(8).weight
    srv.close()


def test_back_to_back_inserts_coalesce_and_inserts_first(gpu_ctx):
    """Inserts queued back to back run as one insert; with inserts_first a query
    submitted after an insert sees it, and every result equals the alone result on
    the graph state it reports."""
    z = load_golden("coresg_n6000_d16_k32")
    n0 = len(z["counts"])
    rng = np.random.default_rng(11)
    rows = [rng.normal(4.0, 1.0, size=(s, int(z["dim"]))).astype(np.float32) for s in (120, 300, 80)]
    n1 = n0 + sum(len(r) for r in rows)
    # arrival order: the first (slow, plan-capturing) sweep lets the inserts queue up
    g = resident(gpu_ctx, z)
    srv = cs.Server(g)
    t0 = srv.extract(4)
    ti = [srv.insert(r) for r in rows]
    t1 = srv.extract(4)
    r0, ri, r1 = srv.wait(t0), [srv.wait(t) for t in ti], srv.wait(t1)
    st = srv.stats()
    srv.close()
    assert r0["n"] == n0 and all(r["status"] == 0 and r["n"] == n1 for r in ri) and r1["n"] == n1
    assert st["inserts"] == 3 and st["insert_batches"] == 1 and st["inserted_rows"] == n1 - n0
    assert r1["weight"] == g.mst(4).weight
    # inserts first: queued inserts overtake queued queries, never the other way round
    g2 = resident(gpu_ctx, z)
    pre = g2.mst(8)
    srv = cs.Server(g2, inserts_first=True)
    e0, l0 = bufs(n1)
    t0 = srv.extract(8, e0, l0)
    ti = [srv.insert(r) for r in rows]
    e1, l1 = bufs(n1)
    t1 = srv.extract(8, e1, l1)
    r0, ri, r1 = srv.wait(t0), [srv.wait(t) for t in ti], srv.wait(t1)
    srv.close()
    post = g2.mst(8)
    assert r1["n"] == n1  # submitted after every insert
    for r, e, lab in ((r0, e0, l0), (r1, e1, l1)):
        want = pre if r["n"] == n0 else post
        assert r["n"] in (n0, n1)
        assert e[: r["nedges"]].tobytes() == want.edges.tobytes()
        assert np.array_equal(lab[: r["n"]], want.component) and r["weight"] == want.weight


def test_batches_between_inserts_reuse_the_last_sweep(gpu_ctx):
    """With k_max <= 32 a sweep solves every mpts; later batches with no insert in
    between are served from its results (no sweep), and after an insert the next batch
    sweeps again.  Every result equals the request served alone on its graph state."""
    z = load_golden("coresg_n3000_d24_k16")
    g = resident(gpu_ctx, z)
    n0 = len(z["counts"])
    alone = {m: g.mst(m) for m in (1, 3, 8, 16)}
    eps = float(np.quantile(alone[8].edges["w"], 0.6))
    srv = cs.Server(g, max_batch=32)
    # first batch: a sweep
    e, lab = bufs(n0)
    r = srv.wait(srv.extract(3, e, lab))
    assert r["status"] == 0 and e[: r["nedges"]].tobytes() == alone[3].edges.tobytes()
    sweeps = srv.stats()["batches"]
    # more batches, nothing inserted: served from that sweep
    for m in (16, 1, 8):
        e, lab = bufs(n0)
        r = srv.wait(srv.extract(m, e, lab))
        assert r["status"] == 0 and e[: r["nedges"]].tobytes() == alone[m].edges.tobytes()
        assert np.array_equal(lab[:n0], alone[m].component) and r["weight"] == alone[m].weight
    cl = np.zeros(n0, np.uint32)
    r = srv.wait(srv.cut(8, eps, cl))
    want, k = cut_labels(alone[8].edges, n0, eps)
    assert r["status"] == 0 and r["ncomp"] == k and np.array_equal(cl, want)
    st = srv.stats()
    assert st["batches"] == sweeps and st["reused_batches"] >= 4
    # an insert: the next query sweeps the grown graph
    rows = np.random.default_rng(9).normal(3.0, 1.0, size=(200, int(z["dim"]))).astype(np.float32)
    assert srv.wait(srv.insert(rows))["status"] == 0
    e, lab = bufs(n0 + len(rows))
    r = srv.wait(srv.extract(8, e, lab))
    st2 = srv.stats()
    srv.close()
    assert st2["batches"] == sweeps + 1
    a = g.mst(8)
    assert r["status"] == 0 and r["n"] == n0 + len(rows)
    assert e[: r["nedges"]].tobytes() == a.edges.tobytes() and r["weight"] == a.weight
