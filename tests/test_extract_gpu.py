"""GPU parity of the extraction path against the reference (golden fixtures) and the
oracle: core distances, CoreSG::edges(mpts), the plain per-mpts MST and the batched
sweep -- bit-exact trees, weights, labels and component counts."""
import hashlib

import numpy as np
import pytest

import coresg_b200 as cs
from conftest import edge_keys, golden_names, load_golden

pytestmark = pytest.mark.gpu


def resident(ctx, z, with_points=False):
    g = cs.CoreSG(ctx, int(z["dim"]), int(z["k"]))
    if with_points:
        g.set_points(z["points"])
    g.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g.set_bridges(z["bridges"])
    return g


def check_tree(oracle, z, edges_list, res, m, n):
    """res: cs.MstResult from the engine; edges_list: the oracle's edges(m)."""
    o = oracle.mst(edges_list, n)
    tree_o = edges_list[o["in_tree"]]
    # the engine returns the tree in ascending edge-index order
    assert res.edges.tobytes() == tree_o.tobytes()
    assert np.array_equal(edge_keys(res.edges), z[f"mst_keys_{m}"])
    assert np.array_equal(np.sort(res.edges["w"]).view(np.uint32), z[f"mst_wbits_{m}"])
    assert res.num_components == int(z[f"mst_ncomp_{m}"])
    if res.component is not None:
        assert np.array_equal(res.component, z[f"mst_labels_{m}"])
    assert res.weight == o["weight"]  # exact sum, bit for bit
    ref_w = float(z[f"mst_weight_{m}"])
    assert abs(res.weight - ref_w) <= 1e-12 * n * max(1.0, ref_w)


@pytest.mark.parametrize("name", golden_names())
def test_core_and_edges_bit_exact(gpu_ctx, oracle, name):
    z = load_golden(name)
    g = resident(gpu_ctx, z)
    info = g.info()
    assert info["knn_edges"] == int(z["undirected"]) and info["bridges"] == len(z["bridges"])
    for m in z["mpts"]:
        m = int(m)
        assert np.array_equal(g.core_distances(m).view(np.uint32), z[f"core_{m}"].view(np.uint32))
        e = g.edges(m)
        assert len(e) == int(z[f"edges_len_{m}"])
        assert hashlib.sha256(e.tobytes()).digest() == z[f"edges_sha_{m}"].tobytes()
    if "edges_full" in z:
        assert g.edges(int(z["edges_full_mpts"])).tobytes() == z["edges_full"].tobytes()


@pytest.mark.parametrize("name", golden_names())
def test_plain_extract_matches_reference(gpu_ctx, oracle, name):
    z = load_golden(name)
    g = resident(gpu_ctx, z)
    n = len(z["counts"])
    for m in z["mpts"]:
        m = int(m)
        e = oracle.edges(m, z["ids"], z["dists"], z["counts"], z["bridges"])
        check_tree(oracle, z, e, g.mst(m), m, n)


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("shape", [(0xFFFFFFFF, 256), (4, 512), (1 << 20, 128)])
def test_sweep_matches_reference(gpu_ctx, oracle, name, shape):
    """never / sometimes / always flatten, three block sizes."""
    z = load_golden(name)
    g = resident(gpu_ctx, z)
    g.set_sweep_shape(*shape)
    n = len(z["counts"])
    mp = [int(m) for m in z["mpts"]]
    res = g.all_msts(mp)
    for m, r in zip(mp, res):
        e = oracle.edges(m, z["ids"], z["dists"], z["counts"], z["bridges"])
        check_tree(oracle, z, e, r, m, n)


def test_pinned_views_keep_their_memory(gpu_ctx):
    """A view of a Pinned array keeps the page-locked memory alive after the Pinned
    object itself is dropped, and the memory is released once the last view goes."""
    import gc
    import weakref

    p = cs.Pinned((4096,), np.uint32)
    mem = weakref.ref(p._mem)
    view = p.array[100:200]
    del p
    gc.collect()
    assert mem() is not None and mem().ptr
    view[:] = 7  # still mapped
    assert int(view.sum()) == 700
    del view
    gc.collect()
    assert mem() is None
    # an explicit free releases the memory at once
    q = cs.Pinned((16,), np.uint32)
    m2 = q._mem
    q.free()
    assert m2.ptr is None and q.array is None


def test_sweep_into_pinned_outputs(gpu_ctx):
    """Trees and labels written into caller-provided page-locked arrays (copied by DMA
    without staging) equal the ones returned in fresh pageable arrays, twice in a row,
    and page-locked k-NN inputs give the same graph."""
    z = load_golden("coresg_n6000_d16_k32")
    g = resident(gpu_ctx, z)
    mp = [1, 4, 8, 16, 32]
    ref = g.all_msts(mp)
    n = len(z["counts"])
    out_e = cs.Pinned((len(mp), n - 1), cs.EDGE_DTYPE)
    out_l = cs.Pinned((len(mp), n), np.uint32)
    ins = [cs.Pinned(a.shape, a.dtype) for a in g.knn()]
    try:
        for p, a in zip(ins, g.knn()):
            p.array[...] = a
        for _ in range(2):
            g.set_knn(*(p.array for p in ins))
            got = g.all_msts(mp, out_edges=out_e.array, out_labels=out_l.array)
            for a, b in zip(ref, got):
                assert a.edges.tobytes() == b.edges.tobytes()
                assert np.array_equal(a.component, b.component)
                assert a.weight == b.weight and a.num_components == b.num_components
    finally:
        for p in ins + [out_e, out_l]:
            p.free()


def test_reserve_keeps_the_graph(gpu_ctx):
    """cs_graph_reserve grows the resident arrays in place (contents kept) and sizes the
    scratch for the capacity: trees before and after are identical, also when the
    capacity was reserved before any data arrived."""
    z = load_golden("coresg_n6000_d16_k32")
    n = len(z["counts"])
    g = resident(gpu_ctx, z)
    mp = [2, 8, 32]
    before = g.all_msts(mp)
    g.reserve(3 * n)
    ids, dists, _, counts = g.knn()
    assert np.array_equal(ids, z["ids"]) and np.array_equal(dists, z["dists"]) and np.array_equal(counts, z["counts"])
    after = g.all_msts(mp)
    g2 = cs.CoreSG(gpu_ctx, int(z["dim"]), int(z["k"]))
    g2.reserve(2 * n)
    g2.set_knn(z["ids"], z["dists"], z["flags"], z["counts"])
    g2.set_bridges(z["bridges"])
    fresh = g2.all_msts(mp)
    for a, b, c in zip(before, after, fresh):
        assert a.edges.tobytes() == b.edges.tobytes() == c.edges.tobytes()
        assert np.array_equal(a.component, b.component) and np.array_equal(a.component, c.component)
        assert a.weight == b.weight == c.weight


def test_full_sweep_1_to_kmax_repeats_and_zero(gpu_ctx, oracle):
    """All mpts 1..k_max, a repeated value and mpts 0 (== 1): 34 MSTs, so two passes."""
    z = load_golden("coresg_n6000_d16_k32")
    g = resident(gpu_ctx, z)
    mp = list(range(1, 33)) + [8, 0]
    res = g.all_msts(mp)
    plain = {m: g.mst(m) for m in (1, 8, 32)}
    for m, r in zip(mp, res):
        mm = max(m, 1)
        if mm in plain:
            assert r.edges.tobytes() == plain[mm].edges.tobytes()
            assert np.array_equal(r.component, plain[mm].component)
            assert r.weight == plain[mm].weight
    # MST weight is monotone in mpts (tests/test_coresg.cpp:135-149)
    w = [r.weight for r in res[:32]]
    assert all(w[i] <= w[i + 1] for i in range(31))


def test_sweep_device_then_fetch(gpu_ctx):
    z = load_golden("coresg_n3000_d24_k16")
    g = resident(gpu_ctx, z)
    ms = g.sweep_device([2, 4, 8])
    assert ms > 0
    r = g.sweep_fetch(1)
    assert np.array_equal(edge_keys(r.edges), z["mst_keys_4"])
    with pytest.raises(cs.CsError):
        g.sweep_fetch(3)


def random_graph(rng, n, k, fill=1.0, tie_levels=None):
    """A random k-NN-shaped state (sorted lists, some short) for edge cases."""
    ids = np.full((n, k), 0xFFFFFFFF, np.uint32)
    dists = np.full((n, k), np.inf, np.float32)
    counts = np.zeros(n, np.uint32)
    for p in range(n):
        c = int(rng.integers(0, k + 1)) if fill < 1.0 else k
        c = min(c, n - 1)
        nb = rng.choice(np.delete(np.arange(n), p), size=c, replace=False)
        if tie_levels:
            d = rng.integers(1, tie_levels + 1, size=c).astype(np.float32)
        else:
            d = rng.uniform(0.1, 5.0, size=c).astype(np.float32)
        o = np.argsort(d, kind="stable")
        ids[p, :c] = nb[o]
        dists[p, :c] = d[o]
        counts[p] = c
    return ids, dists, counts


@pytest.mark.parametrize("case", ["ties", "ragged", "tiny", "isolated"])
def test_edge_cases_against_oracle(gpu_ctx, oracle, case):
    rng = np.random.default_rng(abs(hash(case)) % 1000)
    if case == "ties":  # massive weight ties: only the edge index breaks them
        n, k = 1500, 8
        ids, dists, counts = random_graph(rng, n, k, tie_levels=2)
    elif case == "ragged":  # short and empty neighbourhoods (+inf core distances)
        n, k = 1200, 10
        ids, dists, counts = random_graph(rng, n, k, fill=0.5)
    elif case == "tiny":
        n, k = 2, 1
        ids = np.array([[1], [0]], np.uint32)
        dists = np.array([[1.5], [1.5]], np.float32)
        counts = np.array([1, 1], np.uint32)
    else:  # nodes with no edges at all: a forest with singleton components
        n, k = 50, 3
        ids, dists, counts = random_graph(rng, n, k, fill=0.3)
        counts[10:20] = 0
        ids[10:20] = 0xFFFFFFFF
        dists[10:20] = np.inf
        for p in range(n):  # drop references to the emptied nodes
            keep = [(i, d) for i, d in zip(ids[p, :counts[p]], dists[p, :counts[p]]) if not 10 <= i < 20]
            counts[p] = len(keep)
            ids[p] = 0xFFFFFFFF
            dists[p] = np.inf
            for j, (i, d) in enumerate(keep):
                ids[p, j], dists[p, j] = i, d
    bridges = np.zeros(0, cs.EDGE_DTYPE)
    g = cs.CoreSG(gpu_ctx, 4, k)
    g.set_knn(ids, dists, None, counts)
    g.set_bridges(bridges)
    mp = sorted({1, max(1, k // 2), k})
    sweep = g.all_msts(mp)
    for m, rs in zip(mp, sweep):
        e = oracle.edges(m, ids, dists, counts, bridges)
        assert g.edges(m).tobytes() == e.tobytes()
        o = oracle.mst(e, n)
        for r in (g.mst(m), rs):
            assert r.edges.tobytes() == e[o["in_tree"]].tobytes()
            assert np.array_equal(r.component, o["labels"])
            assert r.num_components == o["ncomp"]
            assert r.weight == o["weight"] or (np.isinf(r.weight) and np.isinf(o["weight"]))


def test_errors_are_statuses(gpu_ctx):
    z = load_golden("coresg_n3000_d24_k16")
    g = resident(gpu_ctx, z)
    with pytest.raises(cs.CsError) as ei:
        g.mst(17)  # k_max = 16
    assert ei.value.status == cs.CS_ERR_INVALID
    with pytest.raises(cs.CsError):
        g.all_msts([1, 99])
    with pytest.raises(cs.CsError):
        g.set_bridges(np.array([(0, 10**7, 1.0)], cs.EDGE_DTYPE))
    # the context is still usable after the errors
    assert np.array_equal(edge_keys(g.mst(4).edges), z["mst_keys_4"])


def test_autotune_picks_a_shape(gpu_ctx):
    z = load_golden("coresg_n6000_d16_k32")
    g = resident(gpu_ctx, z)
    F, B = g.autotune(list(range(1, 9)))
    assert F in (0, 1, 2, 4, 16) and B in (256, 512)
    res = g.all_msts(list(range(1, 9)))
    assert np.array_equal(edge_keys(res[7].edges), z["mst_keys_8"])


@pytest.mark.parametrize("shape", [(4, 512), (0xFFFFFFFF, 256), (2, 256)])
def test_sweep_matches_plain_at_scale(gpu_ctx, shape):
    """At n = 200,000 (enough Boruvka rounds, warps and blocks for races between
    phases to show) every batched tree equals the plain path's, edge for edge."""
    from coresg_b200.datagen import gaussian_mixture

    pts = gaussian_mixture(200_000, 16, 30, (0.2, 1.0), 0.05, seed=77)
    g = cs.CoreSG(gpu_ctx, 16, 32)
    g.build(pts)
    g.set_sweep_shape(*shape)
    mp = list(range(1, 33))
    g.sweep_device(mp)
    for m in (1, 2, 7, 16, 32):
        plain, swept = g.mst(m), g.sweep_fetch(m - 1)
        assert swept.edges.tobytes() == plain.edges.tobytes()
        assert np.array_equal(swept.component, plain.component) and swept.weight == plain.weight


def test_k_max_above_32(gpu_ctx, oracle):
    """k_max = 48: the device build (the 128-element merge network), the bridges, a sweep
    of mpts 1..48 (two chained passes of 32 and 16 lanes) and the plain path against the
    oracle, then a small insert whose bridge re-selection takes the incremental hubness
    refresh with lists longer than 32 (the delta's two halves)."""
    from coresg_b200.datagen import gaussian_mixture, pad_rows
    from test_knn_gpu import validate

    pts = gaussian_mixture(4000, 12, 6, (0.2, 1.0), 0.05, seed=91)
    k, d = 48, 12
    g = cs.CoreSG(gpu_ctx, d, k)
    g.build(pts, sample=16, iters=10, seed=42)
    ids, dists, flags, counts = g.knn()
    n = len(pts)
    validate(ids, dists, counts, n, k)
    br, _, _ = oracle.bridges(pad_rows(pts), d, ids, dists, counts)
    assert g.missing_edges().tobytes() == br.tobytes()
    mp = list(range(1, k + 1))
    res = g.all_msts(mp)
    for m in (1, 17, 32, 33, 40, 48):
        e = oracle.edges(m, ids, dists, counts, br)
        o = oracle.mst(e, n)
        for r in (res[m - 1], g.mst(m)):
            assert r.edges.tobytes() == e[o["in_tree"]].tobytes()
            assert np.array_equal(r.component, o["labels"]) and r.weight == o["weight"]
    extra = gaussian_mixture(40, d, 6, (0.2, 1.0), 0.0, seed=92)
    g.insert(extra)
    allpts = np.concatenate([pts, extra])
    ids, dists, flags, counts = g.knn()
    validate(ids, dists, counts, len(allpts), k)
    st = g.bridge_stats()
    assert st["hub_refreshed"] == int(st["changed"] * 16 <= len(allpts))
    br, _, _ = oracle.bridges(pad_rows(allpts), d, ids, dists, counts)
    assert g.missing_edges().tobytes() == br.tobytes()
