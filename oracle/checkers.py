"""Test infrastructure only: ctypes bindings for the two CPU checkers.

* `Oracle`    -- my C restatement of the reference algorithms (coresg_oracle.c).
* `Reference` -- the reference's own CPU code path compiled from its sources
                 (_ref/libcoresg_ref.so, built by oracle/Makefile; present when the
                 reference sources were available at build time).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline legs use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libcoresg_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcoresg_ref.so")

EDGE_DTYPE = np.dtype([("u", "<u4"), ("v", "<u4"), ("w", "<f4")])

_p = C.c_void_p
_u32, _u64, _i32, _f32, _f64 = C.c_uint32, C.c_uint64, C.c_int32, C.c_float, C.c_double


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _sig(lib, name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


class Oracle:
    """numpy-facing wrapper of libcoresg_oracle.so."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        lib = C.CDLL(path)
        self.lib = lib
        _sig(lib, "orc_l2sqr", _f32, _p, _p, _u32)
        _sig(lib, "orc_dist", _f32, _p, _p, _u32)
        _sig(lib, "orc_core", None, _p, _p, _u32, _u32, _u32, _p)
        _sig(lib, "orc_undirected", _u64, _p, _p, _p, _u32, _u32, _p)
        _sig(lib, "orc_edges", _u64, _u32, _p, _p, _p, _u32, _u32, _p, _u64, _p)
        _sig(lib, "orc_mst", C.c_int, _p, _u64, _u32, _p, _p, _p, _p, _p)
        _sig(lib, "orc_mst_kruskal", C.c_int, _p, _u64, _u32, _p, _p, _p)
        _sig(lib, "orc_exact_sum", _f64, _p, _u64)
        _sig(lib, "orc_rdeg", None, _p, _p, _u32, _u32, _p)
        _sig(lib, "orc_scores", None, _p, _p, _u32, _u32, _u32, _p, _p)
        _sig(lib, "orc_budget", _u64, _u32, _u64, _u32, _f64, _f64, _u64, _u64)
        _sig(lib, "orc_select", _u64, _p, _p, _u32, _u64, _p, _u32, _u32, _p)
        _sig(lib, "orc_conn", _u32, _p, _p, _u32, _u32, _p)
        _sig(lib, "orc_mrd_block", None, _p, _u32, _u32, _p, _u32, _u32, _p)
        _sig(lib, "orc_prim_dense", _u64, _p, _u32, _p)
        _sig(lib, "orc_bridges", _u64, _p, _u32, _u32, _u32, _p, _p, _p, _u32, _p, _u64, _p, _p)
        _sig(lib, "orc_brute_knn", None, _p, _u32, _u32, _u32, _p, _u32, _p, _p)

    # -- distances -------------------------------------------------------------
    def dist(self, a: np.ndarray, b: np.ndarray) -> np.float32:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return np.float32(self.lib.orc_dist(_ptr(a), _ptr(b), a.shape[-1]))

    def l2sqr(self, a, b) -> np.float32:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return np.float32(self.lib.orc_l2sqr(_ptr(a), _ptr(b), a.shape[-1]))

    # -- graph -> edges ----------------------------------------------------------
    def core(self, dists, counts, mpts):
        n, k = dists.shape
        out = np.empty(n, np.float32)
        self.lib.orc_core(_ptr(dists), _ptr(counts), n, k, mpts, _ptr(out))
        return out

    def undirected(self, ids, dists, counts):
        n, k = ids.shape
        m = self.lib.orc_undirected(_ptr(ids), _ptr(dists), _ptr(counts), n, k, None)
        out = np.empty(m, EDGE_DTYPE)
        self.lib.orc_undirected(_ptr(ids), _ptr(dists), _ptr(counts), n, k, _ptr(out))
        return out

    def edges(self, mpts, ids, dists, counts, bridges):
        n, k = ids.shape
        bridges = np.ascontiguousarray(bridges, EDGE_DTYPE)
        m = self.lib.orc_undirected(_ptr(ids), _ptr(dists), _ptr(counts), n, k, None) + len(bridges)
        out = np.empty(m, EDGE_DTYPE)
        self.lib.orc_edges(mpts, _ptr(ids), _ptr(dists), _ptr(counts), n, k, _ptr(bridges),
                           len(bridges), _ptr(out))
        return out

    # -- MST ---------------------------------------------------------------------
    def mst(self, edges, n):
        """Unique MSF under (w bits, edge index): dict(in_tree, labels, ncomp, nedges, weight)."""
        edges = np.ascontiguousarray(edges, EDGE_DTYPE)
        m = len(edges)
        in_tree = np.zeros(max(m, 1), np.uint8)
        labels = np.empty(max(n, 1), np.uint32)
        ncomp, ne, w = _u32(), _u64(), _f64()
        rc = self.lib.orc_mst(_ptr(edges), m, n, _ptr(in_tree), _ptr(labels), C.byref(ncomp),
                              C.byref(ne), C.byref(w))
        assert rc == 0
        return dict(in_tree=in_tree[:m].astype(bool), labels=labels[:n], ncomp=ncomp.value,
                    nedges=ne.value, weight=w.value)

    def mst_kruskal(self, edges, n):
        edges = np.ascontiguousarray(edges, EDGE_DTYPE)
        m = len(edges)
        in_tree = np.zeros(max(m, 1), np.uint8)
        ncomp, ne = _u32(), _u64()
        self.lib.orc_mst_kruskal(_ptr(edges), m, n, _ptr(in_tree), C.byref(ncomp), C.byref(ne))
        return dict(in_tree=in_tree[:m].astype(bool), ncomp=ncomp.value, nedges=ne.value)

    def exact_sum(self, w) -> float:
        w = np.ascontiguousarray(w, np.float32)
        return float(self.lib.orc_exact_sum(_ptr(w), len(w)))

    # -- hubness / bridges ------------------------------------------------------
    def rdeg(self, ids, counts):
        n, k = ids.shape
        out = np.empty(n, np.int32)
        self.lib.orc_rdeg(_ptr(ids), _ptr(counts), n, k, _ptr(out))
        return out

    def scores(self, ids, counts, rdeg, k_for_score=0):
        n, k = ids.shape
        out = np.empty(n, np.float64)
        self.lib.orc_scores(_ptr(ids), _ptr(counts), n, k, k_for_score, _ptr(rdeg), _ptr(out))
        return out

    def budget(self, dim, num_edges, n, multiplier=1.0, max_pair_ops=2e9, min_sel=2, max_sel=0):
        return int(self.lib.orc_budget(dim, num_edges, n, multiplier, max_pair_ops, min_sel, max_sel))

    def select(self, score, rdeg, budget, comp=None, ncomp=0, per=2):
        n = len(score)
        out = np.empty(budget + 2 * max(ncomp, 0) * max(per, 1) + 1, np.uint32)
        cnt = self.lib.orc_select(_ptr(score), _ptr(rdeg), n, budget, _ptr(comp), ncomp, per, _ptr(out))
        return out[:cnt].copy()

    def conn(self, ids, counts):
        n, k = ids.shape
        labels = np.empty(n, np.uint32)
        nc = self.lib.orc_conn(_ptr(ids), _ptr(counts), n, k, _ptr(labels))
        return labels, int(nc)

    def prim_dense(self, mat):
        mat = np.ascontiguousarray(mat, np.float32)
        m = mat.shape[0]
        out = np.empty(max(m, 1), EDGE_DTYPE)
        cnt = self.lib.orc_prim_dense(_ptr(mat), m, _ptr(out))
        return out[:cnt].copy()

    def mrd_block(self, pts, core, r0=0, r1=None):
        pts = np.ascontiguousarray(pts, np.float32)
        m, stride = pts.shape
        r1 = m if r1 is None else r1
        out = np.empty((r1 - r0, m), np.float32)
        self.lib.orc_mrd_block(_ptr(pts), m, stride, _ptr(np.ascontiguousarray(core, np.float32)),
                               r0, r1, _ptr(out))
        return out

    def bridges(self, padded, dim, ids, dists, counts):
        n, stride = padded.shape
        k = ids.shape[1]
        cap = 1 << 16
        out = np.empty(cap, EDGE_DTYPE)
        nsel, nrep = _u64(), _u64()
        cnt = self.lib.orc_bridges(_ptr(padded), n, dim, stride, _ptr(ids), _ptr(dists), _ptr(counts),
                                   k, _ptr(out), cap, C.byref(nsel), C.byref(nrep))
        return out[:min(cnt, cap)].copy(), int(nsel.value), int(nrep.value)

    def brute_knn(self, padded, k, queries=None):
        padded = np.ascontiguousarray(padded, np.float32)
        n, stride = padded.shape
        q = np.arange(n, dtype=np.uint32) if queries is None else np.ascontiguousarray(queries, np.uint32)
        ids = np.empty((len(q), k), np.uint32)
        dists = np.empty((len(q), k), np.float32)
        self.lib.orc_brute_knn(_ptr(padded), n, stride, k, _ptr(q), len(q), _ptr(ids), _ptr(dists))
        return ids, dists


class Reference:
    """The reference's own CPU path (coresg::CoreSG), via oracle/ref_harness.cpp."""

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def __init__(self, path: str = REF_SO):
        lib = C.CDLL(path)
        self.lib = lib
        _sig(lib, "ref_last_error", C.c_char_p)
        _sig(lib, "ref_metric_distance", _f32, _p, _p, _u32)
        _sig(lib, "ref_build", _p, _p, _u64, _u32, _u32, _u32, _u32, _u32, _u64, _u32, _p)
        _sig(lib, "ref_build_m", _p, _p, _u64, _u32, _u32, _u32, _u32, _u32, _u64, _u32, C.c_int, _p)
        _sig(lib, "ref_metric_distance_m", _f32, C.c_int, _p, _p, _u32)
        _sig(lib, "ref_dataset_rows", None, _p, _u64, _u32, C.c_int, _p)
        _sig(lib, "ref_from_state_m", _p, _p, _u64, _u32, _u32, _u32, _p, _p, _p, _p, _p, _u64, _u64, _u32,
             C.c_int)
        _sig(lib, "ref_nndescent_m", C.c_int, _p, _u64, _u32, _u32, _u32, _u32, _f64, _u64, _u32, C.c_int,
             _p, _p, _p, _p, _p)
        _sig(lib, "ref_insert", C.c_int, _p, _p, _u64, _p)
        _sig(lib, "ref_from_state", _p, _p, _u64, _u32, _u32, _u32, _p, _p, _p, _p, _p, _u64, _u64, _u32)
        _sig(lib, "ref_free", None, _p)
        _sig(lib, "ref_save", C.c_int, _p, C.c_char_p)
        _sig(lib, "ref_load", _p, C.c_char_p, _u32)
        _sig(lib, "ref_n", _u64, _p)
        _sig(lib, "ref_k", _u32, _p)
        _sig(lib, "ref_stride", _u32, _p)
        _sig(lib, "ref_get_points", None, _p, _p)
        _sig(lib, "ref_get_knn", None, _p, _p, _p, _p, _p)
        _sig(lib, "ref_bridges", _u64, _p, _p)
        _sig(lib, "ref_repair_count", _u64, _p)
        _sig(lib, "ref_selected", _u64, _p, _p)
        _sig(lib, "ref_scores", None, _p, _p, _p)
        _sig(lib, "ref_conn_labels", _u32, _p, _p)
        _sig(lib, "ref_core", None, _p, _u32, _p)
        _sig(lib, "ref_edges", _u64, _p, _u32, _p)
        _sig(lib, "ref_mst", C.c_int, _p, _u32, C.c_int, _u32, _p, _p, _p, _p, _p, _p, _p)
        _sig(lib, "ref_mst_edges", C.c_int, _p, _u64, _u32, C.c_int, _u32, _p, _p, _p, _p, _p)
        _sig(lib, "ref_mst_dense", _u64, _p, _u64, _p)
        _sig(lib, "ref_sampled_recall", _f64, _p, _u64, _u32, _p, _p, _p, _u32, _u64, _u64, _u32)
        _sig(lib, "ref_nndescent", C.c_int, _p, _u64, _u32, _u32, _u32, _u32, _f64, _u64, _u32,
             _p, _p, _p, _p, _p)
        _sig(lib, "ref_write_edges_tsv", C.c_int, C.c_char_p, _p, _u64)
        _sig(lib, "ref_write_labels_tsv", C.c_int, C.c_char_p, _p, _u64)

    def err(self) -> str:
        return self.lib.ref_last_error().decode()

    def write_edges_tsv(self, path, edges):
        """coresg::write_edges_tsv (src/io.cpp:131-138)."""
        e = np.ascontiguousarray(edges, EDGE_DTYPE)
        if self.lib.ref_write_edges_tsv(str(path).encode(), _ptr(e), len(e)):
            raise RuntimeError(self.err())

    def write_labels_tsv(self, path, labels):
        """coresg::write_labels_tsv (src/io.cpp:140-145)."""
        lab = np.ascontiguousarray(labels, np.uint32)
        if self.lib.ref_write_labels_tsv(str(path).encode(), _ptr(lab), len(lab)):
            raise RuntimeError(self.err())

    def metric_distance(self, a, b, metric=0):
        """metric_distance (include/coresg/distance.hpp) under metric code `metric`
        (0 L2, 1 cosine on normalised rows)."""
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return np.float32(self.lib.ref_metric_distance_m(metric, _ptr(a), _ptr(b), a.shape[-1]))

    def dataset_rows(self, rows, metric=0):
        """The padded rows Dataset::append stores (cosine rows normalised)."""
        rows = np.ascontiguousarray(rows, np.float32)
        n, d = rows.shape
        out = np.empty((n, (d + 7) & ~7), np.float32)
        self.lib.ref_dataset_rows(_ptr(rows), n, d, metric, _ptr(out))
        return out

    def build(self, rows, k_max=32, instances=1, iters=10, sample=16, seed=42, threads=0, metric=0):
        rows = np.ascontiguousarray(rows, np.float32)
        times = np.zeros(4, np.float64)
        h = self.lib.ref_build_m(_ptr(rows), rows.shape[0], rows.shape[1], k_max, instances, iters,
                                 sample, seed, threads, metric, _ptr(times))
        if not h:
            raise RuntimeError(self.err())
        return RefCoreSG(self, h, times)

    def from_state(self, padded, dim, ids, dists, flags, counts, bridges, repair=0, threads=0, metric=0):
        n, stride = padded.shape
        k = ids.shape[1]
        bridges = np.ascontiguousarray(bridges, EDGE_DTYPE)
        h = self.lib.ref_from_state_m(_ptr(padded), n, dim, stride, k, _ptr(ids), _ptr(dists),
                                      _ptr(flags), _ptr(counts), _ptr(bridges), len(bridges), repair,
                                      threads, metric)
        if not h:
            raise RuntimeError(self.err())
        return RefCoreSG(self, h, np.zeros(4))

    def mst_edges(self, edges, n, algo=1, threads=4):
        edges = np.ascontiguousarray(edges, EDGE_DTYPE)
        out = np.empty(max(n, 1), EDGE_DTYPE)
        labels = np.empty(max(n, 1), np.uint32)
        ncomp, ne, w = _u32(), _u64(), _f64()
        rc = self.lib.ref_mst_edges(_ptr(edges), len(edges), n, algo, threads, _ptr(out), _ptr(labels),
                                    C.byref(ncomp), C.byref(ne), C.byref(w))
        if rc:
            raise RuntimeError(self.err())
        return dict(edges=out[:ne.value].copy(), labels=labels[:n].copy(), ncomp=ncomp.value,
                    weight=w.value)

    def sampled_recall(self, rows, ids, dists, counts, k, queries, seed=4242, threads=0):
        rows = np.ascontiguousarray(rows, np.float32)
        return float(self.lib.ref_sampled_recall(_ptr(rows), rows.shape[0], rows.shape[1], _ptr(ids),
                                                 _ptr(dists), _ptr(counts), k, queries, seed,
                                                 threads or os.cpu_count()))

    def nndescent(self, rows, k=32, sample=16, iters=10, delta=0.001, seed=42, threads=0, metric=0):
        rows = np.ascontiguousarray(rows, np.float32)
        n = rows.shape[0]
        ids = np.empty((n, k), np.uint32)
        dists = np.empty((n, k), np.float32)
        counts = np.empty(n, np.uint32)
        ev, sec = _u64(), _f64()
        rc = self.lib.ref_nndescent_m(_ptr(rows), n, rows.shape[1], k, sample, iters, delta, seed,
                                      threads or os.cpu_count(), metric, _ptr(ids), _ptr(dists),
                                      _ptr(counts), C.byref(ev), C.byref(sec))
        if rc:
            raise RuntimeError(self.err())
        return ids, dists, counts, int(ev.value), float(sec.value)


class RefCoreSG:
    """Handle over a reference coresg::CoreSG."""

    def __init__(self, ref: Reference, h, times):
        self.ref, self.lib, self.h = ref, ref.lib, h
        self.times = dict(knn=times[0], hubness=times[1], bridges=times[2], total=times[3])

    def __del__(self):
        try:
            if self.h:
                self.lib.ref_free(self.h)
        except Exception:
            pass

    @property
    def n(self):
        return int(self.lib.ref_n(self.h))

    @property
    def k(self):
        return int(self.lib.ref_k(self.h))

    @property
    def stride(self):
        return int(self.lib.ref_stride(self.h))

    def points(self):
        out = np.empty((self.n, self.stride), np.float32)
        self.lib.ref_get_points(self.h, _ptr(out))
        return out

    def knn(self):
        n, k = self.n, self.k
        ids = np.empty((n, k), np.uint32)
        dists = np.empty((n, k), np.float32)
        flags = np.empty((n, k), np.uint8)
        counts = np.empty(n, np.uint32)
        self.lib.ref_get_knn(self.h, _ptr(ids), _ptr(dists), _ptr(flags), _ptr(counts))
        return ids, dists, flags, counts

    def bridges(self):
        m = self.lib.ref_bridges(self.h, None)
        out = np.empty(m, EDGE_DTYPE)
        self.lib.ref_bridges(self.h, _ptr(out))
        return out

    def repair_count(self):
        return int(self.lib.ref_repair_count(self.h))

    def selected(self):
        m = self.lib.ref_selected(self.h, None)
        out = np.empty(m, np.uint32)
        self.lib.ref_selected(self.h, _ptr(out))
        return out

    def scores(self):
        s = np.empty(self.n, np.float64)
        r = np.empty(self.n, np.int32)
        self.lib.ref_scores(self.h, _ptr(s), _ptr(r))
        return s, r

    def conn_labels(self):
        lab = np.empty(self.n, np.uint32)
        nc = self.lib.ref_conn_labels(self.h, _ptr(lab))
        return lab, int(nc)

    def core(self, mpts):
        out = np.empty(self.n, np.float32)
        self.lib.ref_core(self.h, mpts, _ptr(out))
        return out

    def edges(self, mpts):
        m = self.lib.ref_edges(self.h, mpts, None)
        if m == 2**64 - 1:
            raise RuntimeError(self.ref.err())
        out = np.empty(m, EDGE_DTYPE)
        self.lib.ref_edges(self.h, mpts, _ptr(out))
        return out

    def mst(self, mpts, algo=0, threads=4):
        n = self.n
        out = np.empty(max(n, 1), EDGE_DTYPE)
        labels = np.empty(max(n, 1), np.uint32)
        ncomp, ne, w, s_mst, s_all = _u32(), _u64(), _f64(), _f64(), _f64()
        rc = self.lib.ref_mst(self.h, mpts, algo, threads, _ptr(out), _ptr(labels), C.byref(ncomp),
                              C.byref(ne), C.byref(w), C.byref(s_mst), C.byref(s_all))
        if rc:
            raise RuntimeError(self.ref.err())
        return dict(edges=out[:ne.value].copy(), labels=labels[:n].copy(), ncomp=ncomp.value,
                    weight=w.value, seconds_mst=s_mst.value, seconds_all=s_all.value)

    def insert(self, rows):
        rows = np.ascontiguousarray(rows, np.float32)
        sec = _f64()
        if self.lib.ref_insert(self.h, _ptr(rows), rows.shape[0], C.byref(sec)):
            raise RuntimeError(self.ref.err())
        return sec.value

    def save(self, path):
        if self.lib.ref_save(self.h, path.encode()):
            raise RuntimeError(self.ref.err())
