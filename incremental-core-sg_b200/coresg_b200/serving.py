"""Serving loop binding (cs_server_* of include/coresg_b200.h) and the seeded request
stream of the serving workload.

The loop itself is native: a scheduler thread batches queries into sweeps and a
completion thread copies results out (csrc/server.cu).  This module marshals
requests and owns the pinned result buffers the completion copies write into.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._abi import EDGE_DTYPE, CoreSG, CsError, InsertParams, _ptr, lib

CS_REQ_EXTRACT, CS_REQ_EPS_LABELS, CS_REQ_INSERT = 0, 1, 2


class ServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("max_slots", C.c_uint32), ("inserts_first", C.c_uint32),
                ("reserved0", C.c_uint32), ("reserve_bytes", C.c_uint64), ("insert", InsertParams)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_int32), ("mpts", C.c_uint32), ("eps", C.c_double), ("rows", C.c_void_p),
                ("count", C.c_uint64), ("row_stride", C.c_uint32), ("out_edges", C.c_void_p),
                ("out_edges_cap", C.c_uint64), ("out_labels", C.c_void_p), ("out_labels_cap", C.c_uint64)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("ncomp", C.c_uint32), ("nedges", C.c_uint64), ("n", C.c_uint64),
                ("weight", C.c_double), ("queue_ms", C.c_double), ("latency_ms", C.c_double),
                ("batch", C.c_uint64), ("error", C.c_char * 160)]


class Stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("queries", C.c_uint64), ("inserts", C.c_uint64),
                ("inserted_rows", C.c_uint64), ("insert_batches", C.c_uint64), ("slots", C.c_uint64),
                ("slot_bytes", C.c_uint64), ("max_batch_seen", C.c_uint32), ("sweep_ms", C.c_double),
                ("insert_ms", C.c_double), ("reused_batches", C.c_uint64)]


class _HostMemory:
    """Owns one cs_host_alloc block; frees it when collected or on free()."""

    def __init__(self, nbytes: int):
        self.ptr = lib().cs_host_alloc(max(nbytes, 1))
        if not self.ptr:
            raise MemoryError("cs_host_alloc failed")

    def free(self):
        if self.ptr:
            lib().cs_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Pinned:
    """A page-locked host array (cs_host_alloc).  Every view of `array` keeps the
    memory alive (so `Pinned(shape, dtype).array` alone is safe to hold); it is freed
    once neither this object nor any view is referenced, or at once by free(), after
    which no view may be used."""

    def __init__(self, shape, dtype):
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dtype.itemsize
        self._mem = _HostMemory(nbytes)
        buf = (C.c_char * max(nbytes, 1)).from_address(self._mem.ptr)
        buf._mem = self._mem  # numpy keeps buf alive for every view; buf keeps the memory
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    @property
    def ptr(self):
        return self._mem.ptr

    def free(self):
        self.array = None
        self._mem.free()


class Server:
    """cs_server over a resident CoreSG: submit extract / epsilon-cut / insert
    requests from any thread, wait on their tickets."""

    def __init__(self, graph: CoreSG, max_batch=32, max_slots=64, reserve_bytes=0, inserts_first=False,
                 **insert_params):
        self.graph = graph
        cfg = ServerConfig()
        cfg.max_batch, cfg.max_slots, cfg.reserve_bytes = max_batch, max_slots, reserve_bytes
        cfg.inserts_first = int(bool(inserts_first))
        lib().cs_insert_defaults(C.byref(cfg.insert))
        for key, val in insert_params.items():
            setattr(cfg.insert, key, val)
        self.h = C.c_void_p()
        graph.ctx.check(lib().cs_server_create(graph.h, C.byref(cfg), C.byref(self.h)))
        self._keep = {}  # ticket -> buffers the request writes into

    def close(self):
        if self.h:
            lib().cs_server_destroy(self.h)
            self.h = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _submit(self, req: Request, keep) -> int:
        t = C.c_uint64()
        st = lib().cs_server_submit(self.h, C.byref(req), C.byref(t))
        if st != 0:
            raise CsError(st, lib().cs_last_error(None).decode())
        self._keep[t.value] = keep
        return t.value

    def extract(self, mpts: int, edges: np.ndarray | None = None, labels: np.ndarray | None = None) -> int:
        """Queue extract(mpts); the tree goes into `edges` (EDGE_DTYPE, >= n-1
        entries) and the component labels into `labels` (uint32, >= n), both optional."""
        r = Request()
        r.kind, r.mpts = CS_REQ_EXTRACT, mpts
        if edges is not None:
            assert edges.dtype == EDGE_DTYPE and edges.flags.c_contiguous
            r.out_edges, r.out_edges_cap = edges.ctypes.data, len(edges)
        if labels is not None:
            assert labels.dtype == np.uint32 and labels.flags.c_contiguous
            r.out_labels, r.out_labels_cap = labels.ctypes.data, len(labels)
        return self._submit(r, (edges, labels))

    def cut(self, mpts: int, eps: float, labels: np.ndarray) -> int:
        """Queue the epsilon-cut labels of the mpts tree (dbscan_labels_from_mst)."""
        assert labels.dtype == np.uint32 and labels.flags.c_contiguous
        r = Request()
        r.kind, r.mpts, r.eps = CS_REQ_EPS_LABELS, mpts, float(eps)
        r.out_labels, r.out_labels_cap = labels.ctypes.data, len(labels)
        return self._submit(r, (labels,))

    def insert(self, rows: np.ndarray) -> int:
        rows = np.ascontiguousarray(rows, np.float32)
        r = Request()
        r.kind, r.rows, r.count, r.row_stride = CS_REQ_INSERT, _ptr(rows), rows.shape[0], rows.shape[1]
        return self._submit(r, None)  # the rows are copied at submit

    def wait(self, ticket: int, timeout_ms: int | None = None) -> dict:
        res = Result()
        st = lib().cs_server_wait(self.h, ticket, 0xFFFFFFFF if timeout_ms is None else timeout_ms, C.byref(res))
        if st != 0:
            raise CsError(st, lib().cs_last_error(None).decode())
        self._keep.pop(ticket, None)
        return dict(status=res.status, ncomp=res.ncomp, nedges=res.nedges, n=res.n, weight=res.weight,
                    queue_ms=res.queue_ms, latency_ms=res.latency_ms, batch=res.batch,
                    error=res.error.decode(errors="replace"))

    def stats(self) -> dict:
        s = Stats()
        lib().cs_server_stats_get(self.h, C.byref(s))
        return {name: getattr(s, name) for name, _ in Stats._fields_}


@dataclass
class Arrival:
    t: float          # seconds after the start of the window
    kind: int         # CS_REQ_*
    mpts: int = 0
    quantile: float = 0.0  # epsilon-cut: the merge-height quantile of eps
    size: int = 0     # insert rows
    seed: int = 0     # insert batch seed


def request_stream(seconds: float, rate: float, k_max: int, seed: int, cut_fraction: float = 0.25,
                   insert_fraction: float = 0.10, insert_sizes=(1_000, 100_000)) -> list[Arrival]:
    """Poisson arrivals at `rate` per second over `seconds`: (1 - insert_fraction)
    extract(mpts ~ U{1..k_max}) queries, of which `cut_fraction` ask for
    epsilon-cut labels at a uniform merge-height quantile, and `insert_fraction`
    insert batches of log-uniform size in `insert_sizes`."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    lo, hi = np.log(insert_sizes[0]), np.log(insert_sizes[1])
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            return out
        if rng.random() < insert_fraction:
            out.append(Arrival(t, CS_REQ_INSERT, size=int(round(np.exp(rng.uniform(lo, hi)))),
                               seed=int(rng.integers(1 << 31))))
        else:
            m = int(rng.integers(1, k_max + 1))
            if rng.random() < cut_fraction:
                out.append(Arrival(t, CS_REQ_EPS_LABELS, mpts=m, quantile=float(rng.random())))
            else:
                out.append(Arrival(t, CS_REQ_EXTRACT, mpts=m))


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, np.float64), q)) if len(xs) else None
