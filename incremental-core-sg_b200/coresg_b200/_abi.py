"""ctypes binding of libcoresg_b200.so (declared in include/coresg_b200.h).

The shared library is the product; this module only marshals numpy arrays across
the C ABI.  It raises if the library is missing: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libcoresg_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_DIR), "include", "coresg_b200.h")

EDGE_DTYPE = np.dtype([("u", "<u4"), ("v", "<u4"), ("w", "<f4")])

CS_OK, CS_ERR_INVALID, CS_ERR_CUDA, CS_ERR_OOM, CS_ERR_TIMEOUT, CS_ERR_UNSUPPORTED, CS_ERR_STATE = range(7)
STATUS_NAMES = {0: "CS_OK", 1: "CS_ERR_INVALID", 2: "CS_ERR_CUDA", 3: "CS_ERR_OOM", 4: "CS_ERR_TIMEOUT",
                5: "CS_ERR_UNSUPPORTED", 6: "CS_ERR_STATE"}
CS_METRIC_L2, CS_METRIC_COSINE = 0, 1


class CsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class NndConfig(C.Structure):
    _fields_ = [("n", C.c_uint32), ("dim", C.c_uint32), ("stride", C.c_uint32), ("k", C.c_uint32),
                ("sample", C.c_uint32), ("iters", C.c_uint32), ("seed", C.c_uint64), ("metric", C.c_int32),
                ("delta", C.c_float), ("random_fill", C.c_int32)]


_p, _u32, _u64, _i32, _f32, _f64, _sz = (C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_float,
                                         C.c_double, C.c_size_t)
_pp = C.POINTER(C.c_void_p)

_SIGS = {
    "cs_device_count": (_i32, [_p]),
    "cs_device_props": (_i32, [_i32, C.c_char_p, _sz, _p, _p, _p, _p, _p]),
    "cs_last_error": (C.c_char_p, [_p]),
    "cs_ctx_create": (_i32, [_i32, _pp]),
    "cs_ctx_destroy": (None, [_p]),
    "cs_ctx_trim": (_i32, [_p]),
    "cs_ctx_launches": (_u64, [_p]),
    "cs_device_allocs": (None, [_p, _p]),
    "cs_nndescent": (_i32, [_p, _p, _p, _p, _p, _p, _p, _p]),
    "cs_mrd_block": (_i32, [_p, _p, _sz, _u32, _u32, _i32, _p, _sz, _sz, _p]),
    "cs_graph_create": (_i32, [_p, _u32, _u32, _i32, _pp]),
    "cs_graph_destroy": (None, [_p]),
    "cs_graph_set_points": (_i32, [_p, _p, _u64, _u32]),
    "cs_graph_append_points": (_i32, [_p, _p, _u64, _u32]),
    "cs_graph_set_knn": (_i32, [_p, _p, _p, _p, _p, _u64]),
    "cs_graph_get_knn": (_i32, [_p, _p, _p, _p, _p]),
    "cs_graph_set_bridges": (_i32, [_p, _p, _u64]),
    "cs_graph_get_bridges": (_i32, [_p, _p, _u64, _p]),
    "cs_graph_info": (_i32, [_p, _p, _p, _p, _p, _p, _p]),
    "cs_graph_save": (_i32, [_p, C.c_char_p]),
    "cs_graph_load": (_i32, [_p, C.c_char_p, _pp]),
    "cs_knn_build": (_i32, [_p, _u32, _u32, _f64, _u64, _p, _p]),
    "cs_knn_build_stats": (_i32, [_p, _p, _p]),
    "cs_graph_reserve": (_i32, [_p, _u64]),
    "cs_write_edges_tsv": (_i32, [C.c_char_p, _p, _u64]),
    "cs_write_labels_tsv": (_i32, [C.c_char_p, _p, _u64]),
    "cs_sweep_write_tsv": (_i32, [_p, _u32, C.c_char_p, C.c_char_p]),
    "cs_select_bridges": (_i32, [_p, _p, _p, _p, _p]),
    "cs_insert_defaults": (None, [_p]),
    "cs_insert": (_i32, [_p, _p, _u64, _u32, _p, _p, _p]),
    "cs_insert_stats_get": (_i32, [_p, _p]),
    "cs_get_selected": (_i32, [_p, _p, _u64, _p]),
    "cs_bridge_stats_get": (_i32, [_p, _p]),
    "cs_core_distances": (_i32, [_p, _u32, _p]),
    "cs_edges": (_i32, [_p, _u32, _p, _u64, _p]),
    "cs_extract": (_i32, [_p, _u32, _p, _p, _p, _p, _p]),
    "cs_extract_sweep": (_i32, [_p, _p, _u32, _p, _p, _p, _p, _p]),
    "cs_extract_sweep_device": (_i32, [_p, _p, _u32, _p]),
    "cs_sweep_fetch": (_i32, [_p, _u32, _p, _p, _p, _p, _p]),
    "cs_sweep_fetch_device": (_i32, [_p, _u32, _p, _p, _p, _p, _p]),
    "cs_sweep_timing": (_i32, [_p, _p, _p]),
    "cs_sweep_trace": (_i32, [_p, _p, _u32, _p]),
    "cs_set_sweep_shape": (_i32, [_p, _u32, _u32]),
    "cs_set_sweep_tail": (_i32, [_p, _u32, _u32]),
    "cs_autotune_sweep": (_i32, [_p, _p, _u32, _p, _p]),
    "cs_ctx_stream": (_p, [_p]),
    "cs_mst_noalloc": (_i32, [_p, _p, _p, _u64, _u32, _p, _p, _p, _p, _p, _p]),
    "cs_test_sweep_barrier": (_i32, [_p, _u64, _u64]),
    "cs_test_fail_device_allocs": (None, [_u64]),
    "cs_server_create": (_i32, [_p, _p, _pp]),
    "cs_server_destroy": (None, [_p]),
    "cs_server_submit": (_i32, [_p, _p, _p]),
    "cs_server_wait": (_i32, [_p, _u64, _u32, _p]),
    "cs_server_stats_get": (_i32, [_p, _p]),
    "cs_host_alloc": (_p, [_sz]),
    "cs_host_free": (None, [_p]),
}

_lib = None


def header_symbols(path: str = HEADER_PATH) -> list[str]:
    """Every function name declared in include/coresg_b200.h."""
    text = open(path).read()
    return sorted(set(re.findall(r"\b(cs_[a-z0-9_]+)\s*\(", text)))


def device_allocs() -> tuple:
    """(count, bytes) of the device allocations the library has made in this process."""
    n, b = C.c_uint64(), C.c_uint64()
    lib().cs_device_allocs(C.byref(n), C.byref(b))
    return int(n.value), int(b.value)


def write_edges_tsv(path, edges) -> None:
    """coresg::write_edges_tsv (cs_write_edges_tsv) of a host edge array."""
    e = np.ascontiguousarray(edges, EDGE_DTYPE)
    if lib().cs_write_edges_tsv(str(path).encode(), _ptr(e), len(e)) != CS_OK:
        raise CsError(CS_ERR_INVALID, lib().cs_last_error(None).decode())


def write_labels_tsv(path, labels) -> None:
    """coresg::write_labels_tsv (cs_write_labels_tsv) of a host label array."""
    lab = np.ascontiguousarray(labels, np.uint32)
    if lib().cs_write_labels_tsv(str(path).encode(), _ptr(lab), len(lab)) != CS_OK:
        raise CsError(CS_ERR_INVALID, lib().cs_last_error(None).decode())


def lib() -> C.CDLL:
    """Load libcoresg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `make -C {PKG_DIR}` "
                               "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def device_props(device: int = 0) -> dict:
    """cs_device_props: name, memory, SM count and compute capability of a device."""
    name = C.create_string_buffer(256)
    total, free = C.c_size_t(), C.c_size_t()
    sms, major, minor = C.c_int32(), C.c_int32(), C.c_int32()
    st = lib().cs_device_props(device, name, 256, C.byref(total), C.byref(free), C.byref(sms), C.byref(major),
                               C.byref(minor))
    if st != CS_OK:
        raise CsError(st, lib().cs_last_error(None).decode())
    return dict(name=name.value.decode(), total_mem=total.value, free_mem=free.value, sm_count=sms.value,
                cc=(major.value, minor.value))


def device_count() -> int:
    n = C.c_int32(0)
    lib().cs_device_count(C.byref(n))
    return int(n.value)


class Context:
    """One device, one stream (cs_ctx)."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        st = lib().cs_ctx_create(device, C.byref(self.h))
        if st != CS_OK:
            raise CsError(st, lib().cs_last_error(None).decode())
        self.device = device

    def check(self, st):
        if st != CS_OK:
            raise CsError(st, lib().cs_last_error(self.h).decode())

    @property
    def stream(self) -> int:
        """The context's cudaStream_t (cs_ctx_stream) as an integer handle."""
        return int(lib().cs_ctx_stream(self.h) or 0)

    @property
    def launches(self) -> int:
        return int(lib().cs_ctx_launches(self.h))

    def close(self):
        if self.h:
            lib().cs_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the two entry points of coresg::cuda ---------------------------------
    def nndescent(self, vectors: np.ndarray, k: int, sample=16, iters=10, seed=42, delta=0.001,
                  ids=None, dists=None, flags=None, counts=None, random_fill=True):
        """cs_nndescent on host buffers (drop-in for cuda::nndescent_gpu)."""
        vec = np.ascontiguousarray(vectors, np.float32)
        n, stride = vec.shape
        if ids is None:
            ids = np.full((n, k), 0xFFFFFFFF, np.uint32)
            dists = np.full((n, k), np.inf, np.float32)
            flags = np.zeros((n, k), np.uint8)
            counts = np.zeros(n, np.uint32)
        cfg = NndConfig(n, stride, stride, k, sample, iters, seed, CS_METRIC_L2, delta, int(random_fill))
        upd = C.c_uint64(0)
        self.check(lib().cs_nndescent(self.h, C.byref(cfg), _ptr(vec), _ptr(ids), _ptr(dists), _ptr(flags),
                                      _ptr(counts), C.byref(upd)))
        return ids, dists, flags, counts, int(upd.value)

    def mrd_block(self, pts: np.ndarray, core: np.ndarray, r0=0, r1=None, dim=None):
        pts = np.ascontiguousarray(pts, np.float32)
        m, stride = pts.shape
        r1 = m if r1 is None else r1
        out = np.empty((r1 - r0, m), np.float32)
        self.check(lib().cs_mrd_block(self.h, _ptr(pts), m, dim or stride, stride, CS_METRIC_L2,
                                      _ptr(np.ascontiguousarray(core, np.float32)), r0, r1, _ptr(out)))
        return out


class InsertParams(C.Structure):
    _fields_ = [("sample", C.c_uint32), ("instance_iters", C.c_uint32), ("refine_iters", C.c_uint32),
                ("context_per_new", C.c_double), ("owned_warm_fraction", C.c_double), ("refine_per_new", C.c_double),
                ("refine_max_fraction", C.c_double), ("delta", C.c_double), ("max_expand", C.c_uint32),
                ("reverse_cap", C.c_uint32), ("seed", C.c_uint64), ("reselect_bridges", C.c_int32)]


class InsertStats(C.Structure):
    _fields_ = [("new_points", C.c_uint64), ("instance_nodes", C.c_uint64), ("refine_nodes", C.c_uint64),
                ("updates", C.c_uint64), ("rounds", C.c_uint32), ("reserved0", C.c_uint32),
                ("reverse_ms", C.c_double), ("search_ms", C.c_double), ("instance_ms", C.c_double),
                ("refine_ms", C.c_double), ("finish_ms", C.c_double), ("bridges_ms", C.c_double),
                ("total_ms", C.c_double)]


class BridgeStats(C.Structure):
    _fields_ = [("connectivity_ms", C.c_double), ("hubness_ms", C.c_double), ("edges_ms", C.c_double),
                ("selection_ms", C.c_double), ("bridge_mst_ms", C.c_double), ("repair_ms", C.c_double),
                ("total_ms", C.c_double), ("selected", C.c_uint64), ("bridges", C.c_uint64), ("repair", C.c_uint64),
                ("knn_components", C.c_uint32), ("hub_refreshed", C.c_uint32), ("rescored", C.c_uint64),
                ("changed", C.c_uint64)]


class MstResult:
    """Mirror of coresg::MstResult (include/coresg/mst.hpp:77-85)."""

    def __init__(self, edges, component, num_components, weight):
        self.edges = edges
        self.component = component
        self.num_components = num_components
        self.weight = weight

    def is_tree(self):
        return self.num_components <= 1


class CoreSG:
    """Device-resident CORE-SG behind the C ABI, with the reference CoreSG's method
    names (include/coresg/coresg.hpp:140-188): build, insert, edges, mst, all_msts,
    core_distances, save/load of the CORESG01 format."""

    def __init__(self, ctx: Context, dim: int, k_max: int = 32, metric: int = CS_METRIC_L2):
        self.ctx = ctx
        self.h = C.c_void_p()
        ctx.check(lib().cs_graph_create(ctx.h, dim, k_max, metric, C.byref(self.h)))
        self.dim, self.k_max = dim, k_max

    def close(self):
        if self.h:
            lib().cs_graph_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state -------------------------------------------------------------------
    def set_points(self, rows: np.ndarray):
        rows = np.ascontiguousarray(rows, np.float32)
        self.ctx.check(lib().cs_graph_set_points(self.h, _ptr(rows), rows.shape[0], rows.shape[1]))

    def append_points(self, rows: np.ndarray):
        rows = np.ascontiguousarray(rows, np.float32)
        self.ctx.check(lib().cs_graph_append_points(self.h, _ptr(rows), rows.shape[0], rows.shape[1]))

    def set_knn(self, ids, dists, flags, counts):
        ids = np.ascontiguousarray(ids, np.uint32)
        dists = np.ascontiguousarray(dists, np.float32)
        flags = None if flags is None else np.ascontiguousarray(flags, np.uint8)
        counts = np.ascontiguousarray(counts, np.uint32)
        self.ctx.check(lib().cs_graph_set_knn(self.h, _ptr(ids), _ptr(dists), _ptr(flags), _ptr(counts),
                                              ids.shape[0]))

    def knn(self):
        n = self.n
        ids = np.empty((n, self.k_max), np.uint32)
        dists = np.empty((n, self.k_max), np.float32)
        flags = np.empty((n, self.k_max), np.uint8)
        counts = np.empty(n, np.uint32)
        self.ctx.check(lib().cs_graph_get_knn(self.h, _ptr(ids), _ptr(dists), _ptr(flags), _ptr(counts)))
        return ids, dists, flags, counts

    def set_bridges(self, edges):
        edges = np.ascontiguousarray(edges, EDGE_DTYPE)
        self.ctx.check(lib().cs_graph_set_bridges(self.h, _ptr(edges), len(edges)))

    def missing_edges(self):
        cnt = C.c_uint64(0)
        self.ctx.check(lib().cs_graph_get_bridges(self.h, None, 0, C.byref(cnt)))
        out = np.empty(cnt.value, EDGE_DTYPE)
        self.ctx.check(lib().cs_graph_get_bridges(self.h, _ptr(out), cnt.value, C.byref(cnt)))
        return out

    def info(self):
        n, nk, nb = C.c_uint64(), C.c_uint64(), C.c_uint64()
        k, d, s = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self.ctx.check(lib().cs_graph_info(self.h, C.byref(n), C.byref(k), C.byref(d), C.byref(s),
                                           C.byref(nk), C.byref(nb)))
        return dict(n=n.value, k_max=k.value, dim=d.value, stride=s.value, knn_edges=nk.value, bridges=nb.value)

    def save(self, path: str):
        """CoreSG::save (CORESG01, src/io.cpp:232-261)."""
        self.ctx.check(lib().cs_graph_save(self.h, path.encode()))

    @classmethod
    def load(cls, ctx: Context, path: str) -> "CoreSG":
        """CoreSG::load (CORESG01, src/io.cpp:263-330)."""
        h = C.c_void_p()
        ctx.check(lib().cs_graph_load(ctx.h, path.encode(), C.byref(h)))
        obj = cls.__new__(cls)
        obj.ctx, obj.h = ctx, h
        info = obj.info()
        obj.dim, obj.k_max = info["dim"], info["k_max"]
        return obj

    @property
    def n(self) -> int:
        n = C.c_uint64()
        self.ctx.check(lib().cs_graph_info(self.h, C.byref(n), None, None, None, None, None))
        return int(n.value)

    # -- build -------------------------------------------------------------------
    def build_knn(self, sample=16, iters=10, delta=0.001, seed=42):
        upd, rounds = C.c_uint64(), C.c_uint32()
        self.ctx.check(lib().cs_knn_build(self.h, sample, iters, delta, seed, C.byref(upd), C.byref(rounds)))
        return dict(updates=upd.value, rounds=rounds.value)

    def write_sweep_tsv(self, index: int, edges_path=None, labels_path=None):
        """Result `index` of the last sweep straight to TSV files (cs_sweep_write_tsv)."""
        enc = lambda p: None if p is None else str(p).encode()
        self.ctx.check(lib().cs_sweep_write_tsv(self.h, index, enc(edges_path), enc(labels_path)))

    def reserve(self, rows: int):
        """Dataset::reserve: capacity (arrays and scratch) for `rows` nodes now."""
        self.ctx.check(lib().cs_graph_reserve(self.h, int(rows)))

    def build_stats(self) -> dict:
        """Distance evaluations and device ms of the last build_knn (cs_knn_build_stats)."""
        ev, ms = C.c_uint64(), C.c_double()
        self.ctx.check(lib().cs_knn_build_stats(self.h, C.byref(ev), C.byref(ms)))
        return dict(distance_evals=ev.value, device_ms=ms.value)

    def select_bridges(self):
        sel, br, rep, comp = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
        self.ctx.check(lib().cs_select_bridges(self.h, C.byref(sel), C.byref(br), C.byref(rep), C.byref(comp)))
        return dict(selected=sel.value, bridges=br.value, repair=rep.value, knn_components=comp.value)

    def bridge_stats(self) -> dict:
        """Stages of the last bridge selection (cs_bridge_stats_get)."""
        x = BridgeStats()
        self.ctx.check(lib().cs_bridge_stats_get(self.h, C.byref(x)))
        return {name: getattr(x, name) for name, _ in BridgeStats._fields_}

    def selected(self):
        cnt = C.c_uint64(0)
        self.ctx.check(lib().cs_get_selected(self.h, None, 0, C.byref(cnt)))
        out = np.empty(cnt.value, np.uint32)
        self.ctx.check(lib().cs_get_selected(self.h, _ptr(out), cnt.value, C.byref(cnt)))
        return out

    def insert(self, rows: np.ndarray, **params):
        """CoreSG::insert on the device (cs_insert); params override cs_insert_defaults."""
        rows = np.ascontiguousarray(rows, np.float32)
        p = InsertParams()
        lib().cs_insert_defaults(C.byref(p))
        for key, val in params.items():
            setattr(p, key, val)
        act, upd = C.c_uint64(), C.c_uint64()
        self.ctx.check(lib().cs_insert(self.h, _ptr(rows), rows.shape[0], rows.shape[1], C.byref(p), C.byref(act),
                                       C.byref(upd)))
        return dict(active=act.value, updates=upd.value)

    def insert_stats(self) -> dict:
        """Stages of the last insert (cs_insert_stats_get)."""
        x = InsertStats()
        self.ctx.check(lib().cs_insert_stats_get(self.h, C.byref(x)))
        return {name: getattr(x, name) for name, _ in InsertStats._fields_ if name != "reserved0"}

    def build(self, rows: np.ndarray, sample=16, iters=10, delta=0.001, seed=42):
        """CoreSG::build: points, NN-Descent, bridges (src/coresg.cpp:260-323)."""
        self.set_points(rows)
        st = self.build_knn(sample, iters, delta, seed)
        st.update(self.select_bridges())
        return st

    # -- extraction -----------------------------------------------------------------
    def core_distances(self, mpts: int) -> np.ndarray:
        out = np.empty(self.n, np.float32)
        self.ctx.check(lib().cs_core_distances(self.h, mpts, _ptr(out)))
        return out

    def edges(self, mpts: int) -> np.ndarray:
        cnt = C.c_uint64(0)
        self.ctx.check(lib().cs_edges(self.h, mpts, None, 0, C.byref(cnt)))
        out = np.empty(cnt.value, EDGE_DTYPE)
        self.ctx.check(lib().cs_edges(self.h, mpts, _ptr(out), cnt.value, C.byref(cnt)))
        return out

    def mst(self, mpts: int, labels: bool = True) -> MstResult:
        """Plain per-mpts path (cs_extract)."""
        n = self.n
        edges = np.empty(max(n - 1, 1), EDGE_DTYPE)
        lab = np.empty(max(n, 1), np.uint32) if labels else None
        ne, nc, w = C.c_uint64(), C.c_uint32(), C.c_double()
        self.ctx.check(lib().cs_extract(self.h, mpts, _ptr(edges), _ptr(lab), C.byref(ne), C.byref(nc),
                                        C.byref(w)))
        return MstResult(edges[:ne.value], None if lab is None else lab[:n], nc.value, w.value)

    def all_msts(self, mpts_values, labels: bool = True, out_edges=None, out_labels=None) -> list[MstResult]:
        """Batched sweep (cs_extract_sweep) -- one persistent graph-captured launch.
        out_edges ([K][n-1] EDGE_DTYPE) and out_labels ([K][n] uint32) may be given
        (page-locked ones, e.g. Pinned arrays, are copied into without staging); the
        results are views of them."""
        mp = np.ascontiguousarray(mpts_values, np.uint32)
        K, n = len(mp), self.n
        cap = max(n - 1, 1)
        edges = np.empty((K, cap), EDGE_DTYPE) if out_edges is None else out_edges
        lab = (np.empty((K, max(n, 1)), np.uint32) if out_labels is None else out_labels) if labels else None
        if edges.dtype != EDGE_DTYPE or edges.shape != (K, cap) or not edges.flags.c_contiguous:
            raise ValueError("out_edges must be a C-contiguous [K][n-1] edge array")
        if lab is not None and (lab.dtype != np.uint32 or lab.shape != (K, max(n, 1)) or not lab.flags.c_contiguous):
            raise ValueError("out_labels must be a C-contiguous [K][n] uint32 array")
        ne = np.empty(K, np.uint64)
        nc = np.empty(K, np.uint32)
        w = np.empty(K, np.float64)
        self.ctx.check(lib().cs_extract_sweep(self.h, _ptr(mp), K, _ptr(edges), _ptr(lab), _ptr(ne), _ptr(nc),
                                              _ptr(w)))
        return [MstResult(edges[j, :ne[j]], None if lab is None else lab[j, :n], int(nc[j]), float(w[j]))
                for j in range(K)]

    def sweep_device(self, mpts_values) -> float:
        """Run the sweep leaving the trees on the device; returns the device ms."""
        mp = np.ascontiguousarray(mpts_values, np.uint32)
        ms = C.c_float()
        self.ctx.check(lib().cs_extract_sweep_device(self.h, _ptr(mp), len(mp), C.byref(ms)))
        return float(ms.value)

    def sweep_fetch(self, index: int, labels: bool = True) -> MstResult:
        n = self.n
        edges = np.empty(max(n - 1, 1), EDGE_DTYPE)
        lab = np.empty(max(n, 1), np.uint32) if labels else None
        ne, nc, w = C.c_uint64(), C.c_uint32(), C.c_double()
        self.ctx.check(lib().cs_sweep_fetch(self.h, index, _ptr(edges), _ptr(lab), C.byref(ne), C.byref(nc),
                                            C.byref(w)))
        return MstResult(edges[:ne.value], None if lab is None else lab[:n], nc.value, w.value)

    def sweep_fetch_device(self, index: int, d_edges: int, d_labels: int | None) -> dict:
        """Result `index` of the last sweep into device buffers (raw device addresses
        on this graph's device, e.g. torch tensors' data_ptr()); returns the scalars."""
        ne, nc, w = C.c_uint64(), C.c_uint32(), C.c_double()
        self.ctx.check(lib().cs_sweep_fetch_device(self.h, index, C.c_void_p(d_edges),
                                                   C.c_void_p(d_labels) if d_labels else None, C.byref(ne),
                                                   C.byref(nc), C.byref(w)))
        return dict(nedges=ne.value, ncomp=nc.value, weight=w.value)

    def sweep_trace(self) -> np.ndarray:
        """Per-round profile of the last sweep's first pass: columns phase A ns,
        phase B ns, flatten ns, edges walked, roots walked, flattened, live
        (edge, MST) pairs."""
        out = np.zeros((64, 7), np.uint64)
        r = C.c_uint32()
        self.ctx.check(lib().cs_sweep_trace(self.h, _ptr(out), 64, C.byref(r)))
        return out[: r.value]

    def sweep_timing(self):
        """(graph ms, persistent-kernel ms) of the last sweep."""
        gm, km = C.c_float(), C.c_float()
        self.ctx.check(lib().cs_sweep_timing(self.h, C.byref(gm), C.byref(km)))
        return float(gm.value), float(km.value)

    def set_sweep_shape(self, flatten=0, block=0):
        """flatten: divisor of the flatten rule (0 auto, 0xFFFFFFFF never); block threads."""
        self.ctx.check(lib().cs_set_sweep_shape(self.h, flatten, block))

    def set_sweep_tail(self, tail_div=0xFFFFFFFF, table_slots=0):
        """Contracted tail of later sweeps (cs_set_sweep_tail): start it once a round's
        root list holds at most n / tail_div nodes (0: never; the default 0xFFFFFFFF
        means 4); table_slots caps the tail table (0: the default)."""
        self.ctx.check(lib().cs_set_sweep_tail(self.h, tail_div, table_slots))

    def autotune(self, mpts_values):
        mp = np.ascontiguousarray(mpts_values, np.uint32)
        f, b = C.c_uint32(), C.c_uint32()
        self.ctx.check(lib().cs_autotune_sweep(self.h, _ptr(mp), len(mp), C.byref(f), C.byref(b)))
        return int(f.value), int(b.value)
