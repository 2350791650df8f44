#!/usr/bin/env python3
"""Benchmark of the CORE-SG hot path on B200.

One step = one full mpts sweep (mpts = 1..k_max, K MSTs) over the device-resident
CORE-SG of the workload, solved by the batched path: one persistent cooperative
Boruvka launch replayed from a CUDA graph (cs_extract_sweep_device).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload blobs1m_d16]
    python bench.py --impl reference ...   # the reference's own CPU path, same metric

Reported (one JSON line from rank 0):
  value      whole-job MSTs/s of the batched sweep, inputs resident in HBM, device
             time (CUDA events on the engine stream), max over ranks
  plain      the plain per-mpts GPU path (cs_extract: edges(mpts) materialised per call,
             Boruvka rounds driven from the host) on the same graph
  build_s    device CORE-SG build: NN-Descent + anti-hub bridges, on a fresh graph (its
             device allocations included); rebuild_s the same build again on it
  e2e        the same metric through the C ABI with host buffers: the CORE-SG arrays
             copied host->device and all K trees + labels copied back, every step;
             three graphs in flight on their own contexts (--e2e-inflight), so one
             step's copies overlap another's sweep (e2e.serial: one graph, steps back
             to back)
  roofline   the persistent Boruvka kernel against the measured HBM copy bandwidth
  cpu_baseline  the reference CPU extract (built from its sources) on the same
             CORE-SG, a bounded sample of mpts values, all host threads
  parity     the sweep's trees against the reference's own CoreSG::mst on the same
             CORE-SG for the baseline's mpts values (edges, weight bits, labels,
             components, exact weight)
  build_roofline  the descent's FP32 rate (3 d FLOP per distance evaluation) against
             the CUDA-core FP32 peak at the sampled SM clock
With --gpus N > 1 (torchrun, one rank per GPU) a step is one sweep of mpts 1..K
partitioned across the ranks plus the gather of all K results into rank 0's device
memory (run_partitioned; strong scaling).
Inputs: seeded synthetic Gaussian mixtures with the workload's shapes; the edge list
(12 B x |E|, ~300 MB at n=1M) is larger than L2, so no L2 flush is needed.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "incremental-core-sg_b200"))

METRIC = "mpts-sweep MSTs/s + build s, n=1M k=32 vs plain GPU path; p50/p99 query ms"
FALLBACK_HBM_GBS = 6650.0


def profiled_traffic(workload: str, n: int):
    """DRAM bytes (read + write) of one k_sweep launch on this workload, from the ncu
    capture summarised in profiles/ (a line `traffic_per_launch_bytes: B workload W n N`),
    or None when no capture of this workload and size is committed."""
    import re
    d = os.path.join(ROOT, "profiles")
    for f in sorted(os.listdir(d)) if os.path.isdir(d) else []:
        if not f.startswith("k_sweep_"):
            continue
        for line in open(os.path.join(d, f)):
            m = re.search(r"traffic_per_launch_bytes:\s*(\d+)\s+workload\s+(\S+)\s+n\s+(\d+)", line)
            if m and m.group(2) == workload and int(m.group(3)) == n:
                return int(m.group(1)), f
    return None


def build_recall(g, pts, device: int, queries: int, seed: int) -> dict:
    """recall@k of the resident k-NN graph against FP32 brute force for a seeded sample
    of query points (torch on the device, chunks of 500 queries; a measurement only)."""
    ids, _, _, counts = g.knn()
    return recall_of(ids, counts, pts, device, queries, seed)


def recall_of(ids, counts, pts, device: int, queries: int, seed: int) -> dict:
    """recall@k of k-NN arrays (ids [n][k], counts [n]) against FP32 brute force for a
    seeded sample of query points (torch.cdist on the device, 500 queries a chunk)."""
    import torch

    n, k = ids.shape
    rng = np.random.default_rng(seed)
    q = np.sort(rng.choice(n, size=min(queries, n), replace=False))
    X = torch.from_numpy(np.ascontiguousarray(pts, np.float32)).to(f"cuda:{device}")
    hits = total = 0
    for c0 in range(0, len(q), 500):
        qi = torch.from_numpy(q[c0:c0 + 500]).to(X.device)
        d = torch.cdist(X[qi], X)  # [b, n]
        d[torch.arange(len(qi), device=X.device), qi] = float("inf")  # not its own neighbour
        top = torch.topk(d, k, dim=1, largest=False).indices.cpu().numpy()
        for r, v in enumerate(q[c0:c0 + 500]):
            got = ids[v, :counts[v]]
            hits += len(np.intersect1d(got, top[r], assume_unique=True))
            total += k
        del d
    del X
    torch.cuda.empty_cache()
    return {"recall_at_k": hits / total, "k": k, "queries": int(len(q)),
            "what": "k-NN lists vs FP32 brute force (torch.cdist), sampled queries"}


def reference_gpu_build(cs, ctx, device, pts, w):
    """The reference's own CUDA NN-Descent (coresg::cuda::nndescent_gpu, its sources
    built for sm_100a with its flags by oracle/Makefile) on this workload, once, as
    CudaBackend::run_knn_job runs it: host buffers in and out, its device allocations
    included (sample 16, 10 iterations, delta 0.001); beside it, the engine's
    cs_nndescent at the same boundary.  Wall seconds and recall@k of each."""
    import ctypes as C

    from coresg_b200.datagen import pad_rows

    so = os.path.join(ROOT, "oracle", "_ref", "libcoresg_refgpu.so")
    if not os.path.exists(so):
        return {"unavailable": "oracle/_ref/libcoresg_refgpu.so (the reference's CUDA sources built) is missing"}
    lib = C.CDLL(so)
    lib.refgpu_last_error.restype = C.c_char_p
    P, U32, U64 = C.c_void_p, C.c_uint32, C.c_uint64
    lib.refgpu_nndescent.argtypes = [C.c_int, U32, U32, U32, U32, U32, U32, U64, C.c_int, C.c_float,
                                     P, P, P, P, P, P]
    padded = pad_rows(pts)
    n, stride = padded.shape
    k = w["k_max"]
    ids = np.full((n, k), 0xFFFFFFFF, np.uint32)
    dists = np.full((n, k), np.inf, np.float32)
    flags = np.zeros((n, k), np.uint8)
    counts = np.zeros(n, np.uint32)
    upd = C.c_uint64()
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    t0 = time.perf_counter()
    rc = lib.refgpu_nndescent(device, n, w["dim"], stride, k, 16, 10, 42, 0, 0.001, ptr(padded), ptr(ids),
                              ptr(dists), ptr(flags), ptr(counts), C.byref(upd))
    ref_s = time.perf_counter() - t0
    if rc:
        return {"failed": lib.refgpu_last_error().decode()}
    ref_recall = recall_of(ids, counts, pts, device, 10000, 7)["recall_at_k"]
    t0 = time.perf_counter()
    mids, _, _, mcounts, _ = ctx.nndescent(padded, k=k, sample=16, iters=10, seed=42)
    ours_s = time.perf_counter() - t0
    ours_recall = recall_of(mids, mcounts, pts, device, 10000, 7)["recall_at_k"]
    return {"reference_nndescent_gpu_s": ref_s, "reference_recall_at_k": ref_recall,
            "engine_cs_nndescent_s": ours_s, "engine_recall_at_k": ours_recall,
            "speedup": ref_s / ours_s if ours_s > 0 else None,
            "what": "the reference's cuda::nndescent_gpu (built for sm_100a) vs the engine's cs_nndescent, host "
                    "buffers in and out, sample 16, 10 iterations, same B200; recall vs FP32 brute force, 10,000 "
                    "sampled queries"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device, folder=None):
        """Samples go to `folder`/clocks_rank<device>.csv (a temporary folder when
        None); the summary is what the JSON line carries."""
        import tempfile

        self.device = device
        self.proc = None
        self.path = os.path.join(folder or tempfile.gettempdir(), f"clocks_rank{device}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def sweep_bytes(n, E, K):
    """Algorithmic bytes of one K-mpts sweep: the edge list once (u, v, w) plus,
    per mpts, a core column and the output tree (12 B per tree edge)."""
    return 12 * E + K * (4 * n + 12 * (n - 1))


def sweep_kernel_bytes(n, E, K):
    """Algorithmic bytes of the persistent kernel alone: the edge list once, the
    k-NN distance rows once (every core distance of a node is in its row), and the
    bit-packed tree membership (one 32-bit word per edge per pass of 32 MSTs)."""
    passes = (K + 31) // 32
    return 12 * E + 4 * 32 * n + 4 * E * passes


def config_of(name, w):
    """The workload description both arms print."""
    return {"workload": name, "n": w["n"], "dim": w["dim"], "k_max": w["k_max"], "mpts": f"1..{w['k_max']}",
            "l2": "inputs larger than L2 (edge list 12 B x |E|), no flush"}


# ---------------------------------------------------------------------------------------

def run_reference(args):
    """The reference's own CPU path (oracle/_ref: its sources compiled here) on the
    same workload: CoreSG::build, then CoreSG::mst per mpts (the `coresg_cli extract`
    loop); one step = one mpts value, all-in (edges(mpts) + MST)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from checkers import Reference
    from coresg_b200.datagen import workload

    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference built from source) is missing"}))
        return 0
    ref = Reference()
    pts, w = workload(args.workload, args.n)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    sg = ref.build(pts, k_max=w["k_max"], instances=1, iters=10, sample=16, seed=42, threads=0)
    build_s = time.perf_counter() - t0
    log(f"[reference] build {build_s:.2f}s {sg.times}")
    K = w["k_max"]
    mp = [1 + (i % K) for i in range(args.warmup + args.steps)]
    for m in mp[:args.warmup]:
        sg.mst(m, algo=0)
    secs = []
    for m in mp[args.warmup:]:
        r = sg.mst(m, algo=0)
        secs.append(r["seconds_all"])
    total = sum(secs)
    value = len(secs) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "MSTs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / len(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_of(args.workload, w),
        "step": "one CoreSG::mst(mpts) all-in, mpts cycling 1..k_max",
        "build_s": build_s,
        "cpu_baseline": {"value": value, "unit": "MSTs/s", "cores": cores, "kind": "reference",
                         "sample": f"{len(secs)} extractions (mpts {mp[args.warmup]}..), CoreSG::mst all-in"},
        "e2e": {"value": value, "unit": "MSTs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def cpu_baseline(g, pts, w, ids, dists, flags, counts, bridges):
    """The reference CPU extract on this CORE-SG (a bounded sample of mpts).  Returns
    the baseline and the reference's trees ({mpts: CoreSG::mst result}) for the
    parity check, or (None, {})."""
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from checkers import Reference
        from coresg_b200.datagen import pad_rows

        if not Reference.available():
            return None, {}
        ref = Reference()
        sg = ref.from_state(pad_rows(pts), w["dim"], ids, dists, flags, counts, bridges, threads=0)
        sample = [1, 8, 16, w["k_max"]]
        trees = {m: sg.mst(m, algo=0) for m in sample}
        secs = [trees[m]["seconds_all"] for m in sample]
        return ({"value": len(sample) / sum(secs), "unit": "MSTs/s", "cores": os.cpu_count() or 1,
                 "kind": "reference",
                 "sample": f"CoreSG::mst all-in for mpts {sample} on this CORE-SG ({sum(secs):.1f} s)"}, trees)
    except Exception as e:  # the baseline is reported, never required
        log(f"[cpu_baseline] failed: {e}")
        return None, {}


def parity_at_scale(g, mpts, ref_trees):
    """The engine's batched sweep against the reference's own CoreSG::mst on the same
    CORE-SG, for the mpts values the CPU baseline solved: the tree edges (as sorted
    (u, v) keys), the sorted weight bits, the labels and component count, the exact
    weight of the reference tree (canonical sum, bit for bit) and the reference's own
    double sum (within its reassociation error)."""
    if not ref_trees:
        return {"checked": False, "why": "reference CPU path unavailable"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from checkers import Oracle

    orc = Oracle()
    g.sweep_device(mpts)
    n = g.n

    def keys(e):
        return np.sort((e["u"].astype(np.uint64) << np.uint64(32)) | e["v"].astype(np.uint64))

    per = []
    for m, r in sorted(ref_trees.items()):
        mine = g.sweep_fetch(mpts.index(m))
        same_len = len(mine.edges) == len(r["edges"])
        chk = {
            "mpts": m, "tree_edges": int(len(mine.edges)),
            "edges": bool(same_len and np.array_equal(keys(mine.edges), keys(r["edges"]))),
            "weight_bits": bool(same_len and np.array_equal(np.sort(mine.edges["w"]).view(np.uint32),
                                                            np.sort(r["edges"]["w"]).view(np.uint32))),
            "labels": bool(np.array_equal(mine.component, r["labels"])),
            "components": bool(mine.num_components == r["ncomp"]),
            "exact_weight": bool(mine.weight == orc.exact_sum(r["edges"]["w"])),
            "reference_weight_rel": abs(mine.weight - r["weight"]) / max(1.0, abs(r["weight"])),
        }
        chk["equal"] = all(chk[x] for x in ("edges", "weight_bits", "labels", "components", "exact_weight"))
        per.append(chk)
    return {"checked": True, "mpts": sorted(ref_trees), "equal": all(c["equal"] for c in per), "per_mpts": per,
            "what": "batched sweep vs the reference CoreSG::mst on the same CORE-SG: tree edges, weight bits, "
                    "labels, components, exact weight"}


def run_inserts(cs, ctx, args):
    """The insert workload: a resident CORE-SG of the insert base (n=2M, d=32,
    k_max=24), then 16 seeded batches of U[10k, 200k] rows, odd batches from the
    base clusters and even ones from 10 new clusters; every batch is one cs_insert
    (NN-Descent insert, then the bridges re-selected).  Reports rows/s over all
    batches and the stages of each."""
    from coresg_b200.datagen import insert_batch, workload

    pts, w = workload(args.insert_workload, args.insert_n)
    g = cs.CoreSG(ctx, w["dim"], w["k_max"])
    rng = np.random.default_rng(w["seed"] + 1)
    sizes = [int(x) for x in rng.integers(10_000, 200_001, size=args.insert_batches)]
    # capacity for the base and every batch (Dataset::reserve): the inserts allocate
    # no device memory
    g.reserve(w["n"] + sum(sizes))
    t0 = time.perf_counter()
    g.build(pts, sample=16, iters=10, delta=0.001, seed=44)
    build_s = time.perf_counter() - t0
    del pts
    batches = [insert_batch(w, sz, 1000 + i, new_clusters=10 if i % 2 else 0) for i, sz in enumerate(sizes)]
    per, rows, secs = [], 0, 0.0
    for b in batches:
        t1 = time.perf_counter()
        g.insert(b)
        dt = time.perf_counter() - t1
        st = g.insert_stats()
        secs += dt
        rows += len(b)
        bs = g.bridge_stats()
        per.append({"rows": len(b), "ms": round(1000 * dt, 2),
                    **{k: round(v, 2) for k, v in st.items() if k.endswith("_ms") and k != "total_ms"},
                    "bridge_stages_ms": {k[:-3]: round(v, 3) for k, v in bs.items()
                                         if k.endswith("_ms") and k != "total_ms"},
                    "hub_refreshed": bs["hub_refreshed"], "rescored": bs["rescored"]})
    n_end = g.n
    g.close()
    return {"workload": args.insert_workload, "n_start": w["n"], "n_end": int(n_end), "k_max": w["k_max"],
            "build_s": build_s, "reserved_rows": w["n"] + sum(sizes), "batches": len(batches), "rows": rows,
            "seconds": secs,
            "rows_per_s": rows / secs if secs else None, "per_batch": per,
            "what": "cs_insert per batch: seeding search, instance descent, refinement, bridges re-selected"}


def run_highdim(cs, ctx, args):
    """The d=128 build: n=1M, k_max=16, f32 and its uint8 quantisation (values
    0..255 widened to f32 as the reference does; every partial sum of squared
    differences is an integer below 2^24, so the f32 distances are exact), each
    built on the device and swept over mpts 1..16."""
    from coresg_b200.datagen import quantize_u8, workload

    pts, w = workload("blobs1m_d128")
    out = {"workload": "blobs1m_d128", "n": w["n"], "dim": w["dim"], "k_max": w["k_max"]}
    for name, data in (("f32", pts), ("u8", quantize_u8(pts).astype(np.float32))):
        g = cs.CoreSG(ctx, w["dim"], w["k_max"])
        t0 = time.perf_counter()
        st = g.build(data, sample=8, iters=10, delta=0.001, seed=45)
        build_s = time.perf_counter() - t0
        mp = list(range(1, w["k_max"] + 1))
        g.sweep_device(mp)
        ms = [g.sweep_device(mp) for _ in range(3)]
        out[name] = {"build_s": build_s, "sweep_ms": float(np.median(ms)), "msts_per_s": len(mp) / (np.median(ms) / 1e3),
                     "edges": g.info()["knn_edges"], "bridges": st.get("bridges")}
        g.close()
    return out


def run_e2e(cs, ctx, g, mpts, arrays, steps, inflight, max_over_ranks, world, shape=None):
    """The batched sweep through the C ABI with host buffers (`arrays`: the graph's
    k-NN ids, dists, flags, counts and bridges).  A step is one
    cs_graph_set_knn + cs_graph_set_bridges from page-locked host arrays and one
    cs_extract_sweep into page-locked host outputs (all K trees and labels).
    `inflight` graphs, each with its own context (stream) and a host thread, run
    `steps` steps each, so one graph's uploads and downloads overlap another's sweep
    (the copy engines and the SMs work at once); inflight = 1 is the plain serial loop.
    Each graph runs one untimed step first (its plan is captured there).  Throughput
    = all MSTs / the wall time of the region, max over ranks; `serial` is the same
    loop with one graph.  `shape` (flatten divisor, block) is set on the added
    graphs when the main one was given it; otherwise they take the autotuned shape
    cached for this graph size."""
    import threading

    K, n = len(mpts), g.n

    def pinned_copy(a):
        p = cs.Pinned(a.shape, a.dtype)
        p.array[...] = a
        return p

    host_in = [pinned_copy(a) for a in arrays]
    p_ids, p_dists, p_flags, p_counts, p_bridges = (p.array for p in host_in)
    h2d = sum(p.array.nbytes for p in host_in)
    ctxs = [ctx] + [cs.Context(ctx.device) for _ in range(inflight - 1)]
    graphs = [g] + [cs.CoreSG(c, g.dim, g.k_max) for c in ctxs[1:]]
    if shape:
        for gg in graphs[1:]:
            gg.set_sweep_shape(*shape)
    outs = [(cs.Pinned((K, max(n - 1, 1)), cs.EDGE_DTYPE), cs.Pinned((K, n), np.uint32)) for _ in graphs]
    d2h = [0]

    def step(w):
        gg, (oe, ol) = graphs[w], outs[w]
        gg.set_knn(p_ids, p_dists, p_flags, p_counts)
        gg.set_bridges(p_bridges)
        res = gg.all_msts(mpts, labels=True, out_edges=oe.array, out_labels=ol.array)
        d2h[0] = sum(r.edges.nbytes + r.component.nbytes + 20 for r in res)

    errors = []

    def worker(w):
        try:
            for _ in range(steps):
                step(w)
        except Exception as ex:  # surfaced after the join
            errors.append(repr(ex))

    def timed(ws):
        th = [threading.Thread(target=worker, args=(w,)) for w in ws]
        t0 = time.perf_counter()
        for t in th:
            t.start()
        for t in th:
            t.join()
        return time.perf_counter() - t0

    try:
        for w in range(len(graphs)):
            step(w)  # untimed: plan capture
        serial_s = max_over_ranks(timed([0]))
        piped_s = max_over_ranks(timed(range(len(graphs)))) if inflight > 1 else serial_s
        if errors:
            raise RuntimeError("e2e step failed: " + errors[0])
    finally:
        for p in host_in + [x for o in outs for x in o]:
            p.free()
        for gg in graphs[1:]:
            gg.close()
        for c in ctxs[1:]:
            c.close()
    return {"value": world * K * steps * len(graphs) / piped_s, "unit": "MSTs/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h[0]), "steps": steps * len(graphs), "inflight": len(graphs),
            "serial": {"value": world * K * steps / serial_s, "steps": steps},
            "what": f"cs_graph_set_knn + cs_graph_set_bridges + cs_extract_sweep (trees and labels) per step, page-locked host buffers; {len(graphs)} graph(s) on their own contexts in flight"}


def run_partitioned(cs, args, ranks):
    """--gpus N > 1: one CORE-SG on N GPUs (coresg_b200/partition.py).  Rank 0 builds
    the workload's CORE-SG on its GPU and its state (k-NN arrays and bridges) is
    broadcast over NCCL, so every rank holds the same graph.  A step is one sweep of
    mpts 1..K split across the ranks (rank r sweeps positions r, r + N, ...) followed by
    the gather of every tree, label array and scalar triple into rank 0's device memory
    (NCCL gather).  Each rank times its steps with CUDA events on its engine stream,
    which the fetch and the gather run on too; the job's time is the maximum over
    ranks, and value = K MSTs per step over it (strong scaling: the work per step is
    fixed as N grows).  Rank 0 then checks the gathered results against a one-GPU
    sweep of all K on its own graph."""
    import torch

    from coresg_b200 import partition
    from coresg_b200.datagen import workload

    world, rank, local = ranks.world, ranks.rank, ranks.local
    dist = ranks.group
    dev = f"cuda:{local}"
    ctx = cs.Context(local)
    pts, w = workload(args.workload, args.n)
    n, K = w["n"], w["k_max"]
    mpts = list(range(1, K + 1))
    g = cs.CoreSG(ctx, w["dim"], K)
    state, build_s = None, None
    if rank == 0:
        t0 = time.perf_counter()
        g.build(pts, sample=16, iters=10, delta=0.001, seed=42)
        build_s = time.perf_counter() - t0
        ids, dists, flags, counts = g.knn()
        state = [ids, dists, flags, counts, g.missing_edges().view(np.uint32)]
    ranks.barrier()
    t0 = time.perf_counter()
    got = partition.broadcast_arrays(dist, state, dev)
    torch.cuda.synchronize(dev)
    replicate_s = ranks.max_over_ranks(time.perf_counter() - t0)
    state_bytes = sum(a.nbytes for a in got)
    if rank != 0:
        g.set_knn(*got[:4])
        g.set_bridges(got[4].view(cs.EDGE_DTYPE))
    info = g.info()
    E = info["knn_edges"] + info["bridges"]
    pos = partition.share_positions(K, world, rank)
    mine = [mpts[j] for j in pos]
    bufs = partition.ResultBuffers(partition.max_share(K, world), n, dev)
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    gathered = [None]

    def step():
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            ev0.record(ext)
            if mine:
                g.sweep_device(mine)
                partition.fetch_share(g, range(len(mine)), bufs)
            gathered[0] = partition.gather_results(dist, K, bufs)
            ev1.record(ext)
        ev1.synchronize()
        return ev0.elapsed_time(ev1)

    for _ in range(args.warmup):
        step()
    clk = Clocks(local, args.clocks_dir)
    ranks.barrier()
    torch.cuda.synchronize(dev)
    launches0 = ctx.launches
    clk.start()
    ms = [step() for _ in range(args.steps)]
    clocks = clk.stop()
    launches = ranks.sum_over_ranks(ctx.launches - launches0)
    ranks.barrier()
    total_ms = ranks.max_over_ranks(sum(ms))
    value = K * args.steps / (total_ms / 1000.0)
    sweep_ms = ranks.max_over_ranks(float(np.mean([g.sweep_timing()[0]])) if mine else 0.0)

    check = None
    if rank == 0:
        edges, labels, scalars = gathered[0]
        alone = g.all_msts(mpts)
        ok = True
        for j, r in enumerate(alone):
            ne = int(scalars[j, 0])
            ok &= ne == len(r.edges) and int(scalars[j, 1]) == r.num_components
            ok &= float(scalars[j, 2]) == r.weight
            ok &= partition.unpack(edges[j], ne).tobytes() == r.edges.tobytes()
            ok &= np.array_equal(labels[j].cpu().numpy().view(np.uint32), r.component)
        check = {"equal": bool(ok), "what": "gathered trees, labels and scalars vs a one-GPU sweep of all K "
                                            "on rank 0's graph"}
    gather_bytes = (world - 1) * bufs.L * (bufs.edges[0].numel() * 4 + bufs.labels[0].numel() * 4 + 24)

    # e2e through the public API: every rank uploads the CORE-SG from page-locked host
    # arrays (cs_graph_set_knn + cs_graph_set_bridges) and extracts its share into
    # page-locked host outputs (cs_extract_sweep); wall time, max over ranks
    e2e = None
    if args.e2e_steps > 0 and mine:
        host = [cs.Pinned(a.shape, a.dtype) for a in got]
        for p_, a in zip(host, got):
            p_.array[...] = a
        oe = cs.Pinned((len(mine), max(n - 1, 1)), cs.EDGE_DTYPE)
        ol = cs.Pinned((len(mine), n), np.uint32)

        def e2e_step():
            g.set_knn(*(p_.array for p_ in host[:4]))
            g.set_bridges(host[4].array.view(cs.EDGE_DTYPE))
            return g.all_msts(mine, labels=True, out_edges=oe.array, out_labels=ol.array)

        e2e_step()
        ranks.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            res = e2e_step()
        e2e_s = ranks.max_over_ranks(time.perf_counter() - t0)
        d2h = ranks.sum_over_ranks(sum(r.edges.nbytes + r.component.nbytes + 20 for r in res))
        e2e = {"value": K * args.e2e_steps / e2e_s, "unit": "MSTs/s",
               "h2d_bytes_per_step": int(world * state_bytes), "d2h_bytes_per_step": int(d2h),
               "steps": args.e2e_steps,
               "what": "every rank: cs_graph_set_knn + cs_graph_set_bridges from page-locked host arrays and "
                       "cs_extract_sweep of its mpts share into page-locked host outputs"}
        for p_ in host + [oe, ol]:
            p_.free()
    elif args.e2e_steps > 0:
        # a rank without a share still takes the same collective steps
        ranks.barrier()
        ranks.max_over_ranks(0.0)
        ranks.sum_over_ranks(0.0)
    if rank == 0:
        peak, peak_kind = peaks()
        line = {
            "metric": METRIC, "value": value, "unit": "MSTs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(args.workload, w),
            "graph": {"edges": E, "knn_edges": info["knn_edges"], "bridges": info["bridges"]},
            "multi_gpu": {"mode": "mpts partition + gather to rank 0", "ranks": world,
                          "mpts_per_rank": [len(partition.share_positions(K, world, r)) for r in range(world)],
                          "replicate_s": replicate_s, "replicated_bytes": int(state_bytes),
                          "gather_bytes_per_step": int(gather_bytes), "sweep_ms_max_over_ranks": sweep_ms,
                          "check": check},
            "build_s": build_s, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "roofline": None, "cpu_baseline": None,
            "roofline_note": f"see the one-GPU line; peak source {peak_kind} {peak} GB/s",
        }
        print(json.dumps(line))
    del bufs, gathered
    g.close()
    ranks.close()
    return 0


def run_serving(cs, ctx, args):
    """The serving workload: a resident CORE-SG of the serve workload, Poisson
    arrivals (extract(mpts ~ U{1..k_max}), a quarter of them epsilon-cuts at a random
    merge-height quantile, and 10% insert batches of log-uniform size) submitted on
    schedule from one host thread; a second thread waits on the tickets.  Latency =
    (submit - scheduled arrival) + the server's submit-to-result time."""
    import queue
    import threading

    from coresg_b200.datagen import insert_batch, workload
    from coresg_b200.serving import CS_REQ_EPS_LABELS, CS_REQ_INSERT, Pinned, Server, percentile, request_stream

    pts, w = workload(args.serve_workload)
    n0, K = w["n"], w["k_max"]
    g = cs.CoreSG(ctx, w["dim"], K)
    t0 = time.perf_counter()
    g.build(pts, sample=16, iters=10, delta=0.001, seed=43)
    build_s = time.perf_counter() - t0
    del pts
    stream = request_stream(args.serve_seconds, args.serve_rate, K, seed=w["seed"])
    batches = {i: insert_batch(w, a.size, a.seed) for i, a in enumerate(stream) if a.kind == CS_REQ_INSERT}
    n_max = n0 + sum(len(b) for b in batches.values())
    # capacity for every row the stream will insert (Dataset::reserve), so the window
    # allocates no device memory; the sweep below then sizes its buffers for it too
    g.reserve(n_max)
    # epsilon values: quantiles of each mpts tree's merge heights on the built graph
    mp = list(range(1, K + 1))
    g.sweep_device(mp)
    grid = np.linspace(0.0, 1.0, 101)
    qs = {m: np.quantile(g.sweep_fetch(m - 1, labels=False).edges["w"][::16], grid) for m in mp}
    pool = [Pinned((3 * n_max,), np.uint32) for _ in range(args.serve_buffers)]
    free = queue.Queue()
    for i in range(len(pool)):
        free.put(i)
    srv = Server(g, max_batch=32, max_slots=64, inserts_first=bool(args.serve_inserts_first))
    done, sent = queue.Queue(), queue.Queue()

    def waiter():
        while True:
            item = sent.get()
            if item is None:
                return
            ticket, arr, buf, t_sub = item
            r = srv.wait(ticket)
            if buf is not None:
                free.put(buf)
            done.put((arr, (t_sub - arr.t) * 1000.0 + r["latency_ms"], r, time.perf_counter()))

    th = threading.Thread(target=waiter)
    th.start()
    t_start = time.perf_counter()
    for i, a in enumerate(stream):
        delay = t_start + a.t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        buf = None
        if a.kind == CS_REQ_INSERT:
            ticket = srv.insert(batches.pop(i))
        else:
            buf = free.get()
            arr = pool[buf].array
            if a.kind == CS_REQ_EPS_LABELS:
                eps = float(np.interp(a.quantile, grid, qs[a.mpts]))
                ticket = srv.cut(a.mpts, eps, arr[:n_max])
            else:
                ticket = srv.extract(a.mpts, arr.view(cs.EDGE_DTYPE))
        sent.put((ticket, a, buf, time.perf_counter() - t_start))
    sent.put(None)
    th.join()
    st = srv.stats()
    srv.close()
    qlat, ilat, failed, t_last = [], [], 0, t_start
    while not done.empty():
        arr, ms, r, t_done = done.get()
        failed += r["status"] != 0
        (ilat if arr.kind == CS_REQ_INSERT else qlat).append(ms)
        t_last = max(t_last, t_done)
    for p_ in pool:
        p_.free()
    drain = t_last - t_start
    return {
        "workload": args.serve_workload, "n_start": n0, "n_end": int(g.n), "k_max": K, "build_s": build_s,
        "window_s": args.serve_seconds, "rate_per_s": args.serve_rate,
        "consistency": "inserts_first" if args.serve_inserts_first else "arrival_order",
        "requests": len(stream), "queries": len(qlat), "inserts": len(ilat), "failed": failed,
        "p50_query_ms": percentile(qlat, 50), "p99_query_ms": percentile(qlat, 99),
        "p50_insert_ms": percentile(ilat, 50), "p99_insert_ms": percentile(ilat, 99),
        "p50_ms": percentile(qlat + ilat, 50), "p99_ms": percentile(qlat + ilat, 99),
        "msts_per_s": len(qlat) / drain if drain > 0 else None, "drain_s": drain,
        "sweeps": st["batches"], "batches_from_last_sweep": st["reused_batches"],
        "mean_batch": (st["queries"] / (st["batches"] + st["reused_batches"]))
        if st["batches"] + st["reused_batches"] else None,
        "max_batch": st["max_batch_seen"], "insert_batches": st["insert_batches"],
        "inserted_rows": st["inserted_rows"], "sweep_ms_total": st["sweep_ms"], "insert_ms_total": st["insert_ms"],
        "result_buffers": args.serve_buffers, "result": "extract: tree edges; epsilon-cut: labels (pinned host)",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="blobs1m_d16")
    ap.add_argument("--n", type=int, default=None, help="override the workload's point count")
    ap.add_argument("--e2e-steps", type=int, default=10, help="e2e steps per graph in flight (0: skip)")
    ap.add_argument("--e2e-inflight", type=int, default=3, help="e2e graphs in flight, each on its own context")
    ap.add_argument("--clocks-dir", default=None, help="folder for the raw nvidia-smi samples (default: a temp folder)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--flatten", type=int, default=0, help="sweep flatten divisor (0: autotune)")
    ap.add_argument("--block", type=int, default=0, help="sweep block size (0: autotune)")
    ap.add_argument("--serve-workload", default="blobs4m_d16")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="serving window (0: skip the serving leg)")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-buffers", type=int, default=96, help="pinned host result buffers")
    ap.add_argument("--serve-inserts-first", type=int, default=1)
    ap.add_argument("--insert-workload", default="blobs2m_d32")
    ap.add_argument("--insert-batches", type=int, default=16, help="insert leg batches (0: skip)")
    ap.add_argument("--insert-n", type=int, default=None, help="override the insert workload's base point count")
    ap.add_argument("--highdim", type=int, default=1, help="d=128 f32/u8 build leg (0: skip)")
    ap.add_argument("--ref-gpu", type=int, default=1,
                    help="time the reference's own CUDA NN-Descent (built for sm_100a) once (0: skip)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import coresg_b200 as cs
    from coresg_b200 import replicas
    from coresg_b200.datagen import workload

    ranks = replicas.from_env("nccl", timeout_s=300)
    if ranks.world > 1:
        return run_partitioned(cs, args, ranks)
    world, rank, local = ranks.world, ranks.rank, ranks.local
    barrier, max_over_ranks = ranks.barrier, ranks.max_over_ranks

    ctx = cs.Context(local)
    pts, w = workload(args.workload, args.n)
    n, K = w["n"], w["k_max"]
    mpts = list(range(1, K + 1))
    g = cs.CoreSG(ctx, w["dim"], K)

    # ---- build (device): NN-Descent + bridges.  A small untimed build first loads the
    # library's kernels (a one-time cost of the process, reported as first_use_s)
    t0 = time.perf_counter()
    warm = cs.CoreSG(ctx, w["dim"], K)
    warm.build(pts[:20000], sample=16, iters=2, delta=0.001, seed=7)
    warm.close()
    first_use_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    st = g.build(pts, sample=16, iters=10, delta=0.001, seed=42)
    build_s = time.perf_counter() - t0
    # the same build again on the same resident graph: no fresh device allocations
    t0 = time.perf_counter()
    st = g.build(pts, sample=16, iters=10, delta=0.001, seed=42)
    rebuild_s = time.perf_counter() - t0
    bstats = g.build_stats()
    d_pts = w["dim"]
    bstats["gflops"] = 3.0 * d_pts * bstats["distance_evals"] / (bstats["device_ms"] / 1000.0) / 1e9
    bstats["evals_per_node_round"] = bstats["distance_evals"] / (n * max(st.get("rounds", 1), 1))
    recall = build_recall(g, pts, local, queries=10000, seed=7) if rank == 0 else None
    info = g.info()
    E = info["knn_edges"] + info["bridges"]
    log(f"[rank {rank}] build {build_s:.3f}s (again on the same graph {rebuild_s:.3f}s) {st} |E|={E}")

    # ---- batched sweep
    if args.flatten and args.block:
        flatten, block = args.flatten, args.block
        g.set_sweep_shape(flatten, block)
    else:
        flatten, block = g.autotune(mpts)
    log(f"[rank {rank}] sweep shape flatten_div={flatten} block={block}")
    for _ in range(args.warmup):
        g.sweep_device(mpts)
    clk = Clocks(local, args.clocks_dir)
    barrier()
    launches0 = ctx.launches
    clk.start()
    t_wall = time.perf_counter()
    step_ms, kern_ms = [], []
    for _ in range(args.steps):
        step_ms.append(g.sweep_device(mpts))
        kern_ms.append(g.sweep_timing()[1])
    wall = time.perf_counter() - t_wall
    clocks = clk.stop()
    launches = ctx.launches - launches0
    barrier()
    total_ms = max_over_ranks(sum(step_ms))
    value = replicas.replica_throughput(world, K, args.steps, total_ms)
    ms_per_step = total_ms / args.steps
    kernel_ms = float(np.mean(kern_ms))
    log(f"[rank {rank}] sweep {ms_per_step:.3f} ms/step (kernel {kernel_ms:.3f} ms) wall {wall:.3f}s")
    # per-round profile of the last timed sweep's persistent kernel (cs_sweep_trace)
    trace = [{"phase_a_ms": int(t[0]) / 1e6, "phase_b_ms": int(t[1]) / 1e6, "flatten_ms": int(t[2]) / 1e6,
              "edges": int(t[3]), "roots": int(t[4]), "full_flatten": int(t[5]) & 1,
              "phase_a_walk": ("edges", "edges + tail table", "tail entries")[min(int(t[5]) >> 1, 2)],
              "live_pairs": int(t[6])}
             for t in g.sweep_trace()]

    # ---- plain per-mpts path on the same graph (one pass over 1..K)
    plain = None
    if not args.no_plain:
        ctx_l0 = ctx.launches
        t1 = time.perf_counter()
        for m in mpts:
            cs.lib().cs_extract(g.h, m, None, None, None, None, None)
        plain_s = time.perf_counter() - t1
        plain = {"value": K / plain_s, "unit": "MSTs/s", "ms_per_mst": 1000 * plain_s / K,
                 "kernel_launches": ctx.launches - ctx_l0,
                 "what": "cs_extract per mpts: edges(mpts) materialised, Boruvka rounds host-driven"}

    # ---- e2e through the C ABI with host buffers (run_e2e): every step uploads the
    # CORE-SG's k-NN arrays and bridges and downloads all K trees and labels
    ids, dists, flags, counts = g.knn()
    bridges = g.missing_edges()
    e2e = None
    if args.e2e_steps > 0:
        shape = (args.flatten, args.block) if args.flatten and args.block else None
        e2e = run_e2e(cs, ctx, g, mpts, (ids, dists, flags, counts, bridges), args.e2e_steps, args.e2e_inflight,
                      max_over_ranks, world, shape)

    # ---- roofline of the persistent kernel
    peak, peak_kind = peaks()
    kb = sweep_kernel_bytes(n, E, K)
    achieved = kb / (kernel_ms / 1000.0) / 1e9
    prof = profiled_traffic(args.workload, n)
    roofline = {"bound": "hbm", "kernel": "k_sweep (persistent Boruvka, 32 MSTs, lane = MST)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes": kb, "kernel_ms": kernel_ms,
                "traffic": prof[0] if prof else None,
                "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/{prof[1]}" if prof else None,
                # the bytes the kernel actually moves (every round re-reads the live edges)
                # over its time, against the same peak
                "traffic_gbs": prof[0] / (kernel_ms / 1000.0) / 1e9 if prof else None,
                "traffic_frac": prof[0] / (kernel_ms / 1000.0) / 1e9 / peak if prof else None,
                "sweep_graph": {"algorithmic_bytes": sweep_bytes(n, E, K), "ms": ms_per_step,
                                "achieved_gbs": sweep_bytes(n, E, K) / (ms_per_step / 1000.0) / 1e9}}

    # ---- the build's FP32 roofline: 3 d FLOP per distance evaluation of the local
    # joins (NNDescentStats::distance_evals) over the descent's device time (sample,
    # join and merge kernels of every round), against the FP32 CUDA-core peak at the
    # SM clock sampled during the sweep (128 FP32 lanes x 2 FLOP per SM per cycle)
    sm_count = cs.device_props(local)["sm_count"]
    clk_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    fp32_peak = sm_count * 128 * 2 * clk_mhz * 1e6 / 1e12
    build_roofline = {"bound": "fp32", "achieved": bstats["gflops"] / 1e3, "peak": fp32_peak, "unit": "TFLOP/s",
                      "frac": bstats["gflops"] / 1e3 / fp32_peak,
                      "peak_source": f"{sm_count} SMs x 128 FP32 lanes x 2 FLOP x {clk_mhz:.0f} MHz (sampled)",
                      "what": "3 d x distance evaluations over the descent's device time (sample + join + merge)"}

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, ref_trees = cpu_baseline(g, pts, w, ids, dists, flags, counts, bridges)
        parity = parity_at_scale(g, mpts, ref_trees)
        log(f"[rank {rank}] parity at n={n}: {parity.get('equal')}")
    ref_gpu = None
    if rank == 0 and world == 1 and args.ref_gpu:
        ref_gpu = reference_gpu_build(cs, ctx, local, pts, w)
        log(f"[rank {rank}] reference GPU build {ref_gpu}")

    serving = inserts = highdim = None
    g.close()
    # the serving, insert and d=128 legs describe one GPU: only a single-rank run has them
    if world > 1:
        args.serve_seconds, args.insert_batches, args.highdim = 0, 0, 0
    if args.serve_seconds > 0:
        serving = run_serving(cs, ctx, args)
        log(f"[rank {rank}] serving {serving}")
    if args.insert_batches > 0:
        inserts = run_inserts(cs, ctx, args)
        log(f"[rank {rank}] inserts {dict((k, v) for k, v in inserts.items() if k != 'per_batch')}")
    if args.highdim:
        highdim = run_highdim(cs, ctx, args)
        log(f"[rank {rank}] highdim {highdim}")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "MSTs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(args.workload, w),
            "graph": {"edges": E, "knn_edges": info["knn_edges"], "bridges": info["bridges"]},
            "sweep_shape": {"flatten_div": flatten, "block": block},
            "sweep_trace": trace,
            "parity": parity,
            "build_s": build_s, "rebuild_s": rebuild_s, "build": st, "build_device": bstats,
            "build_roofline": build_roofline,
            "build_reference_gpu": ref_gpu,
            "build_reference_gpu_s": (ref_gpu or {}).get("reference_nndescent_gpu_s"),
            "build_recall": recall, "first_use_s": first_use_s,
            "plain": plain, "speedup_vs_plain": (value / world) / plain["value"] if plain else None,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "p50_query_ms": serving["p50_query_ms"] if serving else None,
            "p99_query_ms": serving["p99_query_ms"] if serving else None, "serving": serving,
            "inserts": inserts, "highdim": highdim,
            "clocks": clocks, "wall_s_timed": wall,
        }
        print(json.dumps(line))
    ranks.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
