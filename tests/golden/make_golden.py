"""Generate the golden fixtures in this directory by running the reference's own
CPU code (the reference sources compiled by oracle/Makefile into
oracle/_ref/libcoresg_ref.so; driven through oracle/ref_harness.cpp).

    python tests/golden/make_golden.py

Each fixture holds a CORE-SG built by the reference (points, k-NN arrays, bridges),
the reference's hubness/connectivity state, and for several mpts the reference's
core distances, CoreSG::edges(mpts) checksum, Boruvka MST (edge keys, sorted weight
bits, labels, component count, discovery-order weight).  The reference NN-Descent's
exhaustive recall on small sets is stored for the k-NN recall bar.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "incremental-core-sg_b200"))

from checkers import EDGE_DTYPE, Oracle, Reference  # noqa: E402
from coresg_b200.datagen import gaussian_mixture  # noqa: E402

CASES = {
    # name: (n, dim, clusters, sigma, noise, k_max, seed, mpts list)
    "coresg_n3000_d24_k16": (3000, 24, 8, (0.2, 1.0), 0.05, 16, 11, [1, 2, 4, 8, 16]),
    "coresg_n6000_d16_k32": (6000, 16, 12, (0.2, 1.0), 0.05, 32, 12, [1, 2, 3, 8, 16, 31, 32]),
    # well separated, no noise, small k: the k-NN graph falls apart and the
    # bridges plus the connectivity repair have real work to do
    "coresg_n2500_d8_k6_split": (2500, 8, 6, (0.05, 0.1), 0.0, 6, 13, [1, 2, 3, 6]),
    # d=40 (stride 40: one 16-block, one 16-block, one 8-wide tail)
    "coresg_n2000_d40_k10": (2000, 40, 5, (0.5, 2.0), 0.02, 10, 14, [1, 5, 10]),
}

RECALL_CASES = {
    # name: (n, dim, clusters, sigma, noise, k, sample, iters, seeds)
    "recall_n20000_d16_k32": (20000, 16, 20, (0.2, 1.0), 0.05, 32, 16, 10, [42, 43, 44]),
    "recall_n20000_d24_k32": (20000, 24, 20, (0.2, 1.0), 0.05, 32, 16, 10, [42, 43, 44]),
}


def edge_keys(e: np.ndarray) -> np.ndarray:
    return np.sort((e["u"].astype(np.uint64) << np.uint64(32)) | e["v"].astype(np.uint64))


def make_case(ref: Reference, orc: Oracle, name, spec):
    n, dim, clusters, sigma, noise, k, seed, mpts_list = spec
    pts = gaussian_mixture(n, dim, clusters, sigma, noise, seed=seed)
    sg = ref.build(pts, k_max=k, instances=1, iters=10, sample=16, seed=42, threads=4)
    padded = sg.points()
    ids, dists, flags, counts = sg.knn()
    bridges = sg.bridges()
    score, rdeg = sg.scores()
    conn, ncomp = sg.conn_labels()
    # points are regenerated from the seeded generator; the checksum guards drift
    out = dict(points_sha=np.frombuffer(hashlib.sha256(pts.tobytes()).digest(), np.uint8),
               spec=np.array([n, dim, clusters, seed], np.int64), sigma=np.array(sigma),
               noise=np.float64(noise), dim=np.uint32(dim), k=np.uint32(k),
               ids=ids, dists=dists, flags=flags, counts=counts, bridges=bridges.view(np.uint8),
               repair=np.uint64(sg.repair_count()), selected=sg.selected(), score=score, rdeg=rdeg,
               conn=conn, ncomp_knn=np.uint32(ncomp), mpts=np.array(mpts_list, np.uint32),
               undirected=np.uint64(len(orc.undirected(ids, dists, counts))))
    for m in mpts_list:
        e = sg.edges(m)
        r = sg.mst(m, algo=1, threads=4)
        out[f"core_{m}"] = sg.core(m)
        out[f"edges_len_{m}"] = np.uint64(len(e))
        out[f"edges_sha_{m}"] = np.frombuffer(hashlib.sha256(e.tobytes()).digest(), np.uint8)
        out[f"mst_keys_{m}"] = edge_keys(r["edges"])
        out[f"mst_wbits_{m}"] = np.sort(r["edges"]["w"]).view(np.uint32)
        out[f"mst_labels_{m}"] = r["labels"]
        out[f"mst_ncomp_{m}"] = np.uint32(r["ncomp"])
        out[f"mst_weight_{m}"] = np.float64(r["weight"])
        print(f"  {name} mpts={m}: |E|={len(e)} tree={len(r['edges'])} comps={r['ncomp']} "
              f"w={r['weight']:.6f}")
    if n <= 3000:  # one full edge list, for element-wise comparisons
        out["edges_full_mpts"] = np.uint32(mpts_list[len(mpts_list) // 2])
        out["edges_full"] = sg.edges(int(out["edges_full_mpts"])).view(np.uint8)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: n={n} d={dim} k={k} bridges={len(bridges)} repair={sg.repair_count()} "
          f"knn components={ncomp}")


def make_recall(ref: Reference, orc: Oracle, name, spec):
    n, dim, clusters, sigma, noise, k, sample, iters, seeds = spec
    pts = gaussian_mixture(n, dim, clusters, sigma, noise, seed=seeds[0] + 1000)
    recalls = []
    for s in seeds:
        ids, dists, counts, evals, sec = ref.nndescent(pts, k=k, sample=sample, iters=iters, seed=s,
                                                       threads=4)
        recalls.append(ref.sampled_recall(pts, ids, dists, counts, k, queries=n, threads=8))
    out = dict(points_sha=np.frombuffer(hashlib.sha256(pts.tobytes()).digest(), np.uint8),
               spec=np.array([n, dim, clusters, seeds[0] + 1000], np.int64), sigma=np.array(sigma),
               noise=np.float64(noise), k=np.uint32(k), sample=np.uint32(sample), iters=np.uint32(iters),
               seeds=np.array(seeds, np.uint64), ref_recall=np.array(recalls, np.float64))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: reference NN-Descent exhaustive recall@{k} per seed = {recalls}")


def main():
    ref = Reference()
    orc = Oracle()
    for name, spec in CASES.items():
        make_case(ref, orc, name, spec)
    for name, spec in RECALL_CASES.items():
        make_recall(ref, orc, name, spec)


if __name__ == "__main__":
    main()
