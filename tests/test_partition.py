"""The multi-GPU partition of a sweep (coresg_b200/partition.py) on the host: two
gloo ranks on CPU stand in for two GPUs.  Rank 0's CORE-SG state is broadcast, each
rank solves its strided share of the mpts values (the oracle's MST stands in for the
device sweep), and rank 0 gathers the trees, labels and scalars: they equal a 1-rank
computation of all K values, in the requested order."""
import os
import socket
import sys

import numpy as np
import pytest

from coresg_b200 import partition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MPTS = [1, 2, 4, 8, 16, 32, 3]


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("K", [1, 2, 5, 7, 16, 32, 33])
@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shares_cover_every_position_once(K, world):
    seen = []
    for r in range(world):
        pos = partition.share_positions(K, world, r)
        assert len(pos) <= partition.max_share(K, world)
        seen += pos
    assert sorted(seen) == list(range(K))
    mp = list(range(1, K + 1))
    assert sorted(sum((partition.mpts_share(mp, world, r) for r in range(world)), [])) == mp


def solve(oracle, state, m, n):
    """Stand-in for one MST of a rank's sweep: the oracle's tree (ascending edge
    index), labels and scalars."""
    ids, dists, flags, counts, bridges = state
    e = oracle.edges(m, ids, dists, counts, bridges)
    o = oracle.mst(e, n)
    return e[o["in_tree"]], o["labels"], (o["nedges"], o["ncomp"], o["weight"])


def _rank_main(rank, world, port, out):
    for p in (os.path.join(ROOT, "incremental-core-sg_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch  # noqa: F401
    from checkers import Oracle
    from conftest import load_golden
    from coresg_b200 import partition as part
    from coresg_b200 import replicas

    r = replicas.from_env("gloo", timeout_s=60)
    try:
        dist = r.group
        z = load_golden("coresg_n6000_d16_k32") if rank == 0 else None
        src = [z["ids"], z["dists"], z["flags"], z["counts"], z["bridges"].view(np.uint32)] if rank == 0 else None
        got = part.broadcast_arrays(dist, src, "cpu")
        state = got[:4] + [got[4].view(partition_edge_dtype())]
        n = len(state[3])
        oracle = Oracle()
        K = len(MPTS)
        pos = part.share_positions(K, world, rank)
        bufs = part.ResultBuffers(part.max_share(K, world), n, "cpu")
        for i, j in enumerate(pos):
            tree, lab, sc = solve(oracle, state, MPTS[j], n)
            bufs.edges[i, :len(tree)] = torch_words(tree)
            bufs.labels[i] = torch_words(lab)
            bufs.scalars[i] = torch_scalars(sc)
        res = part.gather_results(dist, K, bufs)
        if rank == 0:
            edges, labels, scalars = res
            ok = True
            for j, m in enumerate(MPTS):
                tree, lab, sc = solve(oracle, state, m, n)
                ne = int(scalars[j, 0])
                ok &= ne == len(tree) and int(scalars[j, 1]) == sc[1] and float(scalars[j, 2]) == sc[2]
                ok &= part.unpack(edges[j], ne).tobytes() == tree.tobytes()
                ok &= np.array_equal(labels[j].numpy().view(np.uint32), lab)
            out.put(("gather", bool(ok)))
        else:
            # the broadcast delivered rank 0's state bit for bit
            zz = load_golden("coresg_n6000_d16_k32")
            same = all(np.array_equal(a, b) for a, b in zip(state[:4], (zz["ids"], zz["dists"], zz["flags"],
                                                                         zz["counts"])))
            same &= state[4].tobytes() == zz["bridges"].tobytes()
            out.put(("broadcast", bool(same)))
        r.barrier()
    finally:
        r.close()


def partition_edge_dtype():
    from checkers import EDGE_DTYPE

    return EDGE_DTYPE


def torch_words(a):
    import torch

    w = np.ascontiguousarray(a).view(np.int32).reshape(len(a), -1)
    return torch.from_numpy(w if w.shape[1] > 1 else np.ascontiguousarray(w[:, 0]))


def torch_scalars(sc):
    import torch

    return torch.tensor([float(sc[0]), float(sc[1]), float(sc[2])], dtype=torch.float64)


def test_two_gloo_ranks_broadcast_partition_and_gather():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    import queue
    import time

    got = {}
    try:
        t_end = time.time() + 240
        while len(got) < len(procs) and time.time() < t_end:
            try:
                k, v = out.get(timeout=2)
                got[k] = v
            except queue.Empty:
                if any(p.exitcode not in (None, 0) for p in procs):
                    break  # a rank failed: its traceback is in the captured output
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    assert got == {"gather": True, "broadcast": True}
