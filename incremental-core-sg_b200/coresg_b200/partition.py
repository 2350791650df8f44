"""Multi-GPU extraction: the CORE-SG replicated on every rank, the mpts values of a
sweep partitioned across the ranks, and the trees gathered into rank 0's memory.

The K MSTs of a sweep are independent units (CoreSG::all_msts, src/coresg.cpp:412-417,
runs them as K separate extractions; the reference's JobScheduler gives one slot per
device, include/coresg/backend.hpp:131-169).  So a job of one CORE-SG on N GPUs:

1. rank 0 builds the CORE-SG, and its state -- padded points, k-NN arrays, bridges --
   is broadcast to every rank (one collective per array; NCCL over NVLink between
   GPUs, gloo between host processes), so every rank holds the same graph;
2. every rank sweeps its share of the mpts values (a strided split: rank r takes
   positions r, r + N, r + 2N, ...), one persistent launch per pass of <= 32 MSTs;
3. the trees (n - 1 edges each), labels (n each) and per-MST scalars (edge count,
   component count, exact weight) are gathered into rank 0's device memory, which
   then holds the K results in the order of the requested mpts.

Nothing here uses multicast.  The functions take torch tensors and a process group
(torch.distributed), so the same code runs over NCCL on GPUs and over gloo on the
host, where the tests run it with CPU stand-in results.
"""
from __future__ import annotations

import numpy as np

EDGE_WORDS = 3  # a cs_edge is three 32-bit words (u, v, weight bits)


def share_positions(K: int, world: int, rank: int) -> list[int]:
    """Positions of the K requested mpts values that `rank` sweeps (strided split)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return list(range(rank, K, world))


def mpts_share(mpts, world: int, rank: int) -> list[int]:
    """The mpts values `rank` sweeps."""
    mp = list(mpts)
    return [mp[i] for i in share_positions(len(mp), world, rank)]


def max_share(K: int, world: int) -> int:
    """Most positions any rank takes (the padded per-rank size of a gather)."""
    return (K + world - 1) // world


def broadcast_arrays(dist, arrays, device: str, src: int = 0) -> list[np.ndarray]:
    """Rank `src`'s numpy arrays on every rank.  Shapes and dtypes go first as one
    object broadcast; then each array as one tensor broadcast on `device` (the rank's
    GPU under NCCL, "cpu" under gloo).  `arrays` is ignored on the other ranks.
    Returns host arrays (the engine takes host buffers)."""
    import torch

    rank = dist.get_rank()
    meta = [[(a.shape, a.dtype.str) for a in arrays] if rank == src else None]
    dist.broadcast_object_list(meta, src=src)
    out = []
    for i, (shape, dt) in enumerate(meta[0]):
        dtype = np.dtype(dt)
        nbytes = int(np.prod(shape)) * dtype.itemsize
        if rank == src:
            host = np.ascontiguousarray(arrays[i]).view(np.uint8).reshape(-1)
            t = torch.from_numpy(host).to(device)
        else:
            t = torch.empty(nbytes, dtype=torch.uint8, device=device)
        if nbytes:
            dist.broadcast(t, src=src)
        out.append(t.cpu().numpy().view(dtype).reshape(shape) if rank != src else np.asarray(arrays[i]))
    return out


class ResultBuffers:
    """Device buffers (torch) a rank's share of a sweep is fetched into, padded to the
    largest share, so every rank's gather contribution has the same shape:
    edges [L][n-1][3] int32 (cs_edge words), labels [L][n] int32 (uint32 bits),
    scalars [L][3] float64 (tree edges, components, exact weight)."""

    def __init__(self, L: int, n: int, device: str, labels: bool = True):
        import torch

        self.L, self.n = L, n
        self.edges = torch.zeros((L, max(n - 1, 1), EDGE_WORDS), dtype=torch.int32, device=device)
        self.labels = torch.zeros((L, max(n, 1)), dtype=torch.int32, device=device) if labels else None
        self.scalars = torch.zeros((L, 3), dtype=torch.float64, device=device)


def gather_results(dist, K: int, bufs: ResultBuffers, dst: int = 0):
    """Gather every rank's ResultBuffers into rank `dst`'s memory (the buffers'
    device) and put them in the order of the K requested positions.  Returns
    (edges [K][n-1][3], labels [K][n] or None, scalars [K][3]) on `dst`, None on the
    other ranks."""
    import torch

    world, rank = dist.get_world_size(), dist.get_rank()
    parts = {}
    for name in ("edges", "labels", "scalars"):
        t = getattr(bufs, name)
        if t is None:
            parts[name] = None
            continue
        lst = [torch.empty_like(t) for _ in range(world)] if rank == dst else None
        dist.gather(t, gather_list=lst, dst=dst)
        parts[name] = lst
    if rank != dst:
        return None
    out = {}
    for name, lst in parts.items():
        if lst is None:
            out[name] = None
            continue
        full = torch.empty((K,) + tuple(lst[0].shape[1:]), dtype=lst[0].dtype, device=lst[0].device)
        for r in range(world):
            pos = share_positions(K, world, r)
            if pos:
                full[pos] = lst[r][: len(pos)]
        out[name] = full
    return out["edges"], out["labels"], out["scalars"]


def fetch_share(graph, positions_in_sweep, bufs: ResultBuffers) -> None:
    """Copy MSTs `positions_in_sweep` of the graph's last sweep into rows 0.. of
    `bufs` (device to device on the graph's stream, cs_sweep_fetch_device), and their
    scalars into bufs.scalars."""
    import torch

    sc = np.zeros((bufs.L, 3), np.float64)
    for i, j in enumerate(positions_in_sweep):
        lab = bufs.labels[i].data_ptr() if bufs.labels is not None else None
        r = graph.sweep_fetch_device(j, bufs.edges[i].data_ptr(), lab)
        sc[i] = (r["nedges"], r["ncomp"], r["weight"])
    bufs.scalars.copy_(torch.from_numpy(sc))


def unpack(edges_words, nedges: int):
    """The first `nedges` rows of a gathered [n-1][3] int32 tree as cs_edge records."""
    from ._abi import EDGE_DTYPE

    a = edges_words[:nedges].cpu().numpy() if hasattr(edges_words, "cpu") else edges_words[:nedges]
    return np.ascontiguousarray(a).view(EDGE_DTYPE).reshape(-1)
