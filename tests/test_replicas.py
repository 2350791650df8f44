"""The multi-process (replica) path of the benchmark on the host: two gloo ranks on
CPU stand in for two GPUs.  Each rank times its own replica; the job's time is the
maximum over ranks and its throughput counts every rank's MSTs."""
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, totals, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from coresg_b200 import replicas

    r = replicas.from_env("gloo", timeout_s=60)
    try:
        r.barrier()
        slowest = r.max_over_ranks(totals[rank])
        value = replicas.replica_throughput(r.world, 32, 10, slowest)
        r.barrier()
        out.put((r.rank, r.world, slowest, value))
    finally:
        r.close()


def test_two_gloo_ranks_take_the_slowest_time():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    totals = [240.5, 251.25]  # ms of device time per rank over the timed steps
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, totals, out)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(out.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    assert [g[0] for g in got] == [0, 1]
    for rank, world, slowest, value in got:
        assert world == 2
        assert slowest == 251.25
        assert value == pytest.approx(2 * 32 * 10 / 0.25125)


def test_single_rank_needs_no_group(monkeypatch):
    from coresg_b200 import replicas

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    r = replicas.from_env("nccl")
    assert (r.rank, r.world, r.group) == (0, 1, None)
    r.barrier()
    assert r.max_over_ranks(12.5) == 12.5
    assert replicas.replica_throughput(1, 32, 10, 250.0) == pytest.approx(1280.0)
    with pytest.raises(ValueError):
        replicas.replica_throughput(1, 32, 10, 0.0)
