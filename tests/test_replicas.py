"""Multi-GPU runs are independent replicas (one full workload per GPU, no data-path collective):
the only cross-rank steps are the barrier and the max over ranks of the timings, tested here
with world size 2 on the gloo backend (CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    d = bench.Dist(world)
    d.barrier()
    v = d.max(10.0 + rank)  # ranks report different step times; every rank gets the max
    d.barrier()
    q.put((rank, v, d.world))
    d.close()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0, 2), (1, 11.0, 2)]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "1")

    class A:
        pass
    d = bench.Dist(1)
    d.rank = 1
    assert bench.run_reference(A(), d) is None
