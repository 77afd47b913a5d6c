"""The benchmark's multi-rank logic on CPU: two gloo ranks (127.0.0.1) take
the slowest rank's time, count the whole job's work, reconstruct different
objects, and only rank 0 runs the reference arm."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench
from fdk_cuda_impl_b200.workloads import WORKLOADS


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world, timeout=datetime.timedelta(seconds=60))
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower one
        slowest = bench.max_over_ranks(ms, world, "cpu")
        dist.barrier()
        q.put((rank, slowest, bench.job_gups(world, WORKLOADS["c2"].updates, slowest),
               bench.object_seed(rank)))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None, None))


def test_two_gloo_ranks_reduce_to_the_slowest():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, slowest, gups, seed = q.get(timeout=120)
        out[r] = (slowest, gups, seed)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert out[r][0] == 15.0, out
        assert out[r][1] == pytest.approx(2 * WORKLOADS["c2"].updates / 15e-3 / 1e9)
    assert out[0][2] != out[1][2]


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr("sys.argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(bench.parse()) is None
    assert capsys.readouterr().out == ""
