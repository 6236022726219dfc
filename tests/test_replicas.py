"""The multi-process path of bench.py on CPU: two ranks over gloo (127.0.0.1).  The path has no
exchange step (every rank solves its own replica), so the only cross-rank work is the timing:
the slowest rank's time, and the aggregate seconds per solve derived from it; and the reference arm
runs on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 25.0 * rank  # this rank's time per solve
        slowest = bench.max_over_ranks(ms, dist, "cpu")
        e2e = bench.max_over_ranks(0.5 + rank, dist, "cpu")
        out.put((rank, slowest, e2e, bench.replica_seconds(slowest, world)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_timing_is_the_slowest_rank_over_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, e2e, value in res:
        assert slowest == 125.0 and e2e == 1.5
        assert value == pytest.approx(125.0 / 1e3 / world)


def test_one_process_reduces_to_itself():
    assert bench.max_over_ranks(3.25) == 3.25
    assert bench.replica_seconds(420.0, 1) == pytest.approx(0.42)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    class Args:
        workload = "star_f32"
        warmup = 3
        steps = 3
        gpus = 2

    assert bench.run_reference(Args(), rank=1) is None  # returns at once: no mesh, no timing
    assert capsys.readouterr().out == ""
