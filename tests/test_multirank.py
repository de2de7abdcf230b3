"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2).

The step is one coupled grid, so N GPUs run N independent replicas: the
benchmark's only cross-rank operations are the barrier around the timed
region and the max over ranks of the timings.  These tests run that path
with two gloo ranks on 127.0.0.1, and check that the reference arm does its
work on rank 0 only.
"""
import datetime
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        dist.barrier()
        ms = 10.0 + 2.5 * rank   # the second rank is slower
        m = bench.max_over_ranks(ms, world, "cpu")
        q.put((rank, m, bench.job_rate(world, 1000, 5, m)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, rate in res:
        assert m == 12.5                       # every rank sees the slowest rank's time
        assert rate == pytest.approx(2 * 1000 * 5 / 12.5e-3 / 1e6)


def test_single_rank_is_identity():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(3.0, 1, "cpu") == 3.0
    assert bench.job_rate(1, 256 ** 3, 10, 50.0) == pytest.approx(256 ** 3 * 10 / 0.05 / 1e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun only rank 0 times the CPU reference; the others exit 0
    without output."""
    sys.path.insert(0, REPO)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--n", "16", "--steps", "1", "--warmup", "0"])
    assert bench.main() == 0
    assert capsys.readouterr().out == ""
