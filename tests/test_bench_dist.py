"""The multi-process side of bench.py on CPU: two gloo ranks, the max over
ranks reaches every rank, the whole-job rate counts every replica, and the
reference arm does its work on rank 0 only."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = bench.max_over_ranks(10.0 + rank, dist, "cpu")
    rate = bench.whole_job_rate(world, 1000, 50, ms)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ms, rate))


def test_two_gloo_ranks_max_and_aggregate():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]                 # the slowest rank's time, on both ranks
    assert res[0][2] == pytest.approx(2 * 1000 * 50 / 0.011 / 1e6)


def test_single_process_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_rate(1, 4, 10, 1000.0) == pytest.approx(4e-5)


def test_reference_arm_other_ranks_exit_without_work(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup, gpus = 1, 0, 2
    bench.run_reference(A(), rank=1, world=2)
    assert capsys.readouterr().out == ""
