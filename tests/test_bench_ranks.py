"""CPU: the multi-rank arithmetic of bench.py with two gloo ranks.

`bench.py --gpus N` runs one replica of the workload per rank (the step does
not shard: every particle's walk reads the whole tree), times each rank's
steps on its own device, and reports the slowest rank's time and the whole
job's rate.  Here two CPU ranks over gloo stand in for the GPUs: every rank
must see the largest of the ranks' times, and the rate must count every
rank's particles over that time.  The reference arm runs on rank 0 alone.
"""
import importlib.util
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = _bench()
        mine = 10.0 + 5.0 * rank          # this rank's timed milliseconds
        total = b.max_over_ranks(dist, mine, "cpu")
        rate = b.whole_job_rate(world, 1000, 4, total)
        # the reference arm does no work off rank 0
        ref = b.run_reference(None, world, rank) if rank != 0 else "rank0"
        q.put((rank, total, rate, ref))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = 10.0 + 5.0 * (world - 1)
    for rank, total, rate, ref in got:
        assert total == slowest
        assert rate == pytest.approx(world * 1000 * 4 / (slowest * 1e-3))
        if rank != 0:
            assert ref is None


def test_single_rank_needs_no_process_group():
    b = _bench()
    assert b.max_over_ranks(None, 7.5, "cpu") == 7.5
    assert b.whole_job_rate(1, 1 << 20, 30, 24.0) == pytest.approx((1 << 20) * 30 / 0.024)
