"""Multi-rank logic of bench.py on CPU: two `gloo` ranks (127.0.0.1).

Every rank diffuses its own volume; the job's time is the slowest rank's and
the job's rate counts all ranks' voxels.  The reference arm runs on rank 0
alone: the other ranks return without work or output."""
import argparse
import contextlib
import datetime
import io
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
    slowest = bench.max_over_ranks(ms, world, "cpu")
    rate = bench.whole_job_rate(world, 1000, 2, 3, slowest / 1e3)
    dist.barrier()
    dist.destroy_process_group()
    queue.put((rank, slowest, rate))


def test_max_over_ranks_and_whole_job_rate_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r for r, _, _ in results) == [0, 1]
    for _, slowest, rate in results:
        assert slowest == 15.0
        assert rate == pytest.approx(2 * 1000 * 2 * 3 / 0.015 / 1e9)


def test_single_rank_identity():
    import bench
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5


def test_reference_arm_other_ranks_do_no_work():
    import bench
    args = argparse.Namespace(gpus=2, steps=1, warmup=0, workload="bone1024_s8_r100")
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        assert bench.run_reference_arm(args, 1) is None
    assert out.getvalue() == ""
