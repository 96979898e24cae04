"""The multi-GPU plumbing of bench.py on CPU: two ranks with the gloo backend over 127.0.0.1.
Each rank renders its own replica (no data-path collective); the job's time is the maximum of
the ranks' times and the throughput counts every rank's units."""
import datetime
import os
import socket
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    # rank r "took" 10 (r + 1) ms for its replica of 1000 units
    t = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
    dist.barrier()
    q.put((rank, t, bench.weak_scaling_rate(1000, world, t / 1e3)))
    dist.destroy_process_group()


def test_job_time_is_max_over_two_gloo_ranks():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate in out:
        assert t == 20.0  # the slower rank's time, on both ranks
        assert rate == pytest.approx(2 * 1000 / 0.020 / 1e6)


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.weak_scaling_rate(4_194_304, 1, 2.0) == pytest.approx(2.097152)
