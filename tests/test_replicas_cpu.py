"""Several GPUs run independent replicas; the job's time is the slowest rank's (CPU, two gloo
ranks standing in for two GPUs)."""
import datetime
import os
import socket

import pytest

from parallel_admm_b200 import replicas as R


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank's own device time (ms) and end-to-end time (s), reduced in the bench's order
        t_ms = R.max_over_ranks(100.0 + 50.0 * rank)
        e2e_s = R.max_over_ranks(2.0 - rank)
        q.put((rank, t_ms, R.job_throughput(10, world, t_ms / 1e3), e2e_s, R.rank_seed(7, rank)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_is_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [150.0, 150.0]            # max over ranks, on every rank
    assert [o[2] for o in out] == [2 * 10 / 0.150] * 2      # whole-job substeps per second
    assert [o[3] for o in out] == [2.0, 2.0]
    assert [o[4] for o in out] == [7, 8]                     # each rank its own batch


def test_single_process_needs_no_group():
    assert R.max_over_ranks(3.25) == 3.25
    assert R.job_throughput(5, 1, 0.5) == 10.0
