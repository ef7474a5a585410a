"""The replica timing of bench.py on two ranks over gloo (CPU): every rank
gets the slowest rank's time, and the whole-job figure counts every
replica's bytes over that time.  The decode path does not shard across
GPUs (columns and vectors are independent), so N GPUs run N replicas with
no collective on the data path; this covers the host-side logic."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    import datetime
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    bench.barrier(world)
    ms = 10.0 + 5.0 * rank
    q.put((rank, bench.max_over_ranks(ms, world)))
    bench.barrier(world)
    dist.destroy_process_group()


def test_max_over_ranks_and_job_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 15.0, 1: 15.0}
    import sys
    sys.path.insert(0, ROOT)
    import bench
    # 2 replicas x 3 steps x 1.5 GB in 15 ms (the slowest) = 600 GB/s
    assert bench.job_gbs(1_500_000_000, 3, 2, 15.0) == pytest.approx(600.0)
