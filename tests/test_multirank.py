"""The multi-rank bench plumbing on CPU: two gloo ranks (world_size 2) reduce their device times to
the slowest rank, each rank projects its own seeded problem (weak scaling), and the whole-job rate
counts every rank's units over that slowest time."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from waveletpotentials_b200 import fields
    local = [10.0 + 3.0 * rank, 5.0 - rank]
    out = bench.max_over_ranks(local, world)
    seed = bench.rank_seed(7, rank)
    xv, _, _ = fields.velocity3d((8, 8, 8), seed)
    dist.barrier()
    q.put((rank, out, seed, float(np.sum(xv * xv))))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_times_and_use_distinct_problems():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, out0, s0, e0), (r1, out1, s1, e1) = res
    assert out0 == out1 == [13.0, 5.0]
    assert s0 != s1 and e0 != e1


def test_whole_job_rate_counts_all_ranks():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.throughput(1, 25, 1000.0) == 25.0
    assert bench.throughput(4, 25, 2000.0) == 50.0
    assert bench.max_over_ranks([1.5, 2.5], 1) == [1.5, 2.5]
