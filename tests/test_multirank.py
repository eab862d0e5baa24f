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


# ---------------------------------------------------------------- batch sharding across ranks
SPECS = [(256, 256, 256), (64, 64, 64), (128, 64, 64), (32, 32, 32), (128, 128, 128), (512, 256), (64, 64),
         (32, 64, 128), (16, 16, 16), (1024, 1024), (128, 128, 64)]
STEPS = [4, 7, 3, 9, 5, 2, 6, 4, 8, 3, 5]


def _shard_worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from waveletpotentials_b200 import sharding
    costs = [sharding.grid_cost(d, s) for d, s in zip(SPECS, STEPS)]
    owner = sharding.partition(costs, world)
    # each rank reports only its own grids (stand-ins for its BatchProjector's per-grid scalars)
    local = {i: {"max_abs_div": 1e-3 * i, "rank": rank} for i in range(len(SPECS)) if owner[i] == rank}
    merged = sharding.gather_results(local, len(SPECS), world)
    q.put((rank, owner, merged))
    dist.destroy_process_group()


def test_cost_partitioned_batch_on_two_gloo_ranks():
    """Two gloo ranks partition the same batch by cost with no exchange (identical owners on both
    ranks), each grid is projected by exactly one rank, the heavier rank carries at most the mean
    load plus one grid, and the final scalar gather gives both ranks the whole batch in grid order."""
    sys.path.insert(0, ROOT)
    from waveletpotentials_b200 import sharding
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in range(world)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, own0, m0), (_, own1, m1) = res
    assert own0 == own1
    assert m0 == m1
    assert [m["rank"] for m in m0] == own0
    assert [m["max_abs_div"] for m in m0] == [1e-3 * i for i in range(len(SPECS))]
    costs = [sharding.grid_cost(d, s) for d, s in zip(SPECS, STEPS)]
    load = sharding.rank_loads(costs, own0, world)
    assert sum(load) == sum(costs)
    assert max(load) <= sum(costs) / world + max(costs)
    assert set(own0) == {0, 1}


def test_partition_properties():
    """Longest-processing-time rule on random costs: deterministic, every grid owned once, the
    greedy bound max load <= mean + max cost, and no rank idle while another holds two grids."""
    sys.path.insert(0, ROOT)
    from waveletpotentials_b200 import sharding
    rng = np.random.default_rng(5)
    for trial in range(200):
        world = int(rng.integers(1, 9))
        costs = list(rng.integers(1, 10 ** 6, size=int(rng.integers(0, 40))).astype(float))
        owner = sharding.partition(costs, world)
        assert owner == sharding.partition(costs, world)
        assert len(owner) == len(costs) and all(0 <= r < world for r in owner)
        load = sharding.rank_loads(costs, owner, world)
        if costs:
            assert max(load) <= sum(costs) / world + max(costs) + 1e-6
        if len(costs) >= world:
            assert min(load) > 0
    assert sharding.expected_steps(1e-10) == 10 and sharding.expected_steps(1e-6) == 6
    assert sharding.partition([], 3) == []
    import pytest
    with pytest.raises(ValueError):
        sharding.partition([1.0], 0)
    with pytest.raises(RuntimeError):
        sharding.gather_results({0: 1}, 2, 1)
