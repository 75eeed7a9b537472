"""CPU tests of the multi-GPU host logic with two `gloo` ranks: the instance
partition every rank computes alone is identical across ranks, disjoint
and complete, balanced, and the timing reduction is a max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "the-powder-toy-rust-wgpu_b200"))
    import sharding
    import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    shapes = W.config_shapes(5)
    mine = sharding.shard_of(shapes, rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    # the same time-like reduction bench.py does: max over ranks
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    if rank == 0:
        q.put((gathered, float(t.item())))
    dist.destroy_process_group()


def test_two_rank_partition_and_max_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = gathered
    assert set(a).isdisjoint(b) and sorted(a + b) == list(range(128))
    assert tmax == 2.0


def test_partition_balance_and_determinism():
    import sharding
    import workloads as W

    for cid in (4, 5):
        shapes = W.config_shapes(cid)
        costs = [sharding.instance_cost(x, y) for x, y in shapes]
        for world in (1, 2, 4, 8):
            shards = sharding.partition(costs, world)
            assert sorted(i for s in shards for i in s) == list(range(len(shapes)))
            assert shards == sharding.partition(costs, world)
            assert sharding.imbalance(costs, shards) < 1.25
    with pytest.raises(ValueError):
        sharding.partition([1.0], 0)


def test_instance_cost_matches_its_flop_formula():
    """The split-BF16 cost is 3 * (12 X^2 Y + 48 X Y^2) flops (half of the
    full-spectrum F = 24 X^2 Y + 96 X Y^2, times the three split products)
    at 2000 flops per air cell-tick, plus the cells."""
    import sharding

    for x, y in ((400, 225), (32, 36), (512, 41), (153, 96)):
        flops = 3.0 * (12.0 * x * x * y + 48.0 * x * y * y)
        assert sharding.instance_cost(x, y) == pytest.approx(x * y + flops / 2000.0, rel=1e-12)
        assert flops == pytest.approx(1.5 * (24.0 * x * x * y + 96.0 * x * y * y), rel=1e-12)
        assert sharding.instance_cost(x, y, newton_grav=False) == x * y


def test_partition_imbalance_every_world_size():
    """C5 and C4 shapes split over 2..8 ranks stay within 6% of perfect balance."""
    import sharding
    import workloads as W

    for cid in (4, 5):
        costs = [sharding.instance_cost(x, y) for x, y in W.config_shapes(cid)]
        for world in range(2, 9):
            assert sharding.imbalance(costs, sharding.partition(costs, world)) < 1.06
