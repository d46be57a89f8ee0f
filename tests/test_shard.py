"""Multi-GPU ensemble sharding, host logic (CPU, gloo process groups).

Each rank computes the box assignment on its own; the test checks on 2 and 3
ranks that the shares agree across ranks, partition the ensemble, balance the
work within the LPT bound, and that per-box results gather back in box order.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from nmhd_b200.problems import mri_ensemble
from nmhd_b200.shard import assign, box_cost, gather_by_box, my_boxes


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ensemble_configs():
    boxes, _ = mri_ensemble(n_boxes=64, seed=0)
    return [c for c, _ in boxes]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfgs = _ensemble_configs()
        mine = my_boxes(cfgs, rank, world)
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        # a per-box "result" computed where the box lives
        res = gather_by_box(dist, len(cfgs), mine, [("box", i, rank) for i in mine])
        if rank == 0:
            out.put((shares, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_shards_agree_across_ranks_partition_and_balance(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    shares, res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfgs = _ensemble_configs()
    costs = [box_cost(c) for c in cfgs]
    assert shares == assign(costs, world)  # every rank computed the same shares
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(cfgs)))  # a partition of the ensemble
    loads = [sum(costs[i] for i in s) for s in shares]
    assert max(loads) <= sum(costs) / world + max(costs)  # LPT bound
    assert max(loads) / min(loads) < 1.1  # 64 boxes balance well
    for i, (tag, box, rank) in enumerate(res):
        assert box == i and i in shares[rank]


def test_single_rank_takes_everything():
    cfgs = _ensemble_configs()
    assert my_boxes(cfgs, 0, 1) == list(range(len(cfgs)))
    assert gather_by_box(None, 3, [2, 0], ["c", "a"]) == ["a", None, "c"]
