"""Sharding an ensemble of independent boxes over GPUs (one process per GPU).

The boxes never exchange data, so a multi-GPU ensemble is a partition of the
boxes: every rank computes the same assignment from the box sizes alone (no
communication), advances its share with a :class:`~nmhd_b200.batch.BatchSolver`,
and only per-box results are gathered at the end.  The assignment balances the
per-step work (cells, margins included) by longest-processing-time-first:
boxes in decreasing cost, each to the least-loaded rank (lowest rank on ties),
which keeps the busiest rank within 4/3 of the best possible makespan.
"""
from __future__ import annotations


def box_cost(cfg) -> int:
    """Work of one step of a box: its cells, margins included (every cell is
    advanced)."""
    return cfg.size_x * cfg.size_y * cfg.size_z


def assign(costs, world: int):
    """Box indices of each of ``world`` ranks (each list in increasing box
    order); deterministic, so every rank computes the same partition."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    shares = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shares[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shares]


def my_boxes(configs, rank: int, world: int):
    """The indices of the boxes rank ``rank`` advances."""
    return assign([box_cost(c) for c in configs], world)[rank]


def gather_by_box(dist, n_boxes: int, mine, values):
    """Per-box values from every rank, in box order, on every rank.
    ``mine`` are this rank's box indices, ``values`` its values for them
    (any picklable objects).  Without a process group, returns ``values``
    placed by index."""
    pairs = list(zip(mine, values))
    if dist is None or not dist.is_initialized():
        parts = [pairs]
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, pairs)
    out = [None] * n_boxes
    for part in parts:
        for i, v in part:
            out[i] = v
    return out
