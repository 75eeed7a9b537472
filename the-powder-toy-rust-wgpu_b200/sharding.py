"""Sharding of independent sandbox instances over ranks (one process per GPU).

Instances of a batch never exchange data during ticks, so a multi-GPU run
partitions them with no collective in the data path; ranks meet only at the
timing barrier and the max-over-ranks reduction of the elapsed time.

The reference is single-GPU (one wgpu device, crates/tpt-app/src/main.rs:
398-430); this module is the B200 build's own host logic for the batched
workloads.
"""
from __future__ import annotations


def instance_cost(xcells: int, ycells: int, newton_grav: bool = True) -> float:
    """Relative cost of one tick of one instance: the air step is linear in
    the cells; the split-BF16 gravity solve costs the executed flops of the
    DFT-as-GEMM on the Hermitian half-spectrum, half of the full-spectrum
    F = 24*X^2*Y + 96*X*Y^2 per solve, times the 3 split products:
    3 * (12*X^2*Y + 48*X*Y^2), where the x-stage terms are
    6*X*Y*(2X) = 12*X^2*Y and the y-stage terms 12*Y*(2X)*(2Y) = 48*X*Y^2.
    Flops are expressed in cell units at the measured ratio of air to
    gravity time per cell (about one air cell-tick per 2000 gravity flops)."""
    air = float(xcells * ycells)
    if not newton_grav:
        return air
    x_stage = 6.0 * xcells * ycells * (2 * xcells)            # = 12 X^2 Y
    y_stage = 12.0 * ycells * (2 * xcells) * (2 * ycells)     # = 48 X Y^2
    grav_flops = 3.0 * (x_stage + y_stage)
    return air + grav_flops / 2000.0


def partition(costs: list[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first greedy partition of instance indices
    into `world` shards of near-equal total cost. Deterministic: every rank
    computes the same assignment with no communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        shards[r].append(i)
        loads[r] += costs[i]
    for s in shards:
        s.sort()
    return shards


def shard_of(shapes: list[tuple[int, int]], rank: int, world: int, newton_grav: bool = True) -> list[int]:
    """Instance indices rank `rank` owns."""
    return partition([instance_cost(x, y, newton_grav) for x, y in shapes], world)[rank]


def imbalance(costs: list[float], shards: list[list[int]]) -> float:
    """max shard cost / mean shard cost (1.0 = perfect)."""
    loads = [sum(costs[i] for i in s) for s in shards]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0
