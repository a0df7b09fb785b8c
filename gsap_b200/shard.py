"""Job sharding for batched partitioning on several GPUs, one process per GPU.

Independent graphs need no data-path collective: one job list is split
across the ranks, every rank partitions its share on its own GPU
(sbp_partition_batch), and the labels and reports travel to rank 0 once, at
the end, through torch.distributed (NCCL between GPUs, gloo on hosts without
one).  GSAP partitions one graph per process and has no counterpart.

    plan = shard_jobs(costs, world)             # job indices per rank
    mine = plan[rank]
    labels, reports = my_partition(mine)        # this rank's share
    all_labels, all_reports = gather_results(mine, labels, reports, world, rank)
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple


def shard_jobs(costs: Sequence[float], world: int) -> List[List[int]]:
    """Splits jobs 0..n-1 over `world` ranks so that the ranks' summed costs
    (e.g. edge counts) are close: longest job first to the least loaded rank
    (ties to the lower rank).  Each rank's list is in ascending job order, so
    its batch keeps the job list's order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    plan: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        plan[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in plan]


def gather_results(mine: Sequence[int], labels: Sequence, reports: Sequence, world: int,
                   rank: int, group=None) -> Tuple[Optional[list], Optional[list]]:
    """Rank 0 receives every rank's (job index, labels, report) and returns
    labels and reports in job order; the other ranks return (None, None).
    Every rank must call it (it is one collective)."""
    if len(mine) != len(labels) or len(mine) != len(reports):
        raise ValueError("one label array and one report per job")
    local = list(zip([int(i) for i in mine], list(labels), list(reports)))
    if world == 1:
        parts = [local]
    else:
        import torch.distributed as dist
        parts = [None] * world if rank == 0 else None
        dist.gather_object(local, parts, dst=0, group=group)
    if rank != 0:
        return None, None
    rows = sorted((row for part in parts for row in part), key=lambda x: x[0])
    n = len(rows)
    if [r[0] for r in rows] != list(range(n)):
        raise RuntimeError("gathered job indices are not 0..n-1 exactly once")
    return [r[1] for r in rows], [r[2] for r in rows]
