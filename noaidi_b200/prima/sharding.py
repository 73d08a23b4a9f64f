"""Independent LPs across GPUs: one process per GPU, each solving its own
shard of the instances, with no collective on the data path.

This is the multi-GPU form of ``PrimaZio.solveAll``
(modules/prima-zio/.../PrimaZio.scala:61-66): the instances of a sweep are
independent, so they partition across ranks.  A single LP does not split
(each iteration exchanges the whole of x-bar and y), so one LP runs on one
GPU.

``shard`` is a longest-processing-time assignment: instances in order of
decreasing size, each to the rank with the least work so far (ties to the
lower rank), so every rank gets a similar total.  ``solve_sharded`` runs a
rank's shard and, given a process group, gathers every rank's results so
that each rank returns all of them in the caller's order.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np


def instance_size(problem) -> int:
    """Work proxy of one instance: the nonzeros plus both dimensions."""
    return int(problem.constraint_matrix.nnz) + int(problem.num_variables) + int(problem.num_constraints)


def shard(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Instance indices per rank (each list ascending)."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = np.zeros(world, dtype=np.int64)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))  # first minimum: ties go to the lower rank
        out[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(s) for s in out]


def solve_sharded(problems: Sequence, solve: Callable[[list], list], rank: int = 0, world: int = 1,
                  group=None) -> tuple[list, list]:
    """Solve this rank's shard with ``solve(list_of_problems) -> list_of_results``.

    Returns (all results in the order of ``problems``, this rank's indices).
    With a process group (world > 1), every rank's results are gathered with
    ``all_gather_object`` -- the only exchange, after all solving is done.
    """
    parts = shard([instance_size(p) for p in problems], world)
    mine = parts[rank]
    results = solve([problems[i] for i in mine])
    if len(results) != len(mine):
        raise ValueError("solve returned a different number of results")
    if world == 1:
        return list(results), mine
    import torch.distributed as dist
    gathered: list[Optional[list]] = [None] * world
    dist.all_gather_object(gathered, list(zip(mine, results)), group=group)
    out: list = [None] * len(problems)
    for part in gathered:
        for i, res in part:
            out[i] = res
    return out, mine
