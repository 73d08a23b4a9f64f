"""Branch-and-bound over device LP relaxations: ``BranchAndBound.solveWith``
(modules/prima-core/src/main/scala/org/noaidi/prima/BranchAndBound.scala:139-377)
with every node's relaxation solved on the GPU.

The matrix of a MILP never changes from node to node -- a node is its
parent's LP with one variable bound moved -- so the problem is uploaded and
equilibrated once (``DeviceProblem``) and each node only replaces the bounds
(``prima_problem_set_bounds``) and runs a warm-started solve.  The search
itself is the reference's, step for step: depth first, the most fractional
integer column, children pushed ceiling first, pruning only against a bound
lowered by a multiple of the node's own duality gap, and a status
downgraded whenever a relaxation was not conclusive.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Callable, Optional, Sequence

import numpy as np

from .model import LpProblem
from .types import LpSolution, PdhgParams, SolveStatus, WarmStart


class MilpStatus(IntEnum):
    """``MilpStatus`` (BranchAndBound.scala:7-30)."""
    OPTIMAL = 0
    FEASIBLE = 1
    INFEASIBLE = 2
    UNBOUNDED = 3
    NO_SOLUTION_FOUND = 4

    @property
    def is_conclusive(self) -> bool:
        return self in (MilpStatus.OPTIMAL, MilpStatus.INFEASIBLE, MilpStatus.UNBOUNDED)


@dataclass
class MilpSolution:
    """``MilpSolution`` (BranchAndBound.scala:33-60)."""
    status: MilpStatus
    primal: np.ndarray
    objective_value: float
    best_bound: float
    nodes_explored: int
    unproven_nodes: int
    solve_time_millis: int

    @property
    def gap(self) -> float:
        return abs(self.objective_value - self.best_bound)


@dataclass(frozen=True)
class BnbParams:
    """``BnbParams`` (BranchAndBound.scala:63-112)."""
    lp: PdhgParams = field(default_factory=PdhgParams)
    integrality_tolerance: float = 1e-6
    gap_abs: float = 1e-6
    gap_rel: float = 1e-6
    pruning_safety_factor: float = 10.0
    max_nodes: int = 100_000
    time_limit_millis: Optional[int] = None
    warm_start: bool = True

    def copy(self, **kw) -> "BnbParams":
        d = dict(self.__dict__)
        d.update(kw)
        return BnbParams(**d)


# A node solver: (lower, upper, lp params, warm start or None) -> LpSolution.
NodeSolver = Callable[[np.ndarray, np.ndarray, PdhgParams, Optional[WarmStart]], LpSolution]


def device_node_solver(problem: LpProblem, params: BnbParams, precision: int = 64, device: int = 0, ctx=None):
    """Node relaxations on the GPU, sharing one resident copy of the matrix.
    ``precision=64`` has ScalaKernels semantics, the reference's default
    backend for ``BranchAndBound.solve`` (BranchAndBound.scala:160-168)."""
    from . import cuda
    resident = cuda.DeviceProblem(problem, params.lp, ctx=ctx, device=device, precision=precision)

    def solve(lower, upper, lp: PdhgParams, warm: Optional[WarmStart]) -> LpSolution:
        resident.set_bounds(lower, upper)
        return resident.solve(lp, warm_start=warm)

    solve.resident = resident
    return solve


def solve(problem: LpProblem, integers: set, params: BnbParams = BnbParams(), precision: int = 64,
          device: int = 0, ctx=None) -> MilpSolution:
    """``BranchAndBound.solve`` with the relaxations on the GPU."""
    node = device_node_solver(problem, params, precision=precision, device=device, ctx=ctx)
    try:
        return solve_with(problem, integers, params, node)
    finally:
        node.resident.free()


def solve_with(problem: LpProblem, integers: set, params: BnbParams, node_solver: NodeSolver) -> MilpSolution:
    """``BranchAndBound.solveWith`` (BranchAndBound.scala:170-377)."""
    n = problem.num_variables
    for j in integers:
        if not (0 <= j < n):
            raise ValueError(f"requirement failed: integer column {j} is out of range [0, {n})")
    started = time.monotonic()

    def elapsed_ms() -> int:
        return int((time.monotonic() - started) * 1000)

    if not integers:  # the relaxation is the answer (:190-221)
        root = node_solver(problem.variable_lower, problem.variable_upper, params.lp, None)
        status = {SolveStatus.OPTIMAL: MilpStatus.OPTIMAL, SolveStatus.PRIMAL_INFEASIBLE: MilpStatus.INFEASIBLE,
                  SolveStatus.DUAL_INFEASIBLE: MilpStatus.UNBOUNDED}.get(root.status, MilpStatus.NO_SOLUTION_FOUND)
        solved = status == MilpStatus.OPTIMAL
        return MilpSolution(status, root.primal if solved else np.empty(0),
                            root.objective_value if solved else math.inf,
                            root.objective_value if solved else -math.inf, 1,
                            0 if root.status.is_conclusive else 1, elapsed_ms())

    ordered = sorted(integers)
    # a node: (lower, upper, safe bound of its parent, warm start)
    stack: list = [(np.array(problem.variable_lower, dtype=np.float64),
                    np.array(problem.variable_upper, dtype=np.float64), -math.inf, None)]
    incumbent = np.empty(0)
    incumbent_value = math.inf
    nodes = unproven = 0
    root_unbounded = False

    def open_bound() -> float:
        if not stack:
            return incumbent_value
        return min(incumbent_value, min(s[2] for s in stack))

    def out_of_time() -> bool:
        return params.time_limit_millis is not None and elapsed_ms() > params.time_limit_millis

    while stack and nodes < params.max_nodes and not out_of_time():
        lower, upper, parent_safe, warm = stack.pop()
        if skips_before_solving(parent_safe, incumbent_value, incumbent.size > 0):
            continue
        relaxation = node_solver(lower, upper, params.lp, warm if params.warm_start else None)
        nodes += 1
        status = relaxation.status
        if status == SolveStatus.PRIMAL_INFEASIBLE:
            continue  # no integer point here either
        if status == SolveStatus.DUAL_INFEASIBLE:
            if nodes == 1:
                root_unbounded = True
            else:
                unproven += 1  # a spurious deep unboundedness is counted, not trusted (:273-283)
            continue
        conclusive = status.is_conclusive
        if not conclusive:
            unproven += 1
        bound = relaxation.objective_value
        slack = params.pruning_safety_factor * max(abs(relaxation.kkt.absolute_gap), params.lp.eps_abs)
        safe = safe_bound_of(conclusive, bound, slack)
        prunable = conclusive and incumbent.size > 0 and safe >= incumbent_value
        if prunable:
            continue
        j = most_fractional(relaxation.primal, ordered, params.integrality_tolerance)
        if j is None:
            if conclusive:  # integral with a trustworthy bound: a candidate (:318-336)
                snapped = snap(relaxation.primal, ordered)
                value = problem.primal_objective(snapped)
                if value < incumbent_value:
                    incumbent_value = value
                    incumbent = snapped
            continue
        value = relaxation.primal[j]
        floor, ceil = math.floor(value), math.ceil(value)
        child_warm = None
        if params.warm_start:
            try:
                child_warm = WarmStart.from_solution(relaxation)
            except ValueError:
                child_warm = None
        # ceiling first, so the floor branch is explored first (:357-363)
        if ceil <= upper[j]:
            up = lower.copy()
            up[j] = max(up[j], ceil)
            stack.append((up, upper, safe, child_warm))
        if floor >= lower[j]:
            down = upper.copy()
            down[j] = min(down[j], floor)
            stack.append((lower, down, safe, child_warm))

    bound = incumbent_value if not stack else open_bound()
    if root_unbounded:
        status = MilpStatus.UNBOUNDED
    elif incumbent.size == 0 and not stack and unproven == 0:
        status = MilpStatus.INFEASIBLE
    elif incumbent.size == 0:
        status = MilpStatus.NO_SOLUTION_FOUND
    elif unproven > 0:
        status = MilpStatus.FEASIBLE
    elif not stack:
        status = MilpStatus.OPTIMAL
    elif closed(incumbent_value, bound, params):
        status = MilpStatus.OPTIMAL
    else:
        status = MilpStatus.FEASIBLE
    return MilpSolution(status, incumbent, incumbent_value,
                        bound if incumbent.size == 0 else min(bound, incumbent_value), nodes, unproven, elapsed_ms())


def skips_before_solving(safe_bound: float, incumbent: float, have_incumbent: bool) -> bool:
    """``skipsBeforeSolving`` (:389-394): a NaN bound never skips."""
    return have_incumbent and safe_bound >= incumbent


def safe_bound_of(conclusive: bool, bound: float, slack: float) -> float:
    """``safeBoundOf`` (:404-408)."""
    if not conclusive:
        return -math.inf
    candidate = bound - slack
    return candidate if math.isfinite(candidate) else -math.inf


def closed(incumbent: float, bound: float, params: BnbParams) -> bool:
    """``closed`` (:410-413)."""
    absolute = abs(incumbent - bound)
    return absolute <= params.gap_abs or absolute <= params.gap_rel * max(1.0, abs(incumbent))


def most_fractional(x: Sequence[float], integers: Sequence[int], tolerance: float) -> Optional[int]:
    """``mostFractional`` (:421-435): the first column with the largest gap
    to its nearest whole number (``math.round``: half rounds up)."""
    best, worst = -1, tolerance
    for j in integers:
        gap = abs(x[j] - math.floor(x[j] + 0.5))
        if gap > worst:
            worst, best = gap, j
    return None if best < 0 else best


def snap(x: np.ndarray, integers: Sequence[int]) -> np.ndarray:
    """``snap`` (:444-447)."""
    out = np.array(x, dtype=np.float64)
    for j in integers:
        out[j] = math.floor(out[j] + 0.5)
    return out
