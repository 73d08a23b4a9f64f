"""MILP fixtures of BranchAndBoundSuite (modules/prima-core/src/test/scala/
org/noaidi/prima/BranchAndBoundSuite.scala), each with a fractional
relaxation and an optimum worked out by hand, and an oracle node solver:
the reference's FP64 PDHG restated in C, used here only as the oracle."""
import numpy as np

from noaidi_b200.prima import LpProblem, PdhgParams
from noaidi_b200.prima.bnb import BnbParams

PARAMS = BnbParams(lp=PdhgParams(eps_abs=1e-9, eps_rel=1e-9))


def knapsackish():
    """maximise 5a + 4b s.t. 6a + 4b <= 24, a + 2b <= 6, 0 <= a, b <= 10 (:17-25):
    relaxation a = 3, b = 1.5 at -21; integer optimum a = 4, b = 0 at -20."""
    b = LpProblem.builder(2)
    b.objective_coefficient(0, -5.0).objective_coefficient(1, -4.0)
    b.bounds(0, 0.0, 10.0).bounds(1, 0.0, 10.0)
    b.less_than([(0, 6.0), (1, 4.0)], 24.0)
    b.less_than([(0, 1.0), (1, 2.0)], 6.0)
    return b.build()[0]


def no_integer_point():
    """2x = 1, 0 <= x <= 1, x integer (:73-84): infeasible only by branching."""
    b = LpProblem.builder(1)
    b.objective_coefficient(0, 1.0).bounds(0, 0.0, 1.0)
    b.equality_constraint([(0, 2.0)], 1.0)
    return b.build()[0]


def binaries():
    """minimise -(3x + 2y + 4z) s.t. x + y + z <= 2, binary (:86-99): -7 at (1, 0, 1)."""
    b = LpProblem.builder(3)
    for i, c in enumerate((-3.0, -2.0, -4.0)):
        b.objective_coefficient(i, c).bounds(i, 0.0, 1.0)
    b.less_than([(0, 1.0), (1, 1.0), (2, 1.0)], 2.0)
    return b.build()[0]


def hard_knapsack():
    """The 16-item 0/1 knapsack of the pruning-margin test (:173-181)."""
    values = [41.0, 50, 49, 59, 45, 47, 12, 33, 21, 44, 51, 19, 28, 37, 40, 25]
    weights = [31.0, 27, 12, 34, 22, 19, 8, 16, 11, 24, 29, 9, 14, 20, 23, 13]
    b = LpProblem.builder(len(values))
    for i, v in enumerate(values):
        b.objective_coefficient(i, -v).bounds(i, 0.0, 1.0)
    b.less_than([(i, w) for i, w in enumerate(weights)], 120.0)
    return b.build()[0], values, weights


def oracle_node_solver(problem):
    from oracle import oracle as O

    def solve(lower, upper, lp: PdhgParams, warm):
        node = LpProblem(problem.objective, problem.constraint_matrix, problem.rhs, problem.num_equalities,
                         np.asarray(lower, dtype=np.float64), np.asarray(upper, dtype=np.float64),
                         problem.objective_offset)
        return O.solve(node, lp, warm_start=warm)
    return solve


def knapsack_optimum(values, weights, capacity):
    """Exact 0/1 knapsack by dynamic programming over integer weights."""
    best = [0.0] * (int(capacity) + 1)
    for v, w in zip(values, weights):
        for c in range(int(capacity), int(w) - 1, -1):
            best[c] = max(best[c], best[c - int(w)] + v)
    return -max(best)
