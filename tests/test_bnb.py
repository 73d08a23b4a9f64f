"""BranchAndBoundSuite's search logic (noaidi_b200/prima/bnb.py) on CPU, with
the oracle solving each node's relaxation.  The device variant of the same
searches is tests/test_gpu_bnb.py."""
import math

import numpy as np
import pytest

from noaidi_b200.prima import PdhgParams, bnb
from noaidi_b200.prima.bnb import MilpStatus
from noaidi_b200.prima.model import LpBuilder
from tests import bnb_fixtures as X

P = X.PARAMS


def run(problem, integers, params=P):
    return bnb.solve_with(problem, set(integers), params, X.oracle_node_solver(problem))


def test_integer_optimum_differs_from_the_fractional_relaxation():
    m = run(X.knapsackish(), {0, 1})
    assert m.status == MilpStatus.OPTIMAL
    assert m.objective_value == pytest.approx(-20.0, abs=1e-6)
    assert (m.primal[0], m.primal[1]) == (4.0, 0.0)
    assert all(v == round(v) for v in m.primal)


def test_one_integer_column_keeps_the_other_fractional():
    m = run(X.knapsackish(), {0})
    assert m.status == MilpStatus.OPTIMAL
    assert m.objective_value == pytest.approx(-21.0, abs=1e-6)
    assert m.primal[0] == 3.0 and abs(m.primal[1] - 1.5) < 1e-5


def test_empty_integer_set_is_the_relaxation():
    m = run(X.knapsackish(), set())
    assert m.status == MilpStatus.OPTIMAL and m.nodes_explored == 1
    assert m.objective_value == pytest.approx(-21.0, abs=1e-6)


def test_no_integer_point_is_proven_infeasible():
    assert run(X.no_integer_point(), {0}).status == MilpStatus.INFEASIBLE


def test_binaries():
    m = run(X.binaries(), {0, 1, 2})
    assert m.status == MilpStatus.OPTIMAL and m.objective_value == pytest.approx(-7.0, abs=1e-6)
    assert list(m.primal) == [1.0, 0.0, 1.0]


def test_bound_brackets_the_optimum_and_limits_downgrade():
    m = run(X.knapsackish(), {0, 1})
    assert m.best_bound <= m.objective_value + 1e-9 and m.gap <= 1e-6
    capped = run(X.knapsackish(), {0, 1}, P.copy(max_nodes=1))
    assert capped.status != MilpStatus.OPTIMAL and not capped.status.is_conclusive


def test_warm_start_does_not_change_the_answer():
    cold = run(X.knapsackish(), {0, 1}, P.copy(warm_start=False))
    warm = run(X.knapsackish(), {0, 1}, P.copy(warm_start=True))
    assert warm.status == cold.status and warm.objective_value == pytest.approx(cold.objective_value, abs=1e-9)
    assert list(warm.primal) == list(cold.primal)


def test_out_of_range_integer_column_is_rejected():
    with pytest.raises(ValueError):
        run(X.knapsackish(), {0, 7})


def test_nan_bounds_never_skip_and_unknown_bounds_are_minus_infinity():
    assert not bnb.skips_before_solving(math.nan, 10.0, True)
    assert not bnb.skips_before_solving(-math.inf, 10.0, True)
    assert bnb.skips_before_solving(11.0, 10.0, True)
    assert not bnb.skips_before_solving(9.0, 10.0, True)
    assert not bnb.skips_before_solving(11.0, math.inf, False)
    assert bnb.safe_bound_of(True, 5.0, 1.0) == 4.0
    assert bnb.safe_bound_of(True, math.nan, 1.0) == -math.inf
    assert bnb.safe_bound_of(True, 5.0, math.nan) == -math.inf
    assert bnb.safe_bound_of(False, 5.0, 1.0) == -math.inf


def test_most_fractional_and_snap_round_half_up():
    assert bnb.most_fractional([0.5, 0.2, 2.0], [0, 1, 2], 1e-6) == 0
    assert bnb.most_fractional([1.0, 2.0], [0, 1], 1e-6) is None
    assert list(bnb.snap(np.array([0.5, 1.4999, -0.5]), [0, 1, 2])) == [1.0, 1.0, 0.0]


def test_pruning_margin_only_costs_nodes():
    hard, values, weights = X.hard_knapsack()
    optimum = X.knapsack_optimum(values, weights, 120)
    bare = run(hard, range(16), P.copy(pruning_safety_factor=0.0))
    margined = run(hard, range(16))
    for r in (bare, margined):
        assert r.status == MilpStatus.OPTIMAL and r.objective_value == pytest.approx(optimum, abs=1e-6)
    assert margined.nodes_explored >= bare.nodes_explored


def test_an_unconverged_relaxation_downgrades_and_is_counted():
    """BranchAndBoundSuite.scala:213-223: starved nodes prove nothing, so the
    result is not conclusive and says how many nodes were unproven."""
    starved = P.copy(lp=PdhgParams(eps_abs=1e-14, eps_rel=1e-14, max_iterations=2))
    m = bnb.solve_with(X.knapsackish(), {0, 1}, starved, X.oracle_node_solver(X.knapsackish()))
    assert m.status != MilpStatus.OPTIMAL and not m.status.is_conclusive
    assert m.unproven_nodes > 0


def test_a_warm_start_from_an_unusable_solution_is_declined():
    """BranchAndBoundSuite.scala:225-250: a non-finite iterate cannot seed a
    child; WarmStart refuses it and the search declines rather than throws."""
    from noaidi_b200.prima.types import KktError, LpSolution, SolveStatus, WarmStart
    poisoned = LpSolution(SolveStatus.NUMERICAL_ERROR, np.array([1.0, 2.0]), np.array([math.nan]),
                          np.array([0.0, 0.0]), 1.0, 1.0, 1, 0, 0, KktError(0.0, 0.0, 1.0, 1.0))
    with pytest.raises(ValueError):
        WarmStart.from_solution(poisoned)
    from oracle import oracle as O
    good = O.solve(X.knapsackish(), P.lp)
    assert WarmStart.from_solution(good) is not None


def test_an_unbounded_relaxation_is_reported_unbounded():
    b = LpBuilder(1)
    b.objective_coefficient(0, -1.0)
    b.bounds(0, 0.0, math.inf)
    p = b.build()[0]
    assert run(p, {0}).status == MilpStatus.UNBOUNDED


def test_a_time_limit_stops_the_search_without_claiming_optimality():
    """BranchAndBoundSuite.scala:261-288 on the sixteen-item knapsack."""
    p = X.hard_knapsack()[0]
    ints = set(range(p.num_variables))
    full = run(p, ints)
    assert full.status == MilpStatus.OPTIMAL and full.nodes_explored > 50
    limited = run(p, ints, P.copy(time_limit_millis=0))
    assert limited.nodes_explored <= full.nodes_explored
    if full.solve_time_millis > 5:
        assert limited.status != MilpStatus.OPTIMAL and limited.nodes_explored < full.nodes_explored


def test_the_reported_objective_is_that_of_the_reported_point():
    p = X.knapsackish()
    m = run(p, {0, 1})
    assert m.status == MilpStatus.OPTIMAL
    assert m.objective_value == pytest.approx(p.primal_objective(m.primal), abs=1e-12)


def test_no_answer_means_no_point_on_the_short_circuit_path():
    b = LpBuilder(1)
    b.objective_coefficient(0, 1.0)
    b.bounds(0, 0.0, 1.0)
    b.equality_constraint([(0, 1.0)], 5.0)  # outside the box
    m = run(b.build()[0], set())
    assert m.status == MilpStatus.INFEASIBLE and m.primal.size == 0
