"""Branch-and-bound with every node relaxation on the GPU (one resident
matrix, bounds replaced per node by prima_problem_set_bounds) against the
same search with the oracle solving the nodes, and against the hand-derived
optima of BranchAndBoundSuite."""
import pytest

from noaidi_b200.prima import bnb
from noaidi_b200.prima.bnb import MilpStatus
from tests import bnb_fixtures as X

pytestmark = pytest.mark.gpu

P = X.PARAMS

CASES = [
    ("knapsackish", X.knapsackish, {0, 1}, -20.0),
    ("knapsackish-a-only", X.knapsackish, {0}, -21.0),
    ("binaries", X.binaries, {0, 1, 2}, -7.0),
    ("no-integer-point", X.no_integer_point, {0}, None),
]


@pytest.mark.parametrize("name,make,ints,optimum", CASES, ids=[c[0] for c in CASES])
def test_device_search_matches_the_oracle_search(name, make, ints, optimum):
    problem = make()
    dev = bnb.solve(problem, ints, P)
    ref = bnb.solve_with(problem, ints, P, X.oracle_node_solver(problem))
    assert dev.status == ref.status
    if optimum is None:
        assert dev.status == MilpStatus.INFEASIBLE
    else:
        assert dev.status == MilpStatus.OPTIMAL
        assert dev.objective_value == pytest.approx(optimum, abs=1e-6)
        for j in range(len(dev.primal)):  # integer columns are snapped: exact; the rest to the LP tolerance
            if j in ints:
                assert dev.primal[j] == ref.primal[j]
            else:
                assert dev.primal[j] == pytest.approx(ref.primal[j], abs=1e-6)


def test_device_search_on_the_16_item_knapsack():
    hard, values, weights = X.hard_knapsack()
    optimum = X.knapsack_optimum(values, weights, 120)
    dev = bnb.solve(hard, set(range(16)), P)
    assert dev.status == MilpStatus.OPTIMAL
    assert dev.objective_value == pytest.approx(optimum, abs=1e-6)
    assert sum(w for w, x in zip(weights, dev.primal) if x == 1.0) <= 120


def test_set_bounds_then_solve_equals_a_fresh_solve():
    """A node solved on the resident problem equals a one-shot solve of the
    same LP with those bounds, bit for bit (same equilibration, same start)."""
    import numpy as np
    from noaidi_b200.prima import LpProblem, cuda
    problem = X.knapsackish()
    resident = cuda.DeviceProblem(problem, P.lp)
    lo, hi = np.array([0.0, 1.0]), np.array([3.0, 10.0])
    resident.set_bounds(lo, hi)
    got = resident.solve(P.lp)
    fresh = cuda.solve(LpProblem(problem.objective, problem.constraint_matrix, problem.rhs, problem.num_equalities,
                                 lo, hi, problem.objective_offset), P.lp)
    assert (got.status, got.iterations, got.objective_value) == (fresh.status, fresh.iterations, fresh.objective_value)
    assert list(got.primal) == list(fresh.primal)
    with pytest.raises(ValueError):
        resident.set_bounds(np.array([1.0, 0.0]), np.array([0.0, 1.0]))
    resident.free()
