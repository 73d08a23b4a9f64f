"""Branch-and-bound against an exact mixed-integer solver
(MilpAgreementSuite.scala, modules/prima-validation/src/test/scala/org/noaidi/
prima/validation/): the reference checks its search against ojAlgo 57.1.0's
MILP solver, which is absent here; scipy's HiGHS branch-and-cut stands in as
the exact, independent answer.  The search is noaidi_b200.prima.bnb with the
oracle solving every node relaxation, on the ladder of tests/milp_ladder.py.
Objectives are compared, not points: several integer points may share the
optimum."""
import numpy as np
import pytest

from noaidi_b200.prima import bnb
from noaidi_b200.prima.bnb import MilpStatus
from tests import bnb_fixtures as B
from tests import milp_ladder as L


def _search(inst):
    return bnb.solve_with(inst.problem, inst.integers, L.PARAMS, B.oracle_node_solver(inst.problem))


def _fractional(inst) -> int:
    from oracle import oracle as O
    relaxed = O.solve(inst.problem, L.PARAMS.lp)
    assert relaxed.status.name == "OPTIMAL", inst.name
    return sum(1 for j in inst.integers if abs(relaxed.primal[j] - round(relaxed.primal[j])) > 1e-4)


def _close(a, b):
    return abs(a - b) <= 1e-5 * max(1.0, abs(b))


def test_the_search_and_highs_agree_on_every_random_mixed_instance():
    """MilpAgreementSuite.scala:34-68: seeds 1-12, at least ten comparable,
    at least five with a fractional relaxation (so the search branches)."""
    checked = fractional = 0
    for seed in range(1, 13):
        inst = L.random_mixed(seed, 6 + seed % 4, 3 + seed % 3)
        if _fractional(inst) > 0:
            fractional += 1
        mine = _search(inst)
        status, objective = L.highs_milp(inst.problem, inst.integers)
        if status == "optimal":
            assert mine.status == MilpStatus.OPTIMAL, seed
            assert _close(inst.problem.primal_objective(mine.primal), objective), (seed, objective)
            checked += 1
        elif status == "infeasible":
            assert mine.status == MilpStatus.INFEASIBLE, seed
            checked += 1
    assert checked >= 10 and fractional >= 5


def test_the_search_never_beats_the_exact_optimum():
    """MilpAgreementSuite.scala:70-88: the objective of the returned point,
    never below HiGHS's optimum (a point below it would be infeasible)."""
    for seed in range(1, 13):
        inst = L.random_mixed(seed, 7, 4)
        mine = _search(inst)
        status, objective = L.highs_milp(inst.problem, inst.integers)
        if status == "optimal" and mine.primal.size:
            assert inst.problem.primal_objective(mine.primal) >= objective - 1e-5, seed


@pytest.mark.parametrize("inst", L.instances(), ids=lambda i: i.name)
def test_every_ladder_instance_requires_branching(inst):
    """MilpAgreementSuite.scala:90-105."""
    assert _fractional(inst) > 0


@pytest.mark.parametrize("inst", L.instances(), ids=lambda i: i.name)
def test_the_search_matches_highs_across_the_ladder(inst):
    """MilpAgreementSuite.scala:107-121."""
    mine = _search(inst)
    status, objective = L.highs_milp(inst.problem, inst.integers)
    assert status == "optimal" and mine.status == MilpStatus.OPTIMAL
    assert _close(mine.objective_value, objective)


@pytest.mark.parametrize("inst", L.instances(), ids=lambda i: i.name)
def test_the_returned_point_is_integral_and_feasible(inst):
    """MilpAgreementSuite.scala:123-165: integer columns exactly whole,
    bounds within 1e-6, rows within 1e-5 (equalities first, then >=)."""
    mine = _search(inst)
    assert mine.status == MilpStatus.OPTIMAL
    p, x = inst.problem, mine.primal
    for j in inst.integers:
        assert x[j] == round(x[j]), (inst.name, j, x[j])
    assert np.all(x >= p.variable_lower - 1e-6) and np.all(x <= p.variable_upper + 1e-6)
    kx = p.constraint_matrix.multiply(x)
    ne = p.num_equalities
    assert np.all(np.abs(kx[:ne] - p.rhs[:ne]) <= 1e-5)
    assert np.all(kx[ne:] >= p.rhs[ne:] - 1e-5)


def test_the_hand_derived_optima():
    """The ladder's documented optima: -20 for the fractional pair (relaxed
    -21), 2 and 3 for the odd set covers (relaxed 1.5 and 2.5)."""
    from oracle import oracle as O
    by_name = {i.name: i for i in L.instances()}
    for name, relaxed, integral in (("fractional-pair", -21.0, -20.0), ("set-cover-triangle", 1.5, 2.0),
                                    ("set-cover-k5-edges", 2.5, 3.0)):
        inst = by_name[name]
        assert O.solve(inst.problem, L.PARAMS.lp).objective_value == pytest.approx(relaxed, abs=1e-6)
        assert _search(inst).objective_value == pytest.approx(integral, abs=1e-6)
