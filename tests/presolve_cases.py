"""PresolveSuite (modules/prima-core/src/test/scala/org/noaidi/prima/
PresolveSuite.scala) as functions of a solver, so the same checks run with
the oracle on CPU (test_presolve.py) and with the device (test_gpu_presolve.py).

The standard throughout, as in the reference: solving with presolve gives
the same status and objective as solving without, and the restored pair is
feasible and optimal for the ORIGINAL problem, duals and reduced costs
included."""
import math

import numpy as np
import pytest

from noaidi_b200.prima import LpProblem, PdhgParams, SolveStatus, convergence
from noaidi_b200.prima.presolve import presolve
from tests import lp_fixtures as F

PARAMS = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=100_000)


def agrees(problem, solve, hint):
    direct = solve(problem)
    result = presolve(problem)
    if result.proven_status is not None:
        assert result.proven_status == direct.status, hint
        with pytest.raises(RuntimeError):
            result.reduced
        with pytest.raises(RuntimeError):
            result.restore(direct)
        return
    restored = result.restore(solve(result.reduced))
    assert restored.status == direct.status, hint
    if direct.status != SolveStatus.OPTIMAL:
        return
    assert restored.objective_value == pytest.approx(direct.objective_value,
                                                     abs=1e-6 * max(1.0, abs(direct.objective_value))), hint
    kx = problem.constraint_matrix.multiply(restored.primal)
    neq = problem.num_equalities
    assert np.all(np.abs(kx[:neq] - problem.rhs[:neq]) <= 1e-6), hint
    assert np.all(kx[neq:] >= problem.rhs[neq:] - 1e-6), hint
    assert np.all(restored.primal >= problem.variable_lower - 1e-6), hint
    assert np.all(restored.primal <= problem.variable_upper + 1e-6), hint
    assert np.all(restored.dual[neq:] >= -1e-6), hint
    kty = problem.constraint_matrix.transpose.multiply(restored.dual)
    assert np.allclose(restored.reduced_costs, problem.objective - kty, atol=1e-6), hint
    conv = convergence(restored.kkt, float(np.linalg.norm(problem.rhs)), float(np.linalg.norm(problem.objective)),
                       1e-6, 1e-6)
    assert conv.converged, (hint, restored.kkt)


def build(n, objective, bounds, rows):
    """rows: (kind, [(col, coef)], value) with kind in 'eq', 'ge', 'le'."""
    b = LpProblem.builder(n)
    for j, c in enumerate(objective):
        b.objective_coefficient(j, c)
    for j, (lo, hi) in enumerate(bounds):
        b.bounds(j, lo, hi)
    for kind, coefs, value in rows:
        {"eq": b.equality_constraint, "ge": b.greater_than, "le": b.less_than}[kind](coefs, value)
    return b.build()[0]


INF = math.inf


def run_all(solve):
    """Every case of the suite against `solve(problem) -> LpSolution`."""
    for inst in F.conclusive():
        agrees(inst.problem, solve, inst.name)
    for seed in range(1, 9):
        agrees(F.random_feasible(seed, 40, 8, 14, 0.25), solve, f"random seed {seed}")

    # an unbounded objective survives presolve (:99-109)
    r = presolve(F.unbounded().problem)
    assert r.unbounded_if_feasible and r.proven_status is None
    assert r.restore(solve(r.reduced)).status == SolveStatus.DUAL_INFEASIBLE

    # an improving direction on an infeasible problem is not unboundedness (:111-138)
    p = build(3, [-1.0, 0, 0], [(0.0, INF)] * 3, [("ge", [(1, 1.0), (2, 1.0)], 10.0), ("le", [(1, 1.0), (2, 1.0)], 1.0)])
    assert solve(p).status == SolveStatus.PRIMAL_INFEASIBLE
    r = presolve(p)
    assert r.unbounded_if_feasible and r.proven_status is None
    assert r.restore(solve(r.reduced)).status == SolveStatus.PRIMAL_INFEASIBLE

    # a slack singleton row is priced at zero (:140-152)
    p = F.range_row().problem
    r = presolve(p)
    s = r.restore(solve(r.reduced))
    assert s.objective_value == pytest.approx(2.0, abs=1e-6)
    assert np.all(s.dual[p.num_equalities:] >= -1e-9)
    assert s.kkt.absolute_gap == pytest.approx(0.0, abs=1e-5)

    # a variable pinned by its own bounds (:160-181)
    p = build(2, [1.0, 5.0], [(0.0, 10.0), (3.0, 3.0)], [("ge", [(0, 1.0), (1, 1.0)], 4.0)])
    r = presolve(p)
    assert r.stats.fixed_columns == 1 and r.reduced.num_variables == 0
    s = r.restore(solve(r.reduced))
    assert s.status == SolveStatus.OPTIMAL and s.primal[1] == pytest.approx(3.0, abs=1e-9)
    assert s.objective_value == pytest.approx(16.0, abs=1e-6)

    # a singleton row becomes a bound and its dual is recovered (:183-201)
    p = build(1, [1.0], [(0.0, 100.0)], [("ge", [(0, 2.0)], 6.0)])
    r = presolve(p)
    assert r.stats.singleton_rows == 1 and r.reduced.num_constraints == 0
    s = r.restore(solve(r.reduced))
    assert s.primal[0] == pytest.approx(3.0, abs=1e-6) and s.objective_value == pytest.approx(3.0, abs=1e-6)
    assert s.dual[0] == pytest.approx(0.5, abs=1e-5)

    # an empty row that holds is dropped and priced at zero (:203-215)
    p = build(1, [1.0], [(2.0, 2.0)], [("ge", [(0, 1.0)], 1.0)])
    r = presolve(p)
    assert not r.proven_infeasible
    s = r.restore(solve(r.reduced))
    assert s.objective_value == pytest.approx(2.0, abs=1e-6) and s.dual[0] == 0.0

    # empty rows and singleton rows that cannot hold prove infeasibility (:217-236)
    assert presolve(build(1, [1.0], [(0.0, 0.0)], [("ge", [(0, 1.0)], 5.0)])).proven_infeasible
    assert presolve(build(1, [1.0], [(0.0, 1.0)], [("ge", [(0, 1.0)], 5.0)])).proven_infeasible

    # a variable in no row is set from its cost alone (:238-253)
    p = build(2, [1.0, -2.0], [(0.0, 10.0), (0.0, 4.0)], [("ge", [(0, 1.0)], 3.0)])
    r = presolve(p)
    assert r.stats.empty_columns >= 1
    s = r.restore(solve(r.reduced))
    assert s.primal[1] == pytest.approx(4.0, abs=1e-9) and s.objective_value == pytest.approx(-5.0, abs=1e-6)

    # reductions cascade across passes (:255-278)
    p = build(3, [1.0, 1.0, 1.0], [(0.0, 10.0), (0.0, 10.0), (5.0, 5.0)],
              [("eq", [(2, 1.0)], 5.0), ("eq", [(0, 1.0), (2, 1.0)], 9.0), ("eq", [(0, 1.0), (1, 1.0)], 6.0)])
    r = presolve(p)
    assert r.reduced.num_variables == 0
    s = r.restore(solve(r.reduced))
    assert s.primal[2] == pytest.approx(5.0, abs=1e-9)
    assert (s.primal[0], s.primal[1]) == (pytest.approx(4.0, abs=1e-6), pytest.approx(2.0, abs=1e-6))
    assert s.objective_value == pytest.approx(11.0, abs=1e-6)

    # nothing to reduce passes through unchanged (:280-286)
    p = F.economic_dispatch().problem
    r = presolve(p)
    assert r.stats.is_empty
    assert (r.reduced.num_variables, r.reduced.num_constraints) == (p.num_variables, p.num_constraints)
