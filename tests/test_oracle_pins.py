"""Pins the C restatement (the oracle) against every known answer the
reference publishes for this path, before anything is compared against it.

Sources: the validation ladder and its published trajectory
(core/NOTES.md:45-58), the mixed-precision figures (core/NOTES.md:208-240),
the hand-derived fixture optima (LpFixtures.scala:25-159) and an independent
simplex (scipy HiGHS, standing in for the absent ojAlgo oracle).
"""
import json
import math
import os

import numpy as np
import pytest

from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, SolveStatus
from oracle import oracle as O
from tests import lp_fixtures as F

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))
LADDER = {e.name: e for e in F.ladder()}
P9 = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=500_000)


def _size(p):
    return f"{p.num_variables}v/{p.num_constraints}c/{p.constraint_matrix.nnz}nz"


@pytest.mark.parametrize("name", list(PINS["ladder_eps_1e-9"].keys())[2:])
def test_ladder_matches_published_report(name):
    size, iters, restarts, obj, status = PINS["ladder_eps_1e-9"][name]
    e = LADDER[name]
    assert _size(e.problem) == size  # the java.util.Random restatement rebuilt the same instance
    s = O.solve(e.problem, P9)
    assert s.status == SolveStatus[status]
    if obj is not None:
        assert round(s.objective_value, 6) == pytest.approx(obj, abs=1.5e-6)
    if name in PINS["ladder_trajectory_exact"]:
        assert (s.iterations, s.restarts) == (iters, restarts)
    else:
        # one-ulp libm differences (JVM vs glibc pow/exp/log) move these
        # trajectories by whole evaluation periods; the band is what survives
        assert abs(s.iterations - iters) <= 0.25 * iters


def test_ladder_worst_gap_against_highs():
    scipy_opt = pytest.importorskip("scipy.optimize")
    worst = 0.0
    for e in F.ladder():
        if e.expected is not SolveStatus.OPTIMAL:
            continue
        P = e.problem
        K = P.constraint_matrix.to_dense()
        neq = P.num_equalities
        res = scipy_opt.linprog(P.objective, A_ub=-K[neq:] if P.num_constraints > neq else None,
                                b_ub=-P.rhs[neq:] if P.num_constraints > neq else None,
                                A_eq=K[:neq] if neq else None, b_eq=P.rhs[:neq] if neq else None,
                                bounds=list(zip(P.variable_lower, P.variable_upper)), method="highs")
        assert res.status == 0
        s = O.solve(P, P9)
        worst = max(worst, F.relative_gap(s.objective_value, res.fun + P.objective_offset))
    assert worst <= PINS["ladder_worst_gap_bound"]["value"]


@pytest.mark.parametrize("inst", F.optimal(), ids=lambda i: i.name)
@pytest.mark.parametrize("mode", [O.FP64, O.FP32], ids=["fp64", "fp32"])
def test_fixture_optima(inst, mode):
    params = P9 if mode == O.FP64 else PdhgParams(eps_abs=1e-5, eps_rel=1e-5, max_iterations=200_000)
    tol = 1e-6 if mode == O.FP64 else 1e-3
    s = O.solve(inst.problem, params, mode=mode)
    assert s.status == SolveStatus.OPTIMAL
    assert s.objective_value == pytest.approx(inst.expected_objective, abs=tol * max(1.0, abs(inst.expected_objective)))
    if mode == O.FP64:
        for v, e in zip(s.primal, inst.expected_primal):
            assert v == pytest.approx(e, abs=1e-5)


@pytest.mark.parametrize("tol,saved", [(1e-9, 0), (1e-6, 1)])
@pytest.mark.parametrize("name", ["economic-dispatch", "equality-split", "range-row"])
def test_mixed_precision_work_saved(name, tol, saved):
    p = PdhgParams(eps_abs=tol, eps_rel=tol, max_iterations=500_000)
    r = O.mixed_solve(LADDER[name].problem, p)
    cold = O.solve(LADDER[name].problem, p)
    assert r.solution.status == SolveStatus.OPTIMAL
    pct = 100.0 * (1.0 - r.refinement_iterations / cold.iterations) if r.refined else 100.0
    assert math.floor(pct + 0.5) == PINS["mixed_precision_fp64_work_saved_pct"][name][saved]


def test_mixed_precision_published_iteration_counts():
    pins = PINS["mixed_precision_iterations"]
    prob = LADDER["random-600x400"].problem
    r = O.mixed_solve(prob, PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=500_000))
    assert r.reduced_iterations == pins["random-600x400_fp32_pass_to_1e-5"]
    cold = O.solve(prob, PdhgParams(eps_abs=1e-6, eps_rel=1e-6, max_iterations=500_000))
    assert cold.iterations == pins["random-600x400_cold_fp64_1e-6"]


def test_congestion_prices():
    s = O.solve(F.economic_dispatch().problem, P9)
    pin = PINS["fixtures"]["economic_dispatch_prices"]
    assert s.dual[0] == pytest.approx(s.dual[1], abs=1e-4)
    assert abs(s.dual[2] - s.dual[3]) > 1.0
    assert s.dual[2] == pytest.approx(pin["A2"], abs=pin["tolerance"])
    assert s.dual[3] == pytest.approx(pin["B2"], abs=pin["tolerance"])
