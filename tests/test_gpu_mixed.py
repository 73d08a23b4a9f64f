"""MixedPrecisionSuite (core/src/test/.../MixedPrecisionSuite.scala) against
the device mixed-precision solve, in both schemes: the reference's two-pass
(FP32 device pass, FP64 device finish) and the FP32 refinement (residual
problem around an FP64 anchor).  The reported answer must be FP64-validated:
objective within 1e-6 relative of the hand-derived optimum, KKT within the
caller's tolerance, status identical to the oracle's."""
import numpy as np
import pytest

from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, SolveStatus, convergence
from noaidi_b200.prima import generators as G
from oracle import oracle as O
from tests import lp_fixtures as F

pytestmark = pytest.mark.gpu

P9 = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=200_000)
SCHEMES = [0, 1]
IDS = ["two-pass", "refinement"]


def mixed(problem, params=P9, scheme=1, **kw):
    from noaidi_b200.prima import cuda
    return cuda.mixed_solve(problem, params, scheme=scheme, **kw)


@pytest.mark.parametrize("scheme", SCHEMES, ids=IDS)
@pytest.mark.parametrize("inst", F.optimal(), ids=lambda i: i.name)
def test_reaches_known_optimum(inst, scheme):
    r = mixed(inst.problem, scheme=scheme)
    assert r.solution.status == SolveStatus.OPTIMAL, r
    assert r.solution.objective_value == pytest.approx(inst.expected_objective,
                                                       abs=1e-6 * max(1.0, abs(inst.expected_objective)))


@pytest.mark.parametrize("scheme", SCHEMES, ids=IDS)
def test_refined_answer_meets_full_tolerance(scheme):
    p = F.economic_dispatch().problem
    r = mixed(p, scheme=scheme)
    assert r.refined
    conv = convergence(r.solution.kkt, float(np.linalg.norm(p.rhs)), float(np.linalg.norm(p.objective)), 1e-9, 1e-9)
    assert conv.converged, r.solution


@pytest.mark.parametrize("scheme", SCHEMES, ids=IDS)
def test_statuses_and_certificates(scheme):
    for inst in (F.infeasible(), F.unbounded()):
        assert mixed(inst.problem, scheme=scheme).solution.status == inst.expected_status
    strict = mixed(F.infeasible().problem, P9.copy(infeasibility_tolerance=1e-12), scheme=scheme)
    assert strict.refined and strict.solution.status == SolveStatus.PRIMAL_INFEASIBLE
    forced = mixed(F.infeasible().problem, scheme=scheme, mixed=MixedPrecisionParams(always_refine=True))
    assert forced.refined and forced.solution.status == SolveStatus.PRIMAL_INFEASIBLE


def test_float64_device_skips_the_reduced_pass():
    from noaidi_b200.prima import cuda
    r = cuda.mixed_solve(F.product_mix().problem, P9, ctx=cuda.context(0, 64))
    assert r.reduced_iterations == 0 and not r.refined
    assert r.solution.objective_value == pytest.approx(-36.0, abs=1e-6)


def test_two_pass_matches_the_reference_scheme_on_the_oracle():
    """Same scheme as MixedPrecision.solve with Float32Kernels: same statuses,
    objectives within the tolerance, reduced-pass iteration counts within a
    few evaluation periods."""
    for inst in F.optimal():
        ref = O.mixed_solve(inst.problem, P9)
        got = mixed(inst.problem, scheme=0)
        assert got.solution.status == ref.solution.status
        assert F.relative_gap(got.solution.objective_value, ref.solution.objective_value) <= 1e-8
        assert abs(got.reduced_iterations - ref.reduced_iterations) <= 128


@pytest.mark.parametrize("scheme", SCHEMES, ids=IDS)
def test_lopf_agrees_with_fp64_oracle(scheme):
    P = G.dc_lopf(seed=5, buses=150, lines=225, generators=75, snapshots=4)
    p = PdhgParams(eps_abs=1e-8, eps_rel=1e-8, max_iterations=400_000)
    ref = O.solve(P, p)
    r = mixed(P, p, scheme=scheme)
    assert r.solution.status == ref.status == SolveStatus.OPTIMAL
    assert F.relative_gap(r.solution.objective_value, ref.objective_value) <= 1e-8
    conv = convergence(r.solution.kkt, float(np.linalg.norm(P.rhs)), float(np.linalg.norm(P.objective)), 1e-8, 1e-8)
    assert conv.converged
    # the reported vectors really are the FP64-validated point
    check = O.kkt_evaluate(P, r.solution.primal, r.solution.dual)
    assert check.primal_residual_norm <= 1e-8 * (1 + np.linalg.norm(P.rhs)) * 1.01
    assert np.all(r.solution.primal >= P.variable_lower - 1e-12 * (1 + np.abs(P.variable_lower)))
    assert np.all(r.solution.primal <= P.variable_upper + 1e-12 * (1 + np.abs(P.variable_upper)))


def test_refinement_reaches_tolerances_fp32_alone_cannot():
    """Plain FP32 PDHG stalls far above 1e-9 on this LP; the anchored FP32
    refinement reaches it."""
    P = G.dc_lopf(seed=6, buses=100, lines=150, generators=50, snapshots=4)
    p = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=300_000)
    from noaidi_b200.prima import cuda
    plain = cuda.solve(P, p.copy(max_iterations=100_000), precision=32)
    assert plain.status != SolveStatus.OPTIMAL
    r = mixed(P, p, scheme=1)
    assert r.solution.status == SolveStatus.OPTIMAL and r.refined
