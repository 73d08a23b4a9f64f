"""The reference's component suites, restated against the oracle and the
package's model types (CPU only): SparseMatrixSuite, LpBuilderSuite,
ScalingSuite, CertificatesSuite and the solver-behaviour parts of PdhgSuite /
MixedPrecisionSuite (prima-core/src/test/scala/org/noaidi/prima/*)."""
import ctypes
import math

import numpy as np
import pytest

from noaidi_b200.prima import (Direct, LpBuilder, LpProblem, MixedPrecisionParams, Negated, PdhgParams, Range,
                               ScalingParams, SolveStatus, SparseMatrix, WarmStart)
from oracle import oracle as O
from tests import lp_fixtures as F

INF = math.inf
P9 = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=200_000)


# -- SparseMatrixSuite.scala ---------------------------------------------------

def test_triplets_canonicalised_python_and_c():
    r, c, v = [1, 0, 0, 1, 0, 0], [2, 1, 1, 0, 0, 0], [5.0, 2.0, 3.0, 1.0, 4.0, -4.0]
    m = SparseMatrix.from_triplets(2, 3, r, c, v)
    assert m.nnz == 3
    assert list(m.col_indices) == [1, 0, 2]
    assert list(m.values) == [5.0, 1.0, 5.0]
    assert m(0, 1) == 5.0 and m(0, 0) == 0.0 and m(1, 2) == 5.0
    rp, ci, vv = O.csr_from_triplets(2, 3, r, c, v)
    assert list(rp) == list(m.row_ptr) and list(ci) == list(m.col_indices) and list(vv) == list(m.values)


def test_empty_rows_and_transpose():
    m = SparseMatrix.from_triplets(3, 2, [0, 2], [0, 1], [1.0, 2.0])
    assert list(m.row_ptr) == [0, 1, 1, 2]
    assert list(m.multiply([3.0, 4.0])) == [3.0, 0.0, 8.0]
    d = SparseMatrix.from_dense([[1.0, 0.0, 2.0], [0.0, 3.0, 0.0], [4.0, 5.0, 6.0]], 3)
    t = d.transpose
    for r in range(3):
        for c in range(3):
            assert t(c, r) == d(r, c)
    trp, tci, tv = O.csr_transpose(3, 3, d.row_ptr, d.col_indices, d.values)
    assert list(trp) == list(t.row_ptr) and list(tci) == list(t.col_indices) and list(tv) == list(t.values)


def test_norms_and_spectral_bound():
    m = SparseMatrix.from_dense([[1.0, -2.0], [3.0, 0.0]], 2)
    assert m.max_abs == 3.0 and m.norm_inf == 3.0
    assert m.norm_frobenius == pytest.approx(math.sqrt(14.0), abs=1e-12)
    col = SparseMatrix.from_triplets(25, 1, list(range(25)), [0] * 25, [1.0] * 25)
    assert col.norm_inf == 1.0 and col.norm1 == 25.0
    assert col.spectral_norm_bound == pytest.approx(5.0, abs=1e-12)
    assert O.spectral_norm_bound(col) == pytest.approx(5.0, abs=1e-12)


def test_non_finite_and_out_of_range_rejected():
    with pytest.raises(ValueError):
        SparseMatrix.from_triplets(1, 1, [0], [0], [INF])
    with pytest.raises(ValueError):
        SparseMatrix.from_triplets(1, 1, [0], [0], [math.nan])
    with pytest.raises(ValueError, match="row index 2 out of range"):
        SparseMatrix.from_triplets(2, 2, [2], [0], [1.0])
    with pytest.raises(ValueError):
        O.csr_from_triplets(1, 1, [0], [0], [INF])


def test_vstack():
    a = SparseMatrix.from_dense([[1.0, 2.0]], 2)
    s = SparseMatrix.vstack([a, SparseMatrix.zeros(2, 2), a])
    assert s.rows == 4 and s.nnz == 4
    assert list(s.multiply([1.0, 1.0])) == [3.0, 0.0, 0.0, 3.0]


def test_transpose_round_trips_and_keeps_non_square_columns_ascending():
    """SparseMatrixSuite.scala:26-48."""
    d = SparseMatrix.from_dense([[1.0, 0.0, 2.0], [0.0, 3.0, 0.0], [4.0, 5.0, 6.0]], 3)
    back = d.transpose.transpose
    assert list(back.values) == list(d.values) and list(back.col_indices) == list(d.col_indices)
    m = SparseMatrix.from_triplets(2, 4, [0, 0, 1, 1], [3, 1, 0, 3], [1.0, 2.0, 3.0, 4.0])
    t = m.transpose
    assert (t.rows, t.cols) == (4, 2)
    for r in range(t.rows):
        piece = list(t.col_indices[t.row_ptr[r]:t.row_ptr[r + 1]])
        assert piece == sorted(piece)


def test_multiply_agrees_with_the_dense_product_and_vstack_keeps_blocks():
    """SparseMatrixSuite.scala:50-65: index-order sums, exact here."""
    dense = [[1.0, 2.0, 0.0], [0.0, -1.0, 3.0]]
    x = [2.0, 3.0, 4.0]
    assert list(SparseMatrix.from_dense(dense, 3).multiply(x)) == [sum(a * b for a, b in zip(r, x)) for r in dense]
    a = SparseMatrix.from_dense([[1.0, 2.0]], 2)
    b = SparseMatrix.from_dense([[0.0, 3.0], [4.0, 0.0]], 2)
    s = SparseMatrix.vstack([a, b])
    assert (s.rows, s.nnz) == (3, 4) and s.to_dense().tolist() == [[1.0, 2.0], [0.0, 3.0], [4.0, 0.0]]


def test_a_diagonal_has_equal_induced_norms_under_its_spectral_bound():
    """SparseMatrixSuite.scala:82-98, the diagonal half."""
    d = SparseMatrix.from_triplets(3, 3, [0, 1, 2], [0, 1, 2], [2.0, -7.0, 3.0])
    assert d.norm1 == 7.0 and d.norm_inf == 7.0 and d.spectral_norm_bound >= 7.0 - 1e-12
    col = SparseMatrix.from_triplets(25, 1, list(range(25)), [0] * 25, [1.0] * 25)
    assert col.spectral_norm_bound > col.norm_inf


def test_scaled_by_applies_row_and_column_diagonals():
    """SparseMatrixSuite.scala:111-115."""
    m = SparseMatrix.from_dense([[1.0, 2.0], [3.0, 4.0]], 2)
    assert m.scaled_by([2.0, 10.0], [1.0, 0.5]).to_dense().tolist() == [[2.0, 2.0], [30.0, 20.0]]
    with pytest.raises(ValueError):
        m.scaled_by([1.0], [1.0, 1.0])


def test_out_of_range_indices_are_refused_with_the_reference_message():
    """SparseMatrixSuite.scala:117-121."""
    with pytest.raises(ValueError, match=r"row index 2 out of range \[0, 2\)"):
        SparseMatrix.from_triplets(2, 2, [2], [0], [1.0])


# -- LpBuilderSuite.scala ------------------------------------------------------

def test_duals_of_a_negated_row_come_back_with_the_callers_sign():
    """LpBuilderSuite.scala:47-52."""
    b = LpProblem.builder(1)
    b.less_than([(0, 1.0)], 3.0)
    _, t = b.build()
    assert list(t.original_duals([2.0])) == [-2.0]


def test_builder_orders_equalities_first():
    b = LpProblem.builder(2)
    b.greater_than([(0, 1.0)], 1.0)
    b.equality_constraint([(1, 1.0)], 5.0)
    b.less_than([(0, 1.0)], 9.0)
    b.equality_constraint([(0, 1.0), (1, 1.0)], 7.0)
    p, _ = b.build()
    assert p.num_equalities == 2 and p.num_constraints == 4
    assert p.rhs[0] == 5.0 and p.rhs[1] == 7.0


def test_builder_negation_and_ranges():
    b = LpProblem.builder(1)
    b.less_than([(0, 2.0)], 8.0)
    p, t = b.build()
    assert p.constraint_matrix(0, 0) == -2.0 and p.rhs[0] == -8.0
    assert t.expansion_of(0) == Negated(0)
    b = LpProblem.builder(1)
    b.constraint([(0, 1.0)], 2.0, 5.0)
    p, t = b.build()
    assert p.num_constraints == 2 and p.rhs[0] == 2.0 and p.rhs[1] == -5.0
    assert t.expansion_of(0) == Range(0, 1)
    assert list(t.original_duals([3.0, 0.0])) == [3.0]
    assert list(t.original_duals([0.0, 4.0])) == [-4.0]


def test_builder_rejections():
    with pytest.raises(ValueError):
        LpProblem.builder(1).constraint([(0, 1.0)], -INF, INF)
    with pytest.raises(ValueError):
        LpProblem.builder(1).bounds(0, 5.0, 1.0)
    b = LpProblem.builder(2)
    for f in (lambda: b.objective_coefficient(2, 1.0), lambda: b.bounds(-1, 0.0, 1.0),
              lambda: b.greater_than([(5, 1.0)], 0.0)):
        with pytest.raises(ValueError):
            f()
    b = LpProblem.builder(1)
    b.objective_coefficient(0, INF)
    b.bounds(0, 0.0, 1.0)
    b.greater_than([(0, 1.0)], 0.0)
    with pytest.raises(ValueError):
        b.build()


def test_objective_offset():
    b = LpProblem.builder(1)
    b.objective_coefficient(0, 2.0).bounds(0, 0.0, 10.0).objective_offset(100.0).greater_than([(0, 1.0)], 1.0)
    p, _ = b.build()
    assert p.primal_objective([3.0]) == 106.0
    base = F.equality_split().problem
    shifted = LpProblem(base.objective, base.constraint_matrix, base.rhs, base.num_equalities,
                        base.variable_lower, base.variable_upper, -1000.0)
    s = O.solve(shifted)
    assert s.status == SolveStatus.OPTIMAL
    assert s.objective_value == pytest.approx(24.0 - 1000.0, abs=1e-6)


# -- ScalingSuite.scala --------------------------------------------------------

def test_scaling_equilibrates():
    b = LpProblem.builder(3)
    for i in range(3):
        b.bounds(i, 0.0, 1.0)
    b.equality_constraint([(0, 1e6), (1, 2e6)], 1e6)
    b.equality_constraint([(1, 1e-3), (2, 3e-3)], 1e-3)
    p, _ = b.build()
    sv, *_ = O.scale(p)
    m = SparseMatrix(p.constraint_matrix.rows, p.constraint_matrix.cols, p.constraint_matrix.row_ptr,
                     p.constraint_matrix.col_indices, sv)
    for r in range(m.rows):
        vals = np.abs(m.values[m.row_ptr[r]:m.row_ptr[r + 1]])
        assert 0.05 < vals.max() < 20.0
    t = m.transpose
    for c in range(t.rows):
        vals = np.abs(t.values[t.row_ptr[c]:t.row_ptr[c + 1]])
        assert 0.05 < vals.max() < 20.0


def test_scaling_infinite_bounds_and_empty_lines():
    b = LpProblem.builder(2)
    b.bounds(0, -INF, INF).bounds(1, 0.0, INF)
    b.equality_constraint([(0, 3.0), (1, 4.0)], 12.0)
    p, _ = b.build()
    _, _, _, sl, su, _, _ = O.scale(p)
    assert sl[0] == -INF and su[0] == INF and sl[1] == 0.0 and su[1] == INF
    b = LpProblem.builder(2)
    b.bounds(0, 0.0, 1.0).bounds(1, 0.0, 1.0)
    b.equality_constraint([(0, 2.0)], 1.0)
    p, _ = b.build()
    sv, _, _, _, _, rs, cs = O.scale(p)
    assert np.all(np.isfinite(sv)) and np.all(sv != 0)
    assert np.all(np.isfinite(rs) & (rs > 0)) and np.all(np.isfinite(cs) & (cs > 0))


def test_scaling_none_is_identity():
    p = F.product_mix().problem
    sv, sc, sq, sl, su, rs, cs = O.scale(p, 0, False)
    assert list(sv) == list(p.constraint_matrix.values) and list(sq) == list(p.rhs)
    assert np.all(rs == 1.0) and np.all(cs == 1.0)


def test_scaled_optimum_stays_feasible_and_objective_invariant():
    inst = F.economic_dispatch()
    p = inst.problem
    sv, sc, sq, sl, su, rs, cs = O.scale(p)
    x = np.array(inst.expected_primal) / cs
    ms = SparseMatrix(p.constraint_matrix.rows, p.constraint_matrix.cols, p.constraint_matrix.row_ptr,
                      p.constraint_matrix.col_indices, sv)
    assert np.allclose(ms.multiply(x), sq, atol=1e-8)
    assert np.all(x >= sl - 1e-9) and np.all(x <= su + 1e-9)
    assert float(sc @ x) == pytest.approx(float(p.objective @ np.array(inst.expected_primal)), abs=1e-8)


def test_unscaling_recovers_the_original_coordinates():
    """ScalingSuite.scala:31-40: x / colScale then * colScale."""
    p = F.economic_dispatch().problem
    *_, cs = O.scale(p)
    point = 1.0 + 0.5 * np.arange(p.num_variables)
    assert np.allclose((point / cs) * cs, point, rtol=0, atol=1e-12)


# -- CertificatesSuite.scala ---------------------------------------------------

def _contradiction():
    b = LpProblem.builder(1)
    b.bounds(0, -INF, INF).greater_than([(0, 1.0)], 1.0).less_than([(0, 1.0)], 0.0)
    return b.build()[0]


def _absorbed(redundant=100.0):
    b = LpProblem.builder(1)
    b.bounds(0, 0.0, 5.0).less_than([(0, 1.0)], -1.0).less_than([(0, 1.0)], redundant)
    return b.build()[0]


def test_certificates_primal():
    c = _contradiction()
    assert O.primal_infeasibility(c, [1.0, 1.0]) == pytest.approx(0.0, abs=1e-12)
    assert O.primal_infeasibility(c, [1e9, 1e9]) == pytest.approx(O.primal_infeasibility(c, [1.0, 1.0]), abs=1e-12)
    assert O.primal_infeasibility(c, [0.0, 0.0]) is None
    assert O.primal_infeasibility(c, [0.0, 1.0]) is None
    assert O.primal_infeasibility(c, [-1.0, 0.0]) is None
    assert O.primal_infeasibility(_absorbed(), [2.0, 0.0]) == pytest.approx(0.0, abs=1e-12)
    assert O.primal_infeasibility(_absorbed(), [2.0, -1.0]) == pytest.approx(1.0 / math.sqrt(5.0), abs=1e-12)
    assert O.primal_infeasibility(_absorbed(1e10), [2.0, -1.0]) == pytest.approx(1.0 / math.sqrt(5.0), abs=1e-12)


def test_certificates_absorption_and_dilution():
    b = LpProblem.builder(1)
    b.bounds(0, 0.0, 5.0).greater_than([(0, 1.0)], 7.0)
    assert O.primal_infeasibility(b.build()[0], [1.0]) == pytest.approx(0.0, abs=1e-12)
    b = LpProblem.builder(1)
    b.bounds(0, 0.0, INF).greater_than([(0, 1.0)], 7.0)
    r = O.primal_infeasibility(b.build()[0], [1.0])
    assert r is None or r > 1e-6
    b = LpProblem.builder(1)
    b.bounds(0, 0.0, 5.0).less_than([(0, 1.0)], 1e10)
    feas = b.build()[0]
    r = O.primal_infeasibility(feas, [-1.0])
    assert r is None or r > 1e-3
    assert O.classify(feas, [0.0], [-1.0], 1e-8) is None
    b = LpProblem.builder(1)
    b.bounds(0, 0.0, INF).greater_than([(0, 1e-10)], 1.0)
    feas = b.build()[0]
    r = O.primal_infeasibility(feas, [1.0])
    assert r is None or r > 1e-3
    assert O.classify(feas, [0.0], [1.0], 1e-8) is None


def test_certificates_dual():
    b = LpProblem.builder(1)
    b.objective_coefficient(0, -1.0).bounds(0, 0.0, INF).greater_than([(0, 1.0)], 0.0)
    ray = b.build()[0]
    assert O.dual_infeasibility(ray, [1.0]) == pytest.approx(0.0, abs=1e-12)
    assert O.dual_infeasibility(ray, [0.0]) is None and O.dual_infeasibility(ray, [-1.0]) is None
    b = LpProblem.builder(1)
    b.objective_coefficient(0, -1.0).bounds(0, 0.0, 10.0).greater_than([(0, 1.0)], 0.0)
    r = O.dual_infeasibility(b.build()[0], [1.0])
    assert r is None or r > 1e-6
    b = LpProblem.builder(2)
    b.objective_coefficient(0, -1.0).bounds(0, 0.0, INF).bounds(1, 0.0, INF)
    b.equality_constraint([(0, 1.0), (1, 1.0)], 5.0)
    p = b.build()[0]
    for d in ([1.0, 0.0], [1.0, -1.0]):
        r = O.dual_infeasibility(p, d)
        assert r is None or r > 1e-6
    b = LpProblem.builder(2)
    b.objective_coefficient(0, -1e10).bounds(0, 0.0, 1.0).bounds(1, 0.0, 1.0).greater_than([(0, 1.0), (1, 1.0)], 0.0)
    bounded = b.build()[0]
    r = O.dual_infeasibility(bounded, [1.0, 1.0])
    assert r is None or r > 1e-3
    assert O.classify(bounded, [1.0, 1.0], [0.0], 1e-8) is None
    b = LpProblem.builder(1)
    b.objective_coefficient(0, -1.0).bounds(0, 0.0, INF).less_than([(0, 1e-9)], 0.0)
    r = O.dual_infeasibility(b.build()[0], [1.0])
    assert r is None or r > 1e-3


def test_classify_prefers_primal_and_units():
    b = LpProblem.builder(2)
    b.objective_coefficient(1, -1.0).bounds(0, -INF, INF).bounds(1, 0.0, INF)
    b.greater_than([(0, 1.0)], 1.0).less_than([(0, 1.0)], 0.0)
    assert O.classify(b.build()[0], [0.0, 1.0], [1.0, 1.0], 1e-8) == SolveStatus.PRIMAL_INFEASIBLE

    def shortfall(units):
        b = LpProblem.builder(1)
        b.bounds(0, 0.0, INF).greater_than([(0, units)], units * 7.0)
        return O.primal_infeasibility(b.build()[0], [1.0])

    base = shortfall(1.0)
    for t in (1e-8, 1e-4, 1.0, 1e4, 1e8):
        assert shortfall(t) == pytest.approx(base, abs=1e-9)
    s = O.solve(F.economic_dispatch().problem)
    assert O.classify(F.economic_dispatch().problem, s.primal, s.dual, 1e-8) is None


# -- PdhgSuite.scala / MixedPrecisionSuite.scala (solver behaviour) -------------

def test_statuses_and_limits():
    assert O.solve(F.infeasible().problem, P9).status == SolveStatus.PRIMAL_INFEASIBLE
    assert O.solve(F.unbounded().problem, P9).status == SolveStatus.DUAL_INFEASIBLE
    capped = O.solve(F.economic_dispatch().problem, PdhgParams(eps_abs=1e-14, eps_rel=1e-14, max_iterations=3))
    assert capped.status == SolveStatus.ITERATION_LIMIT and capped.iterations == 3
    b = LpProblem.builder(2)
    b.bounds(0, 0.0, 1.0).bounds(1, 0.0, 1.0)
    triv = O.solve(b.build()[0], P9)
    assert triv.status == SolveStatus.OPTIMAL and triv.iterations == 0
    timed = PdhgParams(eps_abs=1e-16, eps_rel=1e-16, max_iterations=50_000_000, time_limit_millis=50)
    s = O.solve(F.random_feasible(5, 200, 40, 80), timed)
    assert s.status == SolveStatus.TIME_LIMIT and s.iterations < 50_000_000


def test_cancellation_is_honoured_at_evaluation_points():
    flag = ctypes.c_int32(1)
    s = O.solve(F.random_feasible(5, 200, 40, 80), PdhgParams(eps_abs=1e-16, eps_rel=1e-16), cancel=flag)
    assert s.status == SolveStatus.INTERRUPTED and s.iterations == 64


def test_parameter_validation():
    for kw in ({"restart_artificial_fraction": 0.0}, {"restart_artificial_fraction": 1.5},
               {"infeasibility_tolerance": -1e-9}):
        with pytest.raises(ValueError):
            PdhgParams(**kw)


def test_stability_bound_and_restarts():
    b = LpProblem.builder(1)
    b.objective_coefficient(0, 1.0).bounds(0, 0.0, 10.0)
    for _ in range(100):
        b.greater_than([(0, 1.0)], 3.0)
    s = O.solve(b.build()[0], P9)
    assert s.status == SolveStatus.OPTIMAL and s.objective_value == pytest.approx(3.0, abs=1e-6)
    s = O.solve(F.random_feasible(7, 40, 8, 12), P9)
    assert s.status == SolveStatus.OPTIMAL and s.restarts > 0


def test_scaling_does_not_change_the_answer():
    unscaled = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, scaling=ScalingParams.none())
    for inst in F.optimal():
        a, b = O.solve(inst.problem, P9), O.solve(inst.problem, unscaled)
        assert b.status == SolveStatus.OPTIMAL
        assert a.objective_value == pytest.approx(b.objective_value, abs=1e-5 * max(1.0, abs(a.objective_value)))


def test_warm_starts():
    p = F.economic_dispatch().problem
    cold = O.solve(p, P9)
    warm = O.solve(p, P9, warm_start=WarmStart.from_solution(cold))
    assert warm.status == SolveStatus.OPTIMAL and warm.iterations < cold.iterations
    wild = WarmStart(np.array([1e6, -1e6]), np.array([-5.0]))
    s = O.solve(F.equality_split().problem, P9, warm_start=wild)
    assert s.status == SolveStatus.OPTIMAL and s.objective_value == pytest.approx(24.0, abs=1e-6)
    with pytest.raises(ValueError):
        O.solve(F.equality_split().problem, P9, warm_start=WarmStart(np.array([1.0]), np.array([0.0])))


def test_mixed_precision_behaviour():
    r = O.mixed_solve(F.economic_dispatch().problem, P9)
    assert r.refined and r.solution.status == SolveStatus.OPTIMAL
    cold = O.solve(F.economic_dispatch().problem, P9)
    assert 0 < r.reduced_iterations and r.refinement_iterations < cold.iterations
    for inst in (F.infeasible(), F.unbounded()):
        assert O.mixed_solve(inst.problem, P9).solution.status == inst.expected_status
    strict = O.mixed_solve(F.infeasible().problem, P9.copy(infeasibility_tolerance=1e-12))
    assert strict.refined and strict.solution.status == SolveStatus.PRIMAL_INFEASIBLE
    forced = O.mixed_solve(F.infeasible().problem, P9, MixedPrecisionParams(always_refine=True))
    assert forced.refined and forced.solution.status == SolveStatus.PRIMAL_INFEASIBLE
