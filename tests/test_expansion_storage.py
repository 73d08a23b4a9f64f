"""The capacity-expansion LOPF with storage over a year of hours
(noaidi_b200/network/synthetic.py): the array-built LP is the LOPF builder's
LP entry for entry, and a small case reaches HiGHS's optimum."""
import numpy as np
import pytest

from noaidi_b200.network import lopf
from noaidi_b200.network import synthetic as S
from noaidi_b200.prima import PdhgParams

SMALL = [(0, 12, 18, 20, 4, 30), (3, 30, 45, 60, 7, 49), (5, 8, 12, 10, 0, 24)]


@pytest.mark.parametrize("args", SMALL)
def test_the_array_built_lp_is_the_builders(args):
    a = lopf.build(S.expansion_storage_network(*args)).problem
    b = S.expansion_storage(*args)
    assert (a.num_variables, a.num_constraints, a.num_equalities) == \
        (b.num_variables, b.num_constraints, b.num_equalities)
    Ka, Kb = a.constraint_matrix, b.constraint_matrix
    for x, y in ((Ka.row_ptr, Kb.row_ptr), (Ka.col_indices, Kb.col_indices), (Ka.values, Kb.values),
                 (a.rhs, b.rhs), (a.objective, b.objective), (a.variable_lower, b.variable_lower),
                 (a.variable_upper, b.variable_upper)):
        assert np.array_equal(x, y)
    assert a.objective_offset == b.objective_offset


def test_a_small_year_slice_matches_highs():
    import scipy.optimize as so
    import scipy.sparse as sp
    from oracle import oracle as O
    p = S.expansion_storage(0, 12, 18, 20, 4, 48)
    s = O.solve(p, PdhgParams(eps_abs=1e-8, eps_rel=1e-8, max_iterations=400_000))
    assert s.status.name == "OPTIMAL"
    K = p.constraint_matrix
    A = sp.csr_matrix((K.values, K.col_indices, K.row_ptr), shape=(p.num_constraints, p.num_variables))
    neq = p.num_equalities
    r = so.linprog(p.objective, A_ub=-A[neq:], b_ub=-p.rhs[neq:], A_eq=A[:neq], b_eq=p.rhs[:neq],
                   bounds=list(zip(p.variable_lower, p.variable_upper)), method="highs")
    assert r.status == 0
    assert s.objective_value == pytest.approx(r.fun + p.objective_offset, rel=1e-8)


def test_the_full_size_has_the_configured_shape():
    """200 buses, 300 lines, 400 extendable generators, 50 storage units,
    8,760 hours: 400 + 8760 (400 + 300 + 4 x 50) columns, balance, state of
    charge and 101 Kirchhoff rows per hour, two capacity rows per generator
    and hour."""
    p = S.expansion_storage()
    T = 8760
    assert p.num_variables == 400 + T * 900
    assert p.num_equalities == T * 200 + 50 * T + T * 101
    assert p.num_constraints == p.num_equalities + 2 * 400 * T
    assert 25e6 < p.constraint_matrix.nnz < 32e6
