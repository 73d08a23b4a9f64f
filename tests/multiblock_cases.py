"""LPs large enough that the device solver runs them on a multi-block team.

A problem of up to 4,096 rows and columns is solved by one block of the
persistent kernel; anything larger is spread over ceil(max(n, m) / 512)
co-resident blocks (at most the whole grid), with a grid-wide team barrier
between phases, FP64 block partials reduced across blocks and phase-B tiles
staged during the barrier.  These instances are that path at test size
(between 16 and 64 blocks), each with the oracle's answer recorded in
``tests/golden/multiblock.json`` by ``tests/golden/make_multiblock_fixtures.py``:
the oracle needs 20-30 s per FP64 solve at this size, too slow to rerun in
every test.

* two DC-LOPF dispatch LPs (``generators.dc_lopf``), the bench workload's
  family at 29k and 32k columns;
* a random sparse LP (``generators.random_sparse_lp``, 8,000 columns) whose
  first row cannot be met inside the box: primal infeasible;
* a random sparse LP whose first column is free above, costs -1 and only
  loosens the rows it touches: dual infeasible (unbounded).
"""
from __future__ import annotations

import numpy as np

from noaidi_b200.prima import generators as G
from noaidi_b200.prima.model import LpProblem, SparseMatrix


def lopf_300x24() -> LpProblem:
    return G.dc_lopf(seed=1, buses=300, lines=450, generators=150, snapshots=24)


def lopf_500x16() -> LpProblem:
    return G.dc_lopf(seed=2, buses=500, lines=750, generators=250, snapshots=16)


def sparse_infeasible() -> LpProblem:
    """Ax <= b, 0 <= x <= 10 with b_0 one below the least value row 0 takes
    on the box (the rows enter standard form negated: -Ax >= -b)."""
    p = G.random_sparse_lp(seed=3, m=5000, n=8000)
    K = p.constraint_matrix
    lo, hi = K.row_ptr[0], K.row_ptr[1]
    a = -K.values[lo:hi]  # row 0 of A
    least = float(np.minimum(0.0, 10.0 * a).sum())
    q = p.rhs.copy()
    q[0] = -(least - 1.0)
    return LpProblem(p.objective, K, q, p.num_equalities, p.variable_lower, p.variable_upper)


def sparse_unbounded() -> LpProblem:
    """Column 0 gets no upper bound, cost -1 and non-positive coefficients in
    A (so raising it only loosens Ax <= b): a recession direction."""
    p = G.random_sparse_lp(seed=4, m=5000, n=8000)
    K = p.constraint_matrix
    vals = K.values.copy()
    col0 = K.col_indices == 0
    vals[col0] = np.abs(vals[col0])  # -A in standard form: A's entries become -|a|
    c = p.objective.copy()
    c[0] = -1.0
    hi = p.variable_upper.copy()
    hi[0] = np.inf
    K2 = SparseMatrix(K.rows, K.cols, K.row_ptr, K.col_indices, vals)
    return LpProblem(c, K2, p.rhs, p.num_equalities, p.variable_lower, hi)


CASES = {
    "lopf-300x24": lopf_300x24,
    "lopf-500x16": lopf_500x16,
    "sparse-infeasible-8000": sparse_infeasible,
    "sparse-unbounded-8000": sparse_unbounded,
}
OPTIMAL = ["lopf-300x24", "lopf-500x16"]
