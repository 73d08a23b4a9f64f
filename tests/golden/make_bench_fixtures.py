"""Records HiGHS's optimum of the bench workload in tests/golden/bench_highs.json.

    python tests/golden/make_bench_fixtures.py [seed ...]      (default: 0 1 2)

The workload is the seeded 1.34M-column DC-LOPF dispatch LP
(``generators.dc_lopf`` with 2,000 buses, 3,000 lines, 1,000 generators and
168 hourly snapshots).  Nothing couples its snapshots -- every row of
snapshot t touches only snapshot t's columns -- so the LP is 168 independent
LPs and its optimum is the sum of theirs.  The script checks that block
structure on the assembled matrix, solves each snapshot's LP with scipy's
HiGHS (dual simplex) and records, per seed, the summed optimum with the
instance's byte hash.  (HiGHS on the assembled 1.34M-column LP runs for
longer than a quarter of an hour on this container's cores; the blocks take
about a minute.)  The bench reports its answer's relative error against
this number.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from noaidi_b200.prima import generators as G  # noqa: E402
from noaidi_b200.prima.generators import problem_hash  # noqa: E402

WORKLOAD = dict(buses=2000, lines=3000, generators=1000, snapshots=168)


def snapshot_blocks(p, T):
    """Row and column ranges of the T diagonal blocks; raises if any row
    reaches outside its snapshot's columns."""
    K = p.constraint_matrix
    m, n = p.num_constraints, p.num_variables
    assert m % T == 0 and n % T == 0
    mr, nc = m // T, n // T
    rows_snap = np.repeat(np.arange(m) // mr, np.diff(K.row_ptr))
    cols_snap = K.col_indices // nc
    assert np.array_equal(rows_snap, cols_snap), "a row couples two snapshots"
    assert p.num_equalities == m, "the dispatch LP has equality rows only"
    return mr, nc


def highs_by_snapshot(p, T):
    import scipy.sparse as sp
    from scipy.optimize import linprog
    mr, nc = snapshot_blocks(p, T)
    K = p.constraint_matrix
    A = sp.csr_matrix((K.values, K.col_indices, K.row_ptr), shape=(K.rows, K.cols))
    total = 0.0
    for t in range(T):
        rs, cs = slice(t * mr, (t + 1) * mr), slice(t * nc, (t + 1) * nc)
        lo, hi = p.variable_lower[cs], p.variable_upper[cs]
        bounds = [(None if np.isinf(a) else a, None if np.isinf(b) else b) for a, b in zip(lo, hi)]
        r = linprog(p.objective[cs], A_eq=A[rs, cs], b_eq=p.rhs[rs], bounds=bounds, method="highs-ds")
        if r.status != 0:
            raise RuntimeError(f"snapshot {t}: HiGHS status {r.status} ({r.message})")
        total += float(r.fun)
    return total


def main(seeds):
    path = os.path.join(HERE, "bench_highs.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for seed in seeds:
        p = G.dc_lopf(seed=seed, **WORKLOAD)
        t = time.time()
        obj = highs_by_snapshot(p, WORKLOAD["snapshots"])
        out[str(seed)] = {"hash": problem_hash(p), "n": p.num_variables, "m": p.num_constraints,
                          "nnz": int(p.constraint_matrix.nnz), "highs_objective": obj,
                          "method": "scipy linprog highs-ds, snapshot by snapshot (the LP's 168 diagonal blocks)"}
        print(seed, out[str(seed)], f"{time.time() - t:.1f} s", flush=True)
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main([int(s) for s in sys.argv[1:]] or [0, 1, 2])
