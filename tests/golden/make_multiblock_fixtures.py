"""Records the oracle's and HiGHS's answers for the multi-block test LPs
(``tests/multiblock_cases.py``) in tests/golden/multiblock.json.

    python tests/golden/make_multiblock_fixtures.py

Per case: the problem's shape and byte hash (so a test can tell that the
generator still builds the same LP), scipy's HiGHS status and optimum, and
the oracle -- the C restatement of Pdhg.Solve -- in FP64 (ScalaKernels) at
relative KKT 1e-9 and in FP32 (Float32Kernels) at 1e-5: status, objective,
iterations and restarts.  About two minutes on one core.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from noaidi_b200.prima import PdhgParams  # noqa: E402
from noaidi_b200.prima.generators import problem_hash  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests import multiblock_cases as M  # noqa: E402

FP64_EPS = 1e-9
FP32_EPS = 1e-5


def highs(p):
    import scipy.sparse as sp
    from scipy.optimize import linprog
    K = p.constraint_matrix
    A = sp.csr_matrix((K.values, K.col_indices, K.row_ptr), shape=(K.rows, K.cols))
    neq = p.num_equalities
    bounds = [(None if np.isinf(a) else a, None if np.isinf(b) else b)
              for a, b in zip(p.variable_lower, p.variable_upper)]
    r = linprog(p.objective, A_ub=-A[neq:] if neq < K.rows else None, b_ub=-p.rhs[neq:] if neq < K.rows else None,
                A_eq=A[:neq] if neq else None, b_eq=p.rhs[:neq] if neq else None, bounds=bounds, method="highs")
    # scipy: 0 optimal, 2 infeasible, 3 unbounded
    return {"status": {0: "OPTIMAL", 2: "PRIMAL_INFEASIBLE", 3: "DUAL_INFEASIBLE"}.get(r.status, str(r.status)),
            "objective": float(r.fun) if r.status == 0 else None}


def oracle(p, mode, eps):
    params = PdhgParams(eps_abs=eps, eps_rel=eps, max_iterations=400_000,
                        infeasibility_tolerance=max(eps, 1e-8))
    s = O.solve(p, params, mode=mode)
    return {"eps": eps, "status": s.status.name, "objective": s.objective_value, "iterations": s.iterations,
            "restarts": s.restarts}


def main():
    out = {}
    for name, make in M.CASES.items():
        p = make()
        rec = {"n": p.num_variables, "m": p.num_constraints, "nnz": int(p.constraint_matrix.nnz),
               "hash": problem_hash(p), "highs": highs(p), "oracle_fp64": oracle(p, O.FP64, FP64_EPS),
               "oracle_fp32": oracle(p, O.FP32, FP32_EPS)}
        out[name] = rec
        print(name, json.dumps(rec), flush=True)
    with open(os.path.join(HERE, "multiblock.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
