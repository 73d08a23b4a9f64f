"""Presolve and postsolve (noaidi_b200/prima/presolve.py) with the oracle
solving both the original and the reduced problem."""
from tests import presolve_cases as X


def test_presolve_suite_with_the_oracle():
    from oracle import oracle as O
    X.run_all(lambda p: O.solve(p, X.PARAMS))
