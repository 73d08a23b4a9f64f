"""The MPS reader (noaidi_b200/prima/mps.py), with the oracle solving the
parsed problems."""
from tests import mps_cases as X


def test_mps_conventions_with_the_oracle():
    from oracle import oracle as O
    X.run_all(lambda p: O.solve(p, X.PARAMS))


def test_malformed_mps_is_rejected():
    X.check_rejections()
