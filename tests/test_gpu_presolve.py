"""Presolve and postsolve around the device solve: PresolveSuite's checks with
the GPU solving both the original and the reduced problem (including reduced
problems with no columns or no rows left)."""
import pytest

from tests import presolve_cases as X

pytestmark = pytest.mark.gpu


def test_presolve_suite_with_the_device():
    from noaidi_b200.prima import cuda
    X.run_all(lambda p: cuda.solve(p, X.PARAMS))


def test_mps_conventions_with_the_device():
    from noaidi_b200.prima import cuda
    from tests import mps_cases as M
    M.run_all(lambda p: cuda.solve(p, M.PARAMS))
