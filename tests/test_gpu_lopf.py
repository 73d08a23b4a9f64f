"""PyPSA's ac-dc-dispatch LOPF solved on the device, in FP64 and with the FP32
refinement scheme, against PyPSA's optimum (LopfSuite.scala:115-207)."""
import pytest

from tests import lopf_cases as X

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", X.NETWORKS)
def test_lopf_matches_pypsa_fp64_device(name):
    from noaidi_b200.prima import cuda
    X.check_against_pypsa(lambda p: cuda.solve(p, X.PARAMS, precision=64), name)


@pytest.mark.parametrize("name", X.NETWORKS)
def test_lopf_matches_pypsa_fp32_refinement(name):
    from noaidi_b200.prima import cuda
    X.check_against_pypsa(lambda p: cuda.mixed_solve(p, X.PARAMS).solution, name)


def test_sclopf_matches_pypsa_on_the_device():
    from noaidi_b200.prima import cuda
    X.check_sclopf_triangle(lambda p: cuda.solve(p, X.PARAMS, precision=64))
    X.check_sclopf_triangle(lambda p: cuda.mixed_solve(p, X.PARAMS).solution)
