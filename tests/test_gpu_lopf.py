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


def test_scigrid_de_on_the_device_at_the_reference_tolerance():
    """scigrid-de (60,552 columns, 23,688 rows) at 1e-4, FP64 on the device,
    against PyPSA's objective within 2e-4 (LopfSuite.scala:519-555)."""
    from noaidi_b200.prima import cuda
    X.check_scigrid(lambda p, params: cuda.solve(p, params, precision=64))


@pytest.mark.parametrize("mixed", [False, True])
def test_scigrid_de_on_the_device_at_1e_6(mixed):
    """The tolerance the reference calls too slow for every commit (281,792
    iterations, 145 s on its CPU path, 2.66e-7 relative error): FP64 PDHG and
    the FP32 refinement scheme on the device, within 1e-5 of PyPSA."""
    from noaidi_b200.prima import PdhgParams, cuda
    params = PdhgParams(eps_abs=1e-6, eps_rel=1e-6, max_iterations=1_000_000)
    if mixed:
        X.check_scigrid(lambda p, q: cuda.mixed_solve(p, q).solution, params, 1e-5)
    else:
        X.check_scigrid(lambda p, q: cuda.solve(p, q, precision=64), params, 1e-5)
