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


@pytest.mark.parametrize("mixed", [False, True])
def test_prices_from_the_device(mixed):
    """Nodal prices (balance-row duals) from the device solve: every interior
    zero-emission generator is priced at its marginal cost."""
    import numpy as np
    from noaidi_b200.network import lopf
    from noaidi_b200.prima import cuda
    n = X.network("ac-dc-dispatch")
    model = lopf.build(n)
    sol = cuda.mixed_solve(model.problem, X.PARAMS).solution if mixed else \
        cuda.solve(model.problem, X.PARAMS, precision=64)
    res = lopf.LopfResult(n, model, sol)
    gens, carriers = n.table("Generator"), n.table("Carrier")
    checked = 0
    for t in range(len(n.snapshots)):
        for g in gens.ids:
            p_nom = float(gens.value("p_nom", g))
            lo, hi = p_nom * gens.at("p_min_pu", g, t), p_nom * gens.at("p_max_pu", g, t)
            p = res.dispatch("Generator", g, t)
            carrier = str(gens.value("carrier", g))
            if float(carriers.value("co2_emissions", carrier)) == 0.0 and lo + 1e-2 < p < hi - 1e-2:
                checked += 1
                assert res.marginal_price(str(gens.value("bus", g)), t) == pytest.approx(
                    gens.at("marginal_cost", g, t), abs=1e-3)
    assert checked >= 2
    assert all(np.isfinite(res.marginal_price(b, t)) for b in n.table("Bus").ids for t in range(len(n.snapshots)))
