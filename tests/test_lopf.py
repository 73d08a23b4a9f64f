"""The dispatch LOPF builder and the PyPSA CSV reader on CPU: the LP solved
by the oracle must reproduce PyPSA's ac-dc-dispatch optimum."""
import numpy as np
import pytest

from noaidi_b200.network import lopf
from tests import lopf_cases as X


@pytest.mark.parametrize("name", X.NETWORKS)
def test_lopf_matches_pypsa_with_the_oracle(name):
    from oracle import oracle as O
    X.check_against_pypsa(lambda p: O.solve(p, X.PARAMS), name)


def test_cycle_basis_has_the_circuit_rank():
    cycles = X.check_cycle_rank()
    assert {c.carrier for c in cycles} <= {"AC", "DC"}


def test_unmodelled_components_are_refused():
    from noaidi_b200.network.pypsa_csv import Table
    n = X.network()
    n.tables["Store"] = Table("Store", ["tank"], {"bus": {"tank": "London"}})
    with pytest.raises(lopf.UnsupportedNetwork):
        lopf.build(n)


def test_sclopf_matches_pypsa_with_the_oracle():
    from oracle import oracle as O
    X.check_sclopf_triangle(lambda p: O.solve(p, X.PARAMS))


def test_lodf_of_a_triangle():
    """Equal reactances: losing one side puts its whole flow on the other two,
    each seeing +-1 times it (a two-line path in series)."""
    n = X.network("sclopf-triangle")
    [(carrier, buses, lines)] = lopf.sub_networks(n)
    names, factors, populated = lopf.lodf(n, carrier, buses, lines)
    assert populated.all() and np.allclose(np.diag(factors), -1.0)
    assert np.allclose(np.abs(factors[~np.eye(3, dtype=bool)]), 1.0)


def test_a_bridge_is_not_a_credible_contingency():
    from noaidi_b200.network.pypsa_csv import Table
    n = X.network("sclopf-triangle")
    lines = n.table("Line")
    lines.ids.append("spur")
    for attr, v in (("bus0", "C"), ("bus1", "D"), ("x", 0.1), ("s_nom", 150.0)):
        lines.static.setdefault(attr, {})["spur"] = v
    bus = n.table("Bus")
    bus.ids.append("D")
    bus.static.setdefault("v_nom", {})["D"] = 380.0
    with pytest.raises(lopf.UnsupportedNetwork):
        lopf.build_sclopf(n, ["spur"])
