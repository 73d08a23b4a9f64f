"""The dispatch LOPF builder and the PyPSA CSV reader on CPU: the LP solved
by the oracle must reproduce PyPSA's ac-dc-dispatch optimum."""
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
    n.tables["StorageUnit"] = Table("StorageUnit", ["battery"], {"bus": {"battery": "London"}})
    with pytest.raises(lopf.UnsupportedNetwork):
        lopf.build(n)
