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
    n.tables["ShuntImpedance"] = Table("ShuntImpedance", ["shunt"], {"bus": {"shunt": "London"}})
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


def _with_generator_attr(attr, value):
    n = X.network("ac-dc-meshed")
    gens = n.table("Generator")
    gens.static[attr] = {g: value for g in gens.ids}
    return n


@pytest.mark.parametrize("attr,value,word", [
    ("overnight_cost", 1000.0, "overnight_cost"),  # annuitised cost is not a per-unit one (LopfSuite.scala:222-238)
    ("p_nom_mod", 100.0, "p_nom_mod"),             # modular capacity is mixed-integer (:240-255)
    ("p_nom_min", -5.0, "p_nom_min"),              # a negative capacity floor
])
def test_expansion_attributes_the_lp_cannot_honour_are_refused(attr, value, word):
    with pytest.raises(lopf.UnsupportedNetwork, match=word):
        lopf.build(_with_generator_attr(attr, value))


def test_expansion_bounds_that_cross_are_refused():
    n = X.network("ac-dc-meshed")
    gens = n.table("Generator")
    g = next(i for i in gens.ids if lopf.extendable(gens, i))
    gens.static.setdefault("p_nom_min", {})[g] = 10.0
    gens.static.setdefault("p_nom_max", {})[g] = 5.0
    with pytest.raises(lopf.UnsupportedNetwork, match="above"):
        lopf.build(n)


def test_a_non_extendable_network_builds_no_capacity_columns():
    model = lopf.build(X.network("ac-dc-dispatch"))
    assert not [k for k in model.columns if k[2] == -1]
    assert model.objective_constant == 0.0


def test_capacity_columns_come_first_and_carry_capital_cost():
    n = X.network("ac-dc-meshed")
    model = lopf.build(n)
    caps = sorted((col, k) for k, col in model.columns.items() if k[2] == -1)
    assert [c for c, _ in caps] == list(range(len(caps)))  # declared before every snapshot column
    for col, (component, entity, _) in caps:
        tab = n.table(component.split("-")[0])
        assert model.problem.objective[col] == pytest.approx(lopf.periodized_cost(tab, entity))


def test_a_store_has_no_power_rating():
    """PyPSA bounds no Store-p: a store's rate follows from its energy band
    and the elapsed hours alone (LopfSuite.scala:392-414)."""
    n = X.network("store-bank")
    model = lopf.build(n)
    for st in n.table("Store").ids:
        for t in range(len(n.snapshots)):
            j = model.columns[("Store-p", st, t)]
            assert model.problem.variable_lower[j] == -np.inf and model.problem.variable_upper[j] == np.inf


def test_the_store_fixture_exercises_its_features():
    """The cyclic wrap, both ends of the energy band and the capacity ceiling
    are all binding in PyPSA's answer (LopfSuite.scala:366-390)."""
    exp = X.expected("store-bank")
    last = len(X.network("store-bank").snapshots) - 1
    assert X.frame_value(exp["store_e"], last, "swing") > 1.0
    assert X.frame_value(exp["store_p"], 0, "swing") > 1.0
    levels = [X.frame_value(exp["store_e"], t, "tank") for t in range(last + 1)]
    assert min(levels) == pytest.approx(20.0, abs=1e-3) and max(levels) == pytest.approx(100.0, abs=1e-3)
    assert exp["nominal_opt"]["Store"]["grow"] == pytest.approx(60.0, abs=1e-3)


@pytest.mark.parametrize("attr,value", [("e_set", 50.0), ("p_set", 1.0), ("marginal_cost_quadratic", 0.5),
                                        ("standing_loss", 1.5), ("e_cyclic_per_period", True)])
def test_store_features_not_built_are_refused(attr, value):
    n = X.network("store-bank")
    st = n.table("Store")
    st.static[attr] = {i: value for i in st.ids}
    with pytest.raises(lopf.UnsupportedNetwork):
        lopf.build(n)
