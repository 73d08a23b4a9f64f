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
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    names, factors, populated = lopf.lodf(n, carrier, buses, branches)
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


def test_a_transformer_is_referred_to_its_rating_and_tap():
    n = X.network("transformer-levels")
    tr = n.table("Transformer")
    assert lopf.impedance(n, "Transformer", "t1", "AC") == pytest.approx(0.1 / 500.0)
    tr.static["tap_ratio"] = {"t1": 1.05, "t2": -1.0}  # a non-positive tap reads as 1
    assert lopf.impedance(n, "Transformer", "t1", "AC") == pytest.approx(0.1 * 1.05 / 500.0)
    assert lopf.impedance(n, "Transformer", "t2", "AC") == pytest.approx(0.12 / 400.0)
    tr.static["s_nom"]["t2"] = 0.0
    with pytest.raises(lopf.UnsupportedNetwork, match="per-unit base"):
        lopf.build(n)


def test_the_phase_shift_leaves_the_optimised_flows_alone():
    """PyPSA's optimised flows on phase-shift equal transformer-levels'
    (LopfSuite.scala:1042-1090): the shift is not in the Kirchhoff rows."""
    a, b = lopf.build(X.network("phase-shift")), lopf.build(X.network("transformer-levels"))
    assert a.problem.constraint_matrix.nnz == b.problem.constraint_matrix.nnz
    assert np.array_equal(a.problem.constraint_matrix.values, b.problem.constraint_matrix.values)
    assert np.array_equal(a.problem.rhs, b.problem.rhs)


def _flows(network, carrier, buses, branches, injection):
    """DC power flow over the given branches: angles from B theta = P with the
    first bus as reference, flow = b (theta0 - theta1)."""
    index = {bus: i for i, bus in enumerate(buses[1:])}
    y = np.array([1.0 / lopf.impedance(network, c, i, carrier) for c, i in branches])
    A = np.zeros((len(branches), len(index)))
    for k, (c, i) in enumerate(branches):
        tab = network.table(c)
        for port, sign in (("bus0", 1.0), ("bus1", -1.0)):
            bus = str(tab.value(port, i))
            if bus in index:
                A[k, index[bus]] += sign
    theta = np.linalg.solve(A.T @ (y[:, None] * A), np.array([injection[bus] for bus in buses[1:]]))
    return y * (A @ theta)


def test_outage_factors_match_a_power_flow_without_the_branch():
    """f_l after losing o equals f_l + LODF[l, o] f_o before, over lines and
    transformers together: the meshed transformer-levels network with a
    second HV line added so that no branch is a bridge."""
    from noaidi_b200.network.pypsa_csv import Table
    n = X.network("transformer-levels")
    lines = n.table("Line")
    lines.ids.append("hv-b")
    for attr, v in (("bus0", "hv1"), ("bus1", "hv2"), ("x", 0.7), ("s_nom", 600.0)):
        lines.static.setdefault(attr, {})["hv-b"] = v
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    assert ("Transformer", "t1") in branches and len(branches) == 5
    names, factors, populated = lopf.lodf(n, carrier, buses, branches)
    rng = np.random.default_rng(3)
    injection = dict(zip(buses, rng.normal(size=len(buses))))
    injection[buses[0]] -= sum(injection.values())
    before = _flows(n, carrier, buses, branches, injection)
    for j, o in enumerate(branches):
        if not populated[j]:
            continue
        rest = [k for k in range(len(branches)) if k != j]
        after = _flows(n, carrier, buses, [branches[k] for k in rest], injection)
        expect = before[rest] + factors[rest, j] * before[j]
        assert np.allclose(after, expect, atol=1e-9)
    assert populated.sum() >= 2


def test_sclopf_monitors_transformers_and_refuses_extendable_branches():
    n = X.network("transformer-levels")
    lines = n.table("Line")
    lines.ids.append("hv-b")
    for attr, v in (("bus0", "hv1"), ("bus1", "hv2"), ("x", 0.7), ("s_nom", 600.0)):
        lines.static.setdefault(attr, {})["hv-b"] = v
    plain = lopf.build(n)
    secure = lopf.build_sclopf(n, [("Line", "hv"), ("Line", "hv-b")])
    assert secure.problem.num_constraints > plain.problem.num_constraints
    from oracle import oracle as O
    a, b = O.solve(plain.problem, X.PARAMS), O.solve(secure.problem, X.PARAMS)
    assert a.status.name == b.status.name == "OPTIMAL"
    assert b.objective_value >= a.objective_value - 1e-6 * abs(a.objective_value)
    with pytest.raises(lopf.UnsupportedNetwork, match="passive branch"):
        lopf.build_sclopf(n, [("Link", "hv")])
    with pytest.raises(lopf.UnsupportedNetwork, match="extendable"):
        lopf.build_sclopf(X.network("ac-dc-meshed"))


def test_scigrid_de_matches_pypsa_at_the_reference_tolerance():
    """The oracle reaches 1e-4 on scigrid-de in 14,848 iterations with a
    relative objective error of -1.05e-4 -- both the numbers the reference
    records for its own solver on this network."""
    from oracle import oracle as O
    res = X.check_scigrid(lambda p, params: O.solve(p, params))
    assert res.solution.iterations == 14_848
    target = X.expected("scigrid-de")["objective"]
    assert (res.objective - target) / target == pytest.approx(-1.05e-4, abs=0.01e-4)


def test_sclopf_expands_types_before_computing_outage_factors():
    """LopfSuite.scala:846-875: on standard-types the contingency rows need
    the typed impedances; a secure dispatch costs at least the plain one, up
    to the 1e-9 relative KKT tolerance both solves stop at."""
    from oracle import oracle as O
    n = X.network("standard-types")
    outages = [("Line", "hv12"), ("Line", "hv23"), ("Line", "hv31")]
    model, plain = lopf.build_sclopf(n, outages), lopf.build(n)
    assert model.problem.num_constraints > plain.problem.num_constraints
    a, b = O.solve(plain.problem, X.PARAMS), O.solve(model.problem, X.PARAMS)
    assert b.status.name == "OPTIMAL" and b.objective_value >= a.objective_value * (1 - 1e-8)


def _chp_network(efficiency2):
    """Gas into a combined heat and power link: electricity out at 0.4, heat
    at efficiency2; a heat dump takes what the heat load does not."""
    from noaidi_b200.network.pypsa_csv import Network, Table
    T = len(efficiency2)
    series = {} if T == 1 else {"efficiency2": np.array([[e, np.nan] for e in efficiency2])}
    tables = {
        "Bus": Table("Bus", ["gas", "elec", "heat"], {}),
        "Generator": Table("Generator", ["supply", "dump"], {
            "bus": {"supply": "gas", "dump": "heat"}, "p_nom": {"supply": 1000.0, "dump": 1000.0},
            "p_min_pu": {"supply": 0.0, "dump": -1.0}, "p_max_pu": {"supply": 1.0, "dump": 0.0},
            "marginal_cost": {"supply": 20.0, "dump": 0.0}}),
        "Link": Table("Link", ["chp", "boiler"], {
            "bus0": {"chp": "gas", "boiler": "gas"}, "bus1": {"chp": "elec", "boiler": "elec"},
            "bus2": {"chp": "heat", "boiler": ""}, "p_nom": {"chp": 1000.0, "boiler": 1000.0},
            "efficiency": {"chp": 0.4, "boiler": 0.3}, "efficiency2": {"chp": efficiency2[0], "boiler": np.nan},
            "marginal_cost": {"chp": 0.0, "boiler": 50.0}}, series),
        "Load": Table("Load", ["e", "h"], {"bus": {"e": "elec", "h": "heat"}, "p_set": {"e": 40.0, "h": 30.0}}),
    }
    return Network("chp", list(range(T)), {}, tables)


@pytest.mark.parametrize("efficiency2", [[0.5], [0.5, 0.6]])
def test_a_multi_port_link_delivers_at_every_port(efficiency2):
    """Topology.portsOf/portEfficiency: bus2 receives efficiency2 x p0 (a
    series over the static value); a link leaving bus2 empty has two ports."""
    from oracle import oracle as O
    n = _chp_network(efficiency2)
    model = lopf.build(n)
    res = lopf.LopfResult(n, model, O.solve(model.problem, X.PARAMS))
    assert res.status.name == "OPTIMAL"
    for t, e2 in enumerate(efficiency2):
        assert res.dispatch("Link", "chp", t) == pytest.approx(100.0, abs=1e-5)   # 40 MW of power at 0.4
        assert res.dispatch("Link", "boiler", t) == pytest.approx(0.0, abs=1e-5)
        assert res.dispatch("Generator", "dump", t) == pytest.approx(30.0 - 100.0 * e2, abs=1e-5)
    assert res.objective == pytest.approx(2000.0 * len(efficiency2), rel=1e-8)


def test_a_link_port_on_an_unknown_bus_is_refused():
    n = _chp_network([0.5])
    n.table("Link").static["bus2"]["chp"] = "steam"
    with pytest.raises(lopf.UnsupportedNetwork, match="steam"):
        lopf.build(n)


def test_prices_are_duals_that_close_the_gap():
    """LopfSuite.scala:620-655: the dual side is a real optimum (strong
    duality) and every nodal price is finite."""
    from oracle import oracle as O
    n = X.network("ac-dc-dispatch")
    model = lopf.build(n)
    res = lopf.LopfResult(n, model, O.solve(model.problem, X.PARAMS))
    sol = res.solution
    assert sol.objective_value == pytest.approx(sol.dual_objective_value, abs=1e-6 * max(1.0, abs(sol.objective_value)))
    for bus in n.table("Bus").ids:
        for t in range(len(n.snapshots)):
            assert np.isfinite(res.marginal_price(bus, t))


def test_an_interior_clean_generator_sets_its_bus_price():
    """LopfSuite.scala:713-747: a zero-emission generator strictly inside
    its limits is marginal, so its bus price equals its marginal cost."""
    from oracle import oracle as O
    n = X.network("ac-dc-dispatch")
    model = lopf.build(n)
    res = lopf.LopfResult(n, model, O.solve(model.problem, X.PARAMS))
    gens, carriers = n.table("Generator"), n.table("Carrier")
    checked = 0
    for t in range(len(n.snapshots)):
        for g in gens.ids:
            p_nom = float(gens.value("p_nom", g))
            lo, hi = p_nom * gens.at("p_min_pu", g, t), p_nom * gens.at("p_max_pu", g, t)
            p = res.dispatch("Generator", g, t)
            carrier = str(gens.value("carrier", g))
            clean = carrier in carriers.ids and float(carriers.value("co2_emissions", carrier)) == 0.0
            if clean and lo + 1e-2 < p < hi - 1e-2:
                checked += 1
                assert res.marginal_price(str(gens.value("bus", g)), t) == pytest.approx(
                    gens.at("marginal_cost", g, t), abs=1e-3), (t, g)
    assert checked >= 2


def test_storage_accessors_follow_pypsas_conventions():
    from oracle import oracle as O
    n = X.network("storage-cycle")
    exp = X.expected("storage-cycle")
    model = lopf.build(n)
    res = lopf.LopfResult(n, model, O.solve(model.problem, X.PARAMS))
    for u in n.table("StorageUnit").ids:
        for t in range(len(n.snapshots)):
            assert res.dispatch("StorageUnit", u, t) == pytest.approx(res.discharging(u, t) - res.charging(u, t))
            assert res.state_of_charge(u, t) == pytest.approx(
                X.frame_value(exp["storage_state_of_charge"], t, u), abs=1e-3)
            assert res.spill(u, t) == pytest.approx(X.frame_value(exp["storage_spill"], t, u), abs=1e-3)


@pytest.mark.parametrize("name", ["ac-dc-meshed", "storage-hvdc"])
def test_base_rows_stay_one_for_one_under_expansion(name):
    """SclopfSuite.scala:538-555: every equality block is emitted before the
    first inequality, so original row r is standard-form row r."""
    from noaidi_b200.prima.model import Direct, Negated
    model = lopf.build(X.network(name))
    t = model.translation
    for r in range(t.num_original_rows):
        e = t.expansion_of(r)
        assert isinstance(e, (Direct, Negated)) and e.row == r, (r, e)


def test_every_post_contingency_flow_stays_within_its_rating():
    """SclopfSuite.scala:128-157: each post-outage flow rebuilt from the
    solved flows and the factors respects the rating."""
    from oracle import oracle as O
    n = X.network("sclopf-triangle")
    outages = X.expected("sclopf-triangle")["sclopf"]["branch_outages"]
    model = lopf.build_sclopf(n, outages)
    res = lopf.LopfResult(n, model, O.solve(model.problem, X.PARAMS))
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    names, factors, _ = lopf.lodf(n, carrier, buses, branches)
    lines = n.table("Line")
    checked = 0
    for t in range(len(n.snapshots)):
        for j, (_, o) in enumerate(names):
            for k, (_, l) in enumerate(names):
                if k == j:
                    continue
                after = res.dispatch("Line", l, t) + factors[k, j] * res.dispatch("Line", o, t)
                assert abs(after) <= float(lines.value("s_nom", l)) + 1e-3, (t, o, l, after)
                checked += 1
    assert checked >= 12


def test_no_security_rows_cross_a_sub_network_boundary():
    """SclopfSuite.scala:240-272: two islands; outaging one triangle line adds
    rows for the other two triangle lines only."""
    from noaidi_b200.network.pypsa_csv import Network, Table
    lines = {"AB": ("A", "B"), "BC": ("B", "C"), "AC": ("A", "C"), "XY1": ("X", "Y"), "XY2": ("X", "Y")}
    n = Network("split", [0], {}, {
        "Bus": Table("Bus", list("ABCXY"), {"v_nom": dict.fromkeys("ABCXY", 380.0)}),
        "Line": Table("Line", list(lines), {"bus0": {k: v[0] for k, v in lines.items()},
                                            "bus1": {k: v[1] for k, v in lines.items()},
                                            "x": dict.fromkeys(lines, 0.1), "s_nom": dict.fromkeys(lines, 150.0)}),
        "Generator": Table("Generator", ["g1", "g2"], {"bus": {"g1": "A", "g2": "X"},
                                                       "p_nom": {"g1": 400.0, "g2": 400.0},
                                                       "marginal_cost": {"g1": 10.0, "g2": 10.0}}),
        "Load": Table("Load", ["l1", "l2"], {"bus": {"l1": "C", "l2": "Y"}, "p_set": {"l1": 100.0, "l2": 100.0}}),
    })
    assert len(lopf.sub_networks(n)) == 2
    base = lopf.build(n).problem.num_constraints
    one = lopf.build_sclopf(n, [("Line", "AB")])
    assert one.problem.num_constraints - base == 4  # two two-sided rows


def test_sclopf_under_an_emissions_cap_keeps_the_caps_sign():
    """SclopfSuite.scala:274-310: a network with a CO2 cap builds security
    rows, and the cap stays a negated (<=) row through the rebuild."""
    from noaidi_b200.prima.model import Negated
    n = X.network("ac-dc-co2")
    base = lopf.build(n)
    secure = lopf.build_sclopf(n, ["0", "1", "5"])
    assert secure.problem.num_constraints > base.problem.num_constraints
    count = lambda t, k: sum(isinstance(t.expansion_of(r), Negated) for r in range(k))
    k = base.translation.num_original_rows
    assert count(base.translation, k) > 0
    assert count(secure.translation, k) == count(base.translation, k)


def test_extendable_generation_alone_is_allowed_under_security():
    """SclopfSuite.scala:440-500: with the lines fixed, an expansion network
    builds security rows and the secure optimum costs at least the plain one."""
    from oracle import oracle as O
    n = X.network("ac-dc-meshed")
    lines = n.table("Line")
    lines.static["s_nom_extendable"] = dict.fromkeys(lines.ids, False)
    plain, secure = lopf.build(n), lopf.build_sclopf(n, ["0", "1", "5"])
    assert secure.problem.num_constraints > plain.problem.num_constraints
    params = X.PARAMS.copy(eps_abs=1e-7, eps_rel=1e-7)
    a, b = O.solve(plain.problem, params), O.solve(secure.problem, params)
    assert a.status.name == b.status.name == "OPTIMAL"
    assert b.objective_value >= a.objective_value - 1e-6 * abs(a.objective_value)


def test_a_state_of_charge_set_point_is_honoured_and_costs_something():
    """LopfSuite.scala:557-593: pinning one unit's state of charge at every
    snapshot holds it there, leaves the others free, and costs more."""
    from oracle import oracle as O
    free_net = X.network("storage-cycle")
    free_model = lopf.build(free_net)
    unconstrained = O.solve(free_model.problem, X.PARAMS).objective_value
    n = X.network("storage-cycle")
    units = n.table("StorageUnit")
    units.static["state_of_charge_set"] = {u: (90.0 if u == "battery" else float("nan")) for u in units.ids}
    model = lopf.build(n)
    res = lopf.LopfResult(n, model, O.solve(model.problem, X.PARAMS))
    assert res.status.name == "OPTIMAL"
    for t in range(len(n.snapshots)):
        assert res.state_of_charge("battery", t) == pytest.approx(90.0, abs=1e-4)
    others = [u for u in units.ids if u != "battery"]
    assert max(res.state_of_charge(u, t) for u in others for t in range(len(n.snapshots))) > 1.0
    assert res.objective > unconstrained + 1.0


def test_a_storage_power_set_point_is_refused():
    n = X.network("storage-cycle")
    units = n.table("StorageUnit")
    units.static["p_set"] = dict.fromkeys(units.ids, 10.0)
    with pytest.raises(lopf.UnsupportedNetwork, match="p_set"):
        lopf.build(n)


def test_a_discharge_only_extendable_unit_has_no_nan_bound():
    """LopfSuite.scala:876-895: p_min_pu = 0 on an extendable unit gives the
    charging column [0, inf), not an inf x 0 NaN."""
    n = X.network("storage-hvdc")
    units = n.table("StorageUnit")
    units.static["p_min_pu"] = dict.fromkeys(units.ids, 0.0)
    model = lopf.build(n)
    for u in units.ids:
        for t in range(len(n.snapshots)):
            j = model.columns[("StorageUnit-p_store", u, t)]
            assert not np.isnan(model.problem.variable_upper[j])


def test_the_co2_cap_is_respected_and_reached():
    """LopfSuite.scala:677-712: emissions, summed with the generators
    weighting (named here independently of the builder), stay under the cap
    and reach it -- an absent or mis-signed row exceeds it, an over-tight one
    stays well below."""
    from oracle import oracle as O
    n = X.network("ac-dc-co2")
    model = lopf.build(n)
    res = lopf.LopfResult(n, model, O.solve(model.problem, X.PARAMS))
    gens, carriers = n.table("Generator"), n.table("Carrier")
    emitted = 0.0
    for t in range(len(n.snapshots)):
        for g in gens.ids:
            intensity = float(carriers.value("co2_emissions", str(gens.value("carrier", g))))
            emitted += res.dispatch("Generator", g, t) * intensity / gens.at("efficiency", g, t) * \
                n.weighting("generators", t)
    cap = float(n.table("GlobalConstraint").value("constant", "co2_limit"))
    assert emitted <= cap + 1e-6 * max(1.0, cap)
    assert emitted >= cap - 1e-3 * max(1.0, cap)


def test_a_nan_capacity_floor_is_refused():
    """LopfSuite.scala:434-450: a NaN p_nom_min is not a capacity."""
    n = X.network("ac-dc-meshed")
    gens = n.table("Generator")
    g = next(i for i in gens.ids if lopf.extendable(gens, i))
    gens.static.setdefault("p_nom_min", {})[g] = float("nan")
    with pytest.raises(lopf.UnsupportedNetwork, match="p_nom_min"):
        lopf.build(n)


def _series(tab, attr, values_by_id, T):
    arr = np.array([[values_by_id.get(i, float(tab.value(attr, i))) for i in tab.ids] for _ in range(T)])
    tab.series[attr] = arr


def test_standing_losses_are_checked_where_the_balance_reads_them():
    """LopfSuite.scala:917-1040: a bad loss given only per snapshot is
    refused; a bad static loss that a series fully overrides is not; a
    series on one unit does not excuse a bad static value on another."""
    T = len(X.network("storage-cycle").snapshots)
    n = X.network("storage-cycle")
    _series(n.table("StorageUnit"), "standing_loss", {"battery": 1.5}, T)
    with pytest.raises(lopf.UnsupportedNetwork, match="standing_loss"):
        lopf.build(n)
    n = X.network("storage-cycle")
    units = n.table("StorageUnit")
    units.static["standing_loss"] = {u: (1.5 if u == "battery" else 0.0) for u in units.ids}
    _series(units, "standing_loss", {"battery": 0.01}, T)
    lopf.build(n)  # the series is what the balance reads
    n = X.network("storage-cycle")
    units = n.table("StorageUnit")
    other = next(u for u in units.ids if u != "battery")
    units.static["standing_loss"] = {u: (1.5 if u == other else 0.0) for u in units.ids}
    units.series["standing_loss"] = np.array([[0.01 if u == "battery" else 1.5 for u in units.ids]
                                              for _ in range(T)])
    with pytest.raises(lopf.UnsupportedNetwork, match=other):
        lopf.build(n)


def test_an_extendable_stores_energy_is_free_at_both_ends():
    """LopfSuite.scala:934-967: e_min_pu may be negative, so an extendable
    store's energy column carries both ends in rows, not a zero bound."""
    n = X.network("store-bank")
    model = lopf.build(n)
    st = n.table("Store")
    ext = [i for i in st.ids if lopf.extendable(st, i)]
    assert ext
    for s_ in ext:
        for t in range(len(n.snapshots)):
            j = model.columns[("Store-e", s_, t)]
            assert model.problem.variable_lower[j] == -np.inf and model.problem.variable_upper[j] == np.inf


def test_the_storage_fixtures_flags_are_load_bearing():
    """LopfSuite.scala:488-517: PyPSA's storage-cycle answer uses every
    feature the fixture sets -- a cyclic unit ends holding energy, a unit
    spills, and the standing loss is non-zero where set."""
    exp = X.expected("storage-cycle")
    n = X.network("storage-cycle")
    units = n.table("StorageUnit")
    T = len(n.snapshots)
    spilled = sum(X.frame_value(exp["storage_spill"], t, u) for t in range(T) for u in units.ids)
    assert spilled > 1.0
    cyclic = [u for u in units.ids if bool(units.value("cyclic_state_of_charge", u)) is True]
    assert cyclic and max(X.frame_value(exp["storage_state_of_charge"], T - 1, u) for u in cyclic) > 1.0
    assert any(float(units.value("standing_loss", u)) > 0.0 for u in units.ids)


def _cycles_network(tmp_path, buses, lines, carrier="AC", v_nom=1.0, x=1.0, r=0.0):
    from noaidi_b200.network.pypsa_csv import read
    d = tmp_path / "net"
    d.mkdir(exist_ok=True)
    (d / "buses.csv").write_text("name,v_nom,carrier\n" + "".join(f"{b},{v_nom},{carrier}\n" for b in buses))
    (d / "lines.csv").write_text("name,bus0,bus1,x,r,s_nom\n" +
                                 "".join(f"{i},{a},{b},{x},{r},100.0\n" for i, a, b in lines))
    (d / "snapshots.csv").write_text(",snapshot\n0,2015-01-01 00:00:00\n")
    return read(str(d), "cycles")


def _signs(cycle):
    return {e: o for _, e, o in cycle.terms}


def test_a_triangle_gives_one_consistently_traversed_cycle(tmp_path):
    """CyclesSuite.scala:54-71: head-to-tail lines, one cycle, one sign."""
    cycles = lopf.cycle_basis(_cycles_network(tmp_path, "LMN", [("a", "L", "M"), ("b", "M", "N"), ("c", "N", "L")]))
    assert len(cycles) == 1
    s = _signs(cycles[0])
    assert set(s) == {"a", "b", "c"} and len(set(s.values())) == 1 and abs(s["a"]) == 1.0


def test_a_parallel_pair_gives_opposing_branches(tmp_path):
    cycles = lopf.cycle_basis(_cycles_network(tmp_path, "AB", [("a", "A", "B"), ("b", "A", "B")]))
    assert len(cycles) == 1
    s = _signs(cycles[0])
    assert set(s) == {"a", "b"} and s["a"] == -s["b"]


def test_a_tree_has_no_cycles(tmp_path):
    assert lopf.cycle_basis(_cycles_network(tmp_path, "ABCD", [("a", "A", "B"), ("b", "B", "C"), ("c", "B", "D")])) == []


def test_two_independent_loops_give_one_cycle_per_component(tmp_path):
    lines = [("a", "A", "B"), ("b", "B", "C"), ("c", "C", "A"), ("x", "X", "Y"), ("y", "Y", "Z"), ("z", "Z", "X")]
    cycles = lopf.cycle_basis(_cycles_network(tmp_path, "ABCXYZ", lines))
    assert len(cycles) == 2
    assert {e for c in cycles for e in _signs(c)} == {"a", "b", "c", "x", "y", "z"}


def test_a_square_with_a_chord_gives_two_closed_triangles(tmp_path):
    """CyclesSuite.scala:110-128: each basis cycle is a triangle and a closed
    walk -- every bus it touches entered and left once."""
    lines = [("a", "A", "B"), ("b", "B", "C"), ("c", "C", "D"), ("d", "D", "A"), ("e", "A", "C")]
    ends = {i: (p, q) for i, p, q in lines}
    cycles = lopf.cycle_basis(_cycles_network(tmp_path, "ABCD", lines))
    assert len(cycles) == 2
    for c in cycles:
        s = _signs(c)
        assert len(s) == 3 and all(abs(o) == 1.0 for o in s.values())
        net = {}
        for e, o in s.items():  # o x (out of bus0, into bus1) must cancel at every bus
            p, q = ends[e]
            net[p] = net.get(p, 0.0) - o
            net[q] = net.get(q, 0.0) + o
        assert all(v == 0.0 for v in net.values()), net


def test_cycles_over_a_dc_island_use_resistance(tmp_path):
    """CyclesSuite.scala:130-: with x = 0 and r = 0.5 over v_nom 2, the
    Kirchhoff coefficients are +-0.5 / 4, not zero."""
    n = _cycles_network(tmp_path, "ABC", [("a", "A", "B"), ("b", "B", "C"), ("c", "C", "A")], carrier="DC",
                        v_nom=2.0, x=0.0, r=0.5)
    [cycle] = lopf.cycle_basis(n)
    for _, e, _ in cycle.terms:
        assert lopf.impedance(n, "Line", e, cycle.carrier) == pytest.approx(0.5 / 4.0)


def _triangle_with_spur():
    n = X.network("sclopf-triangle")
    lines = n.table("Line")
    lines.ids.append("CD")
    for attr, v in (("bus0", "C"), ("bus1", "D"), ("x", 0.1), ("s_nom", 150.0)):
        lines.static.setdefault(attr, {})["CD"] = v
    n.table("Bus").ids.append("D")
    n.table("Bus").static.setdefault("v_nom", {})["D"] = 380.0
    return n


def test_an_unrequested_bridge_column_is_marked_not_computed():
    """SclopfSuite.scala:368-393: with only AB requested, AB's and BC's
    columns are computed and the bridge CD's is not -- marked so rather than
    read as a zero meaning no effect."""
    n = _triangle_with_spur()
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    names, factors, populated = lopf.lodf(n, carrier, buses, branches, {("Line", "AB")})
    at = {key: k for k, key in enumerate(names)}
    assert populated[at[("Line", "AB")]] and abs(factors[at[("Line", "BC")], at[("Line", "AB")]]) > 0.0
    assert populated[at[("Line", "BC")]] and abs(factors[at[("Line", "AB")], at[("Line", "BC")]]) > 0.0
    assert not populated[at[("Line", "CD")]]


def test_a_bridge_elsewhere_does_not_block_a_well_posed_contingency():
    """SclopfSuite.scala:224-238: naming the spur is refused, an outage on
    the triangle still builds its security rows."""
    n = _triangle_with_spur()
    with pytest.raises(lopf.UnsupportedNetwork, match="bridge"):
        lopf.build_sclopf(n, [("Line", "CD")])
    model = lopf.build_sclopf(n, [("Line", "AB")])
    assert model.problem.num_constraints > lopf.build(n).problem.num_constraints


def test_an_outage_naming_no_passive_branch_is_refused():
    """SclopfSuite.scala:193-200."""
    with pytest.raises(lopf.UnsupportedNetwork, match="nonexistent"):
        lopf.build_sclopf(X.network("sclopf-triangle"), [("Line", "nonexistent")])


def test_the_default_outage_set_is_every_passive_branch_and_security_costs_more():
    """SclopfSuite.scala:81-98, :202-210: with no list every passive branch
    is a contingency, which on the triangle is PyPSA's list, 14,100 against
    the plain dispatch's 6,900."""
    from oracle import oracle as O
    n = X.network("sclopf-triangle")
    exp = X.expected("sclopf-triangle")
    assert sorted(exp["sclopf"]["branch_outages"]) == sorted(n.table("Line").ids)
    secure = O.solve(lopf.build_sclopf(n).problem, X.PARAMS)
    plain = O.solve(lopf.build(n).problem, X.PARAMS)
    assert secure.objective_value == pytest.approx(14100.0, abs=1e-3)
    assert plain.objective_value == pytest.approx(exp["objective"], abs=1e-3)
    assert secure.objective_value > plain.objective_value + 1.0


@pytest.mark.parametrize("ratio", [1e2, 1e4, 1e6])
def test_factors_stay_bounded_near_a_bridge(tmp_path, ratio):
    """SclopfSuite.scala:395-424: a stiff branch beside a path ratio times
    weaker -- losing either moves all its flow, so every factor is at most
    one in magnitude, however close the network is to a bridge."""
    n = _cycles_network(tmp_path, "ABC", [("AB", "A", "B"), ("AC", "A", "C"), ("CB", "C", "B")], v_nom=380.0)
    lines = n.table("Line")
    lines.static["x"] = {"AB": 0.1, "AC": 0.1 * ratio, "CB": 0.1 * ratio}
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    _, factors, populated = lopf.lodf(n, carrier, buses, branches)
    off = [abs(factors[i, j]) for i in range(3) for j in range(3) if i != j and populated[j]]
    assert max(off) == pytest.approx(1.0, abs=1e-6)


def test_an_extendable_transformer_is_refused_under_security():
    n = X.network("transformer-levels")
    tr = n.table("Transformer")
    tr.static["s_nom_extendable"] = dict.fromkeys(tr.ids, True)
    with pytest.raises(lopf.UnsupportedNetwork, match="Transformer"):
        lopf.build_sclopf(n, [("Line", "hv")])


def test_an_empty_outage_list_is_the_dispatch_model_even_when_extendable():
    n = X.network("ac-dc-meshed")
    assert lopf.build_sclopf(n, []).problem.num_constraints == lopf.build(n).problem.num_constraints


BODF_NETWORKS = [n for n in X.NETWORKS if "bodf" in X.expected(n)]


def _our_factors(n):
    """Every populated (affected, outage) factor over all sub-networks, with
    no contingency requested so that a bridge is left unpopulated."""
    from noaidi_b200.network import standard_types
    n = standard_types.expand(n)
    out, bridges = {}, set()
    for carrier, buses, branches in lopf.sub_networks(n):
        keys, f, populated = lopf.lodf(n, carrier, buses, branches, set())
        for j, o in enumerate(keys):
            if not populated[j]:
                bridges.add(o)
                continue
            for i, a in enumerate(keys):
                out[(a, o)] = f[i, j]
    return out, bridges


@pytest.mark.parametrize("name", BODF_NETWORKS)
def test_outage_factors_match_pypsa_bodf(name):
    """LodfSuite.scala:32-65, over every golden network PyPSA computed a
    BODF for: the same branches per sub-network and every factor within
    1e-9; the only columns left out are bridges, whose PyPSA column is the
    -1 diagonal of a one-branch island."""
    ours, bridges = _our_factors(X.network(name))
    ours_branches = {a for a, _ in ours} | bridges
    compared = 0
    for block in X.expected(name)["bodf"].values():
        keys = [tuple(b) for b in block["branches"]]
        assert set(keys) <= ours_branches
        for i, a in enumerate(keys):
            for j, o in enumerate(keys):
                if o in bridges:
                    assert len(keys) == 1 and block["bodf"][i][j] == pytest.approx(-1.0)
                    continue
                assert ours[(a, o)] == pytest.approx(block["bodf"][i][j], abs=1e-9), (a, o)
                compared += 1
    assert compared == len(ours)


def test_the_meshed_fixture_can_tell_a_stub_from_the_factors():
    """LodfSuite.scala:54-64: at least six off-diagonal factors of lodf-mesh
    differ from +-1, which a stub returning +-1 would get wrong."""
    block = next(iter(X.expected("lodf-mesh")["bodf"].values()))
    m = len(block["branches"])
    assert sum(1 for i in range(m) for j in range(m)
               if i != j and abs(abs(block["bodf"][i][j]) - 1.0) > 1e-6) >= 6


def test_a_single_cycle_gives_factors_of_magnitude_one():
    """LodfSuite.scala:67-79: one cycle has one alternative path, so every
    factor is +-1 whatever the impedances."""
    ours, _ = _our_factors(X.network("sclopf-triangle"))
    for a, o in (("AB", "BC"), ("AB", "AC"), ("BC", "AC")):
        assert abs(ours[(("Line", a), ("Line", o))]) == pytest.approx(1.0, abs=1e-9)


@pytest.mark.parametrize("x", [0.0, -0.1, float("nan")])
def test_a_branch_without_susceptance_is_refused_by_the_outage_factors(x):
    """Branches.susceptance (Branches.scala:74-79): the factors refuse a
    reactance that is not positive, where the Kirchhoff rows would carry it."""
    n = X.network("lodf-mesh")
    n.table("Line").static["x"]["AB"] = x
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    with pytest.raises(lopf.UnsupportedNetwork, match="no susceptance"):
        lopf.lodf(n, carrier, buses, branches, set())


def test_a_line_at_a_bus_without_voltage_is_refused_by_the_outage_factors():
    n = X.network("lodf-mesh")
    bus0 = str(n.table("Line").value("bus0", "AB"))
    n.table("Bus").static.setdefault("v_nom", {})[bus0] = 0.0
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    with pytest.raises(lopf.UnsupportedNetwork, match="v_nom"):
        lopf.lodf(n, carrier, buses, branches, set())


def test_a_non_finite_factor_is_refused_for_a_requested_outage():
    """Lodf.scala:224-229: a reactance so small its susceptance overflows
    gives non-finite factors; a requested contingency refuses them."""
    n = X.network("lodf-mesh")
    n.table("Line").static["x"]["AB"] = 1e-310
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    with np.errstate(all="ignore"), pytest.raises(lopf.UnsupportedNetwork, match="non-finite"):
        lopf.lodf(n, carrier, buses, branches, {("Line", "AB")})


def test_solve_sclopf_builds_the_secure_model_and_solves_it(monkeypatch):
    """Sclopf.solve (Sclopf.scala:66-74): the device call is replaced by the
    oracle here, so this checks which LP reaches it and what comes back."""
    from noaidi_b200.prima import cuda
    from oracle import oracle as O
    seen = []

    def fake_solve(problem, params, **kw):
        seen.append(problem)
        return O.solve(problem, params)
    monkeypatch.setattr(cuda, "solve", fake_solve)
    n = X.network("sclopf-triangle")
    res = lopf.solve_sclopf(n, params=X.PARAMS)
    assert res.objective == pytest.approx(14100.0, abs=1e-3)
    assert seen[0].num_constraints == lopf.build_sclopf(n).problem.num_constraints
    plain = lopf.solve_sclopf(n, [], params=X.PARAMS)
    assert plain.objective == pytest.approx(6900.0, abs=1e-3)


def test_a_factor_is_read_by_branch_and_refuses_what_was_not_computed():
    """Lodf.factor / factorOrZero (Lodf.scala:40-66): an unknown branch and an
    uncomputed column are errors; only another sub-network is a zero."""
    n = _triangle_with_spur()
    [(carrier, buses, branches)] = lopf.sub_networks(n)
    f = lopf.lodf(n, carrier, buses, branches, {("Line", "AB")})
    assert ("Line", "AB") in f and ("Line", "XY") not in f
    assert abs(f.factor(("Line", "BC"), ("Line", "AB"))) == pytest.approx(1.0, abs=1e-9)
    assert f.factor(("Line", "AB"), ("Line", "AB")) == -1.0
    with pytest.raises(KeyError, match="not computed"):
        f.factor(("Line", "AB"), ("Line", "CD"))
    with pytest.raises(KeyError, match="not computed"):
        f.factor_or_zero(("Line", "AB"), ("Line", "CD"))
    with pytest.raises(KeyError, match="no branch"):
        f.factor(("Line", "AB"), ("Line", "typo"))
    assert f.factor_or_zero(("Line", "AB"), ("Line", "elsewhere")) == 0.0
