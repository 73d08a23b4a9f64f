"""Sub-network decomposition and bus references (``Topology``,
modules/network-model/src/main/scala/org/noaidi/network/Topology.scala), with
the cases of TopologySuite.scala (all but the schema-role one, which concerns
the reference's component registry).  Networks written here go through the
CSV reader, where column typing happens."""
import pytest

from noaidi_b200.network import lopf
from noaidi_b200.network.pypsa_csv import MalformedNetwork, read
from tests import lopf_cases as X


def _via_reader(tmp_path, files):
    files = {"snapshots.csv": ",snapshot\n0,2015-01-01 00:00:00\n", **files}
    for name, body in files.items():
        (tmp_path / name).write_text(body)
    return read(str(tmp_path), "fixture")


def _chain(tmp_path, order, carriers=None):
    """Buses in the given file order, lines joining them in sorted order."""
    carriers = carriers or {}
    buses = "name,v_nom,carrier\n" + "".join(f"{b},380.0,{carriers.get(b, 'AC')}\n" for b in order)
    ids = sorted(order)
    lines = "name,bus0,bus1,x,s_nom\n" + "".join(f"l{k},{a},{b},0.1,100\n" for k, (a, b) in enumerate(zip(ids, ids[1:])))
    return _via_reader(tmp_path, {"buses.csv": buses, "lines.csv": lines})


def test_links_do_not_merge_sub_networks():
    """TopologySuite.scala:83-95: the AC/DC network is joined by links only."""
    n = X.network("ac-dc-meshed")
    assert len(n.table("Link")) > 0
    subs = lopf.sub_networks(n)
    assert len(subs) == 4
    assert {s.carrier for s in subs} == {"AC", "DC"}


def test_a_series_chain_forms_one_island_with_its_buses_sorted(tmp_path):
    """TopologySuite.scala:122-135, with the buses written out of order."""
    [island] = lopf.sub_networks(_chain(tmp_path, ["c", "a", "e", "b", "d"]))
    assert island.buses == ["a", "b", "c", "d", "e"]
    assert island.branches == [("Line", f"l{k}") for k in range(4)]
    assert not island.mixed_carriers


def test_the_ac_side_splits_into_three_islands_one_a_singleton():
    """TopologySuite.scala:137-142."""
    ac = [s for s in lopf.sub_networks(X.network("ac-dc-meshed")) if s.carrier == "AC"]
    assert len(ac) == 3 and any(len(s.buses) == 1 for s in ac)


def test_islands_come_in_order_of_their_first_bus():
    subs = lopf.sub_networks(X.network("ac-dc-meshed"))
    firsts = [s.buses[0] for s in subs]
    assert firsts == sorted(firsts)


def test_a_multi_port_link_with_numeric_bus_names_reads_correctly(tmp_path):
    """TopologySuite.scala:197-215: bus2 holds names that parse as numbers."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\n0,380.0,AC\n1,380.0,AC\n2,380.0,AC\n",
                               "links.csv": "name,bus0,bus1,bus2\nk,0,1,2\n"})
    links = n.table("Link")
    assert lopf.link_ports(links) == ["bus0", "bus1", "bus2"]
    assert links.endpoint("bus2", "k") == "2"
    assert lopf.dangling_references(n) == []


def test_a_blank_endpoint_is_dangling_not_an_absent_edge(tmp_path):
    """TopologySuite.scala:217-231."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\n",
                               "lines.csv": "name,bus0,bus1\nl0,a,\n"})
    [(component, entity, port, bus)] = lopf.dangling_references(n)
    assert (component, entity, port, bus) == ("Line", "l0", "bus1", "")
    with pytest.raises(MalformedNetwork):
        lopf.sub_networks(n)


def test_a_blank_endpoint_does_not_match_a_bus_named_nan(tmp_path):
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nnan,380.0,AC\n",
                               "lines.csv": "name,bus0,bus1\nl0,a,\n"})
    with pytest.raises(MalformedNetwork, match="bus1"):
        lopf.sub_networks(n)


def test_a_branch_table_missing_an_endpoint_column_is_rejected(tmp_path):
    """TopologySuite.scala:233-244."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\n",
                               "lines.csv": "name,bus0\nl0,a\n"})
    with pytest.raises(MalformedNetwork, match="bus1"):
        lopf.sub_networks(n)


def test_a_stale_link_reference_does_not_block_decomposition(tmp_path):
    """TopologySuite.scala:246-260: reported by the full check, but the
    passive-only decomposition still works."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\n",
                               "lines.csv": "name,bus0,bus1\nl0,a,b\n",
                               "links.csv": "name,bus0,bus1\nk,a,gone\n"})
    assert any(bus == "gone" for _, _, _, bus in lopf.dangling_references(n))
    assert [s.buses for s in lopf.sub_networks(n)] == [["a", "b"]]


def test_the_carrier_label_agrees_with_the_sorted_bus_list(tmp_path):
    """TopologySuite.scala:262-276: file order b, a; sorted order a, b."""
    [island] = lopf.sub_networks(_chain(tmp_path, ["b", "a"], {"b": "DC", "a": "AC"}))
    assert island.buses == ["a", "b"]
    assert island.carrier == "AC" and island.mixed_carriers


def test_a_mixed_island_takes_its_kirchhoff_impedance_from_the_label(tmp_path):
    """Cycles.scala:43-53: the cycle's carrier, which picks x or r, is the
    island's label rather than that of the bus the walk starts from."""
    buses = "name,v_nom,carrier\nb,380.0,DC\na,380.0,AC\nc,380.0,AC\n"
    lines = "name,bus0,bus1,x,r,s_nom\nab,a,b,0.1,0.2,100\nbc,b,c,0.1,0.2,100\nca,c,a,0.1,0.2,100\n"
    n = _via_reader(tmp_path, {"buses.csv": buses, "lines.csv": lines})
    [cycle] = lopf.cycle_basis(n)
    assert cycle.carrier == "AC"


def test_an_unused_extra_port_is_not_a_dangling_reference(tmp_path):
    """TopologySuite.scala:278-295: a two-port link in a table with a bus2
    column leaves it blank."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\nc,380.0,AC\n",
                               "links.csv": "name,bus0,bus1,bus2\nthree,a,b,c\ntwo,a,b,\n"})
    assert lopf.dangling_references(n) == []


def test_a_links_table_missing_bus1_does_not_block_decomposition(tmp_path):
    """TopologySuite.scala:297-309; the dispatch builder still refuses it."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\n",
                               "lines.csv": "name,bus0,bus1\nl0,a,b\n",
                               "links.csv": "name,bus0\nk,a\n"})
    assert [s.buses for s in lopf.sub_networks(n)] == [["a", "b"]]
    with pytest.raises(MalformedNetwork, match="bus1"):
        lopf.dangling_bus_references(n)


@pytest.mark.parametrize("name", X.NETWORKS)
def test_every_bus_belongs_to_exactly_one_sub_network(name):
    """TopologySuite.scala:311-320."""
    n = X.network(name)
    seen = [b for s in lopf.sub_networks(n) for b in s.buses]
    assert len(seen) == len(set(seen)) and set(seen) == set(n.table("Bus").ids)


def test_a_branch_referencing_an_unknown_bus_is_rejected(tmp_path):
    """TopologySuite.scala:375-382."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\n",
                               "lines.csv": "name,bus0,bus1\nl0,a,typo\n"})
    with pytest.raises(MalformedNetwork, match="typo"):
        lopf.sub_networks(n)


def test_no_golden_island_is_mixed():
    """TopologySuite.scala:384-400, the well-formed half."""
    for name in X.NETWORKS:
        assert not any(s.mixed_carriers for s in lopf.sub_networks(X.network(name))), name


def test_an_empty_network_has_no_sub_networks(tmp_path):
    """TopologySuite.scala:402-405."""
    assert lopf.sub_networks(_via_reader(tmp_path, {})) == []


@pytest.mark.parametrize("table,row", [
    ("loads.csv", "d1,gone,10"),
    ("generators.csv", "g1,gone,10,1"),
    ("links.csv", "k1,a,gone,10"),
    ("lines.csv", "l1,a,,0.1,10"),
])
def test_the_dispatch_model_refuses_a_reference_to_no_bus(tmp_path, table, row):
    """Lopf.rejectDanglingBuses (Lopf.scala:593-606): a stale load would
    vanish from the balance and a stale branch end become a free source."""
    files = {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\n",
             "lines.csv": "name,bus0,bus1,x,s_nom\nl0,a,b,0.1,100\n",
             "links.csv": "name,bus0,bus1,p_nom\nk0,a,b,10\n",
             "generators.csv": "name,bus,p_nom,marginal_cost\ng0,a,100,1\n",
             "loads.csv": "name,bus,p_set\nd0,b,10\n"}
    (tmp_path / "ok").mkdir()
    lopf.build(_via_reader(tmp_path / "ok", files))  # the network as written builds
    files[table] += row + "\n"
    (tmp_path / "bad").mkdir()
    with pytest.raises(lopf.UnsupportedNetwork, match="unknown bus"):
        lopf.build(_via_reader(tmp_path / "bad", files))


def test_a_multi_port_branch_connects_all_of_its_ports(tmp_path):
    """TopologySuite.scala:144-195: every pair, so connectivity over the link
    is transitive, and the third port is not isolated."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,carrier\na,380.0,AC\nb,380.0,AC\nc,380.0,AC\n",
                               "links.csv": "name,bus0,bus1,bus2\nk,a,b,c\n"})
    assert lopf.link_ports(n.table("Link")) == ["bus0", "bus1", "bus2"]
    assert len(lopf.controllable_branches(n)) == 3
    assert lopf.isolated_buses(n) == []


def test_attached_components_are_found_by_their_bus():
    """TopologySuite.scala:322-333."""
    n = X.network("ac-dc-meshed")
    at = lopf.attached_to(n, "Manchester")
    assert at and all(n.table(c).endpoint("bus", i) == "Manchester" for c, i in at)
    assert not any(c in ("Line", "Link") for c, _ in at)


def test_an_isolated_bus_is_reported(tmp_path):
    """TopologySuite.scala:335-345."""
    n = _via_reader(tmp_path, {"buses.csv": "name\nconnected0\nconnected1\nnowhere\n",
                               "lines.csv": "name,bus0,bus1\nl0,connected0,connected1\n"})
    assert lopf.isolated_buses(n) == ["nowhere"]


def test_no_golden_network_with_branches_has_an_isolated_bus():
    """TopologySuite.scala:347-373: unit-commitment, one bus and no
    branches, is the degenerate shape and is excluded."""
    with_branches = [name for name in X.NETWORKS
                     if lopf.passive_branches(X.network(name)) or lopf.controllable_branches(X.network(name))]
    assert len(with_branches) >= 5
    for name in with_branches:
        assert lopf.isolated_buses(X.network(name)) == [], name
    single = X.network("unit-commitment")
    assert len(single.table("Bus")) == 1 and lopf.passive_branches(single) == []


def test_component_roles_come_from_pypsas_category():
    """TopologySuite.scala:31-45: Process is a second controllable branch
    and a shunt an attached one-port without either being named."""
    assert lopf.PASSIVE == ("Line", "Transformer")
    assert set(lopf.BRANCHES) - set(lopf.PASSIVE) == {"Link", "Process"}
    assert {"Generator", "Load", "ShuntImpedance", "StorageUnit", "Store"} == set(lopf.ONE_PORTS)
    assert not {"Bus", "Carrier", "LineType"} & set(lopf.BRANCHES + lopf.ONE_PORTS)


@pytest.mark.parametrize("name", X.NETWORKS)
def test_each_golden_network_decomposes_into_pypsas_sub_networks(name):
    """TopologySuite.scala:57-82: the islands PyPSA's
    determine_network_topology found, as a set (PyPSA numbers them its own
    way), and ours in order of their first bus."""
    expected = {(sn["carrier"], tuple(sorted(sn["buses"]))) for sn in X.expected(name)["sub_networks"]}
    actual = [(s.carrier, tuple(s.buses)) for s in lopf.sub_networks(X.network(name))]
    assert len(actual) == len(expected) and set(actual) == expected
    heads = [b[0] for _, b in actual]
    assert heads == sorted(heads)
