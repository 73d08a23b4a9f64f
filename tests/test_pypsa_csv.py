"""The PyPSA CSV reader (``CsvReader``, modules/network-model/src/main/scala/
org/noaidi/network/CsvReader.scala): the GoldenNetworkSuite.scala cases and
the typing rules the reference applies to each cell."""
import math

import numpy as np
import pytest

from noaidi_b200.network import pypsa_csv
from noaidi_b200.network.pypsa_csv import MalformedNetwork, read, split_line
from tests import lopf_cases as X

SNAPSHOTS = ",snapshot\n0,2015-01-01 00:00:00\n1,2015-01-01 01:00:00\n"


def _via_reader(tmp_path, files):
    files = {"snapshots.csv": SNAPSHOTS, **files}
    for name, body in files.items():
        (tmp_path / name).write_text(body)
    return read(str(tmp_path), "fixture")


def test_a_varying_attribute_resolves_per_entity_falling_back_to_the_static_value():
    """GoldenNetworkSuite.scala:139-159."""
    n = X.network("ac-dc-meshed")
    gens = n.table("Generator")
    with open(f"{X.HERE}/ac-dc-meshed/generators-p_max_pu.csv") as f:
        covered = [c.strip() for c in f.readline().rstrip("\n").split(",")[1:]]
    assert 0 < len(covered) < len(gens)
    for g in gens.ids:
        v = gens.at("p_max_pu", g, 0)
        if g not in covered:
            assert v == float(gens.value("p_max_pu", g)) and math.isfinite(v)
    assert gens.at("p_max_pu", "Manchester Wind", 0) == pytest.approx(0.930019875)


def test_custom_columns_outside_the_schema_are_preserved(tmp_path):
    """GoldenNetworkSuite.scala:161-175."""
    n = _via_reader(tmp_path, {"buses.csv": "name,v_nom,country\nLondon,380,UK\nParis,380,FR\n"})
    assert "country" not in pypsa_csv.SCHEMA["Bus"]
    assert n.table("Bus").value("country", "London") == "UK"


def test_a_blank_cell_resolves_to_the_schema_default_not_to_zero(tmp_path):
    """GoldenNetworkSuite.scala:177-189; an explicit nan stays NaN."""
    n = _via_reader(tmp_path, {"buses.csv": "name\na\n",
                               "generators.csv": "name,bus,efficiency,p_nom_max\ng,a,,\nh,a,nan,1e3\n"})
    gens = n.table("Generator")
    assert gens.value("efficiency", "g") == 1.0 and gens.value("p_nom_max", "g") == math.inf
    assert math.isnan(gens.value("efficiency", "h")) and gens.value("p_nom_max", "h") == 1000.0
    for g in X.network("ac-dc-meshed").table("Generator").ids:
        assert math.isfinite(X.network("ac-dc-meshed").table("Generator").value("efficiency", g))


def test_an_omitted_column_resolves_to_the_schema_default():
    """GoldenNetworkSuite.scala:191-199."""
    buses = X.network("ac-dc-meshed").table("Bus")
    assert len(buses.static) < len(pypsa_csv.SCHEMA["Bus"])
    assert buses.value("v_mag_pu_set", buses.ids[0]) == 1.0
    assert buses.value("type", buses.ids[0]) == ""


def test_entity_ids_and_static_values_match_the_file():
    """GoldenNetworkSuite.scala:201-209."""
    buses = X.network("ac-dc-meshed").table("Bus")
    assert "London" in buses.ids
    assert buses.value("v_nom", "London") > 0.0 and buses.value("carrier", "London") == "AC"


def test_csv_fields_are_unquoted_and_doubled_quotes_collapse():
    """GoldenNetworkSuite.scala:211-217."""
    assert split_line('a,"b,c","say ""hi""",') == ["a", "b,c", 'say "hi"', ""]


def test_a_quoted_name_with_a_comma_is_one_entity(tmp_path):
    n = _via_reader(tmp_path, {"buses.csv": 'name,v_nom\n"Frankfurt, Main",380\nb,220\n'})
    assert n.table("Bus").ids == ["Frankfurt, Main", "b"]
    assert n.table("Bus").value("v_nom", "Frankfurt, Main") == 380.0


def test_the_schema_types_and_defaults_the_builders_read():
    """PyPSA 1.2.4's registry, as Schema.fromJson reads it."""
    s = pypsa_csv.SCHEMA
    assert s["Bus"]["carrier"] == ("str", "AC") and s["Bus"]["v_nom"] == ("float", 1.0)
    assert s["Generator"]["p_nom_extendable"] == ("bool", False)
    assert s["Generator"]["up_time_before"] == ("int", 1)
    assert s["Line"]["s_nom_max"] == ("float", math.inf)
    assert s["StorageUnit"]["state_of_charge_set"][0] == "float"
    assert math.isnan(s["StorageUnit"]["state_of_charge_set"][1])
    assert pypsa_csv.LIST_NAMES["StorageUnit"] == "storage_units"


@pytest.mark.parametrize("cell,value", [
    ("1.5", 1.5), (" 2 ", 2.0), ("1e3", 1000.0), (".5", 0.5), ("3.", 3.0), ("1d", 1.0), ("2.5F", 2.5),
    ("0x1p3", 8.0), ("-0x1.8p1", -3.0), ("Infinity", math.inf), ("-Infinity", -math.inf), ("inf", math.inf),
    ("+INF", math.inf), ("-inf", -math.inf), ("NaN", math.nan), ("na", math.nan), ("nan", math.nan),
])
def test_a_float_cell_follows_the_java_number_grammar(tmp_path, cell, value):
    """CsvReader.parseFloat (CsvReader.scala:212-225): Double.parseDouble,
    then the lower-case spellings of infinity and not-a-number."""
    n = _via_reader(tmp_path, {"buses.csv": f"name,v_nom\na,{cell}\n"})
    got = n.table("Bus").value("v_nom", "a")
    assert (math.isnan(got) and math.isnan(value)) or got == value


@pytest.mark.parametrize("cell", ["abc", "1_000", "1;5", "0x10", "1e", "--1"])
def test_a_float_cell_that_is_not_a_number_is_refused(tmp_path, cell):
    with pytest.raises(MalformedNetwork, match=r"buses\.v_nom"):
        _via_reader(tmp_path, {"buses.csv": f"name,v_nom\na,{cell}\n"})


@pytest.mark.parametrize("cell,value", [("True", True), ("true", True), ("1", True), ("1.0", True), ("TRUE", True),
                                        ("False", False), ("0", False), ("yes", False), ("", False)])
def test_a_boolean_cell_is_true_only_as_true_or_one(tmp_path, cell, value):
    """CsvReader.scala:173-177; a blank takes the default (false)."""
    n = _via_reader(tmp_path, {"buses.csv": "name\na\n", "generators.csv": f"name,bus,p_nom_extendable\ng,a,{cell}\n"})
    assert n.table("Generator").value("p_nom_extendable", "g") is value


@pytest.mark.parametrize("cell,value", [("3", 3), ("3.0", 3), ("3.7", 3), ("-2.5", -2), ("", 1), ("x", 1),
                                        ("9999999999", 2**31 - 1), ("-1e20", -2**31), ("NaN", 0), ("nan", 1)])
def test_an_integer_cell_is_truncated(tmp_path, cell, value):
    """CsvReader.scala:165-171: pandas may write 3 as 3.0; a blank or
    unreadable cell takes the default (up_time_before: 1)."""
    n = _via_reader(tmp_path, {"buses.csv": "name\na\n", "generators.csv": f"name,bus,up_time_before\ng,a,{cell}\n"})
    assert n.table("Generator").value("up_time_before", "g") == value


def test_a_custom_column_is_typed_from_all_its_values(tmp_path):
    """CsvReader.inferColumn (CsvReader.scala:191-204)."""
    n = _via_reader(tmp_path, {"buses.csv": "name,score,flag,note,bus2\na,1.5,True,7,0\nb,,False,x,1\n"})
    b = n.table("Bus")
    assert b.value("score", "a") == 1.5 and math.isnan(b.value("score", "b"))
    assert b.value("flag", "a") is True and b.value("flag", "b") is False
    assert b.value("note", "a") == "7" and b.value("note", "b") == "x"  # one text cell keeps the column text
    assert b.value("bus2", "a") == "0"  # a port holds bus names


def test_a_series_must_have_one_row_per_snapshot(tmp_path):
    """CsvReader.readSeries (CsvReader.scala:237-241)."""
    with pytest.raises(MalformedNetwork, match="1 rows but the network has 2 snapshots"):
        _via_reader(tmp_path, {"buses.csv": "name\na\n", "loads.csv": "name,bus\nd,a\n",
                               "loads-p_set.csv": "snapshot,d\n0,5\n"})


def test_a_series_cell_blank_is_nan_and_an_uncovered_entity_keeps_its_static_value(tmp_path):
    n = _via_reader(tmp_path, {"buses.csv": "name\na\n", "loads.csv": "name,bus,p_set\nd,a,3\ne,a,4\n",
                               "loads-p_set.csv": "snapshot,d\n0,\n1,inf\n"})
    loads = n.table("Load")
    assert math.isnan(loads.at("p_set", "d", 0)) and loads.at("p_set", "d", 1) == math.inf
    assert loads.at("p_set", "e", 0) == 4.0 and loads.at("p_set", "e", 1) == 4.0


def test_a_series_cell_that_is_not_a_number_is_refused(tmp_path):
    with pytest.raises(MalformedNetwork, match="loads-p_set: 'five'"):
        _via_reader(tmp_path, {"buses.csv": "name\na\n", "loads.csv": "name,bus\nd,a\n",
                               "loads-p_set.csv": "snapshot,d\n0,5\n1,five\n"})


def test_snapshot_weightings_default_to_one_and_labels_sit_in_the_second_column(tmp_path):
    """CsvReader.readSnapshots (CsvReader.scala:87-107): without a snapshot
    header the second column labels; a weighting that is not a number is 1."""
    n = _via_reader(tmp_path, {"snapshots.csv": ",when,objective,generators\n0,t0,2,\n1,t1,x,3\n",
                               "buses.csv": "name\na\n"})
    assert n.snapshots == ["t0", "t1"]
    assert list(n.weightings["objective"]) == [2.0, 1.0] and list(n.weightings["generators"]) == [1.0, 3.0]
    assert n.weighting("stores", 0) == 1.0


def test_lines_end_only_at_line_feeds_and_carriage_returns(tmp_path):
    """Files.readAllLines: LF, CR and CR LF end a line; a form feed is text."""
    (tmp_path / "snapshots.csv").write_bytes(b",snapshot\r\n0,t0\r1,t1\n")
    (tmp_path / "buses.csv").write_bytes(b"name,v_nom\r\na\x0cb,380\r\n\r\nc,220\n")
    n = read(str(tmp_path))
    assert n.snapshots == ["t0", "t1"] and n.table("Bus").ids == ["a\x0cb", "c"]


def test_a_missing_folder_is_malformed(tmp_path):
    with pytest.raises(MalformedNetwork):
        read(str(tmp_path / "absent"))


def test_files_the_schema_does_not_name_are_ignored(tmp_path):
    n = _via_reader(tmp_path, {"buses.csv": "name\na\n", "widgets.csv": "name\nw\n", "network.csv": "name\nx\n"})
    assert set(n.tables) == {"Bus"}


def test_every_golden_network_reads_with_its_series_shaped_by_its_snapshots():
    for name in X.NETWORKS:
        n = X.network(name)
        for tab in n.tables.values():
            for arr in tab.series.values():
                assert arr.shape == (len(n.snapshots), len(tab.ids)), name
                assert not np.isnan(arr).all() or len(tab.ids) == 0, name


def test_the_number_grammar_agrees_with_the_oracles_restatement():
    """Seeded random cells: the reader's parse (Java trim, then
    Double.parseDouble) and the MPS oracle's independent restatement of the
    same Java grammar accept the same strings with the same values --
    including refusing digits outside ASCII, which Python's own float takes."""
    from oracle.mps import java_double
    rng = np.random.default_rng(7)
    alphabet = list("0123456789+-.eExXpPfFdDaA ") + ["NaN", "Infinity", "0x", "١", "\t", "_"]
    for _ in range(20000):
        cell = "".join(rng.choice(alphabet, size=int(rng.integers(1, 9))))
        ours = pypsa_csv._java_double(pypsa_csv._java_trim(cell)) if pypsa_csv._java_trim(cell) else None
        theirs = java_double(cell) if cell.strip("".join(chr(i) for i in range(0x21))) else None
        if theirs is None or ours is None:
            assert ours is None and theirs is None, repr(cell)
        else:
            assert (math.isnan(ours) and math.isnan(theirs)) or ours == theirs, repr(cell)
    with pytest.raises(MalformedNetwork):
        pypsa_csv._number("١٢", "buses.v_nom")
