"""Unit commitment (noaidi_b200/network/unit_commitment.py) on CPU, with the
oracle solving every branch-and-bound node."""
import os

import pytest

from noaidi_b200.network import unit_commitment as U
from noaidi_b200.network.pypsa_csv import Table, read
from tests import bnb_fixtures as B
from tests import uc_cases as X


def oracle_solve(n):
    model = U.build(n)
    return U.solve(n, U.DEFAULT_PARAMS, node_solver=B.oracle_node_solver(model.problem))


def test_unit_commitment_matches_pypsa_with_the_oracle():
    X.check_against_pypsa(oracle_solve)


def test_a_unit_part_way_through_its_minimum_up_time_is_held_on(tmp_path):
    X.check_residual(oracle_solve, str(tmp_path / "residual"))


def test_only_status_columns_are_integer():
    model = U.build(X.network())
    kinds = {k for (k, _, _), j in model.columns.items() if j in model.integers}
    assert kinds == {"u"} and len(model.integers) == 2 * 8


@pytest.mark.parametrize("mutate, word", [
    (lambda n: n.table("Generator").static.__setitem__("ramp_limit_up", {g: 0.5 for g in n.table("Generator").ids}),
     "ramp"),
    (lambda n: n.tables.__setitem__("Line", Table("Line", ["l"], {"bus0": {"l": "bus"}, "bus1": {"l": "bus"}})),
     "Line"),
    (lambda n: n.table("Load").static.__setitem__("bus", {"d": "buss"}), "buss"),
    (lambda n: n.tables.__setitem__("GlobalConstraint", Table("GlobalConstraint", ["co2"], {})),
     "global constraint"),
    (lambda n: n.table("Generator").static.__setitem__("stand_by_cost", {g: 5.0 for g in n.table("Generator").ids}),
     "stand_by_cost"),
])
def test_what_the_formulation_does_not_model_is_refused(mutate, word):
    n = X.network()
    mutate(n)
    with pytest.raises(U.UnsupportedNetwork, match=word):
        U.build(n)


def test_a_series_only_stand_by_cost_is_refused(tmp_path):
    """UnitCommitmentSuite.scala:306-319: PyPSA writes the attribute as its
    own file when only the series is non-default; there is no static column."""
    import shutil
    src = os.path.join(X.HERE, "unit-commitment")
    for f in os.listdir(src):
        shutil.copy(os.path.join(src, f), tmp_path / f)
    (tmp_path / "generators-stand_by_cost.csv").write_text(
        ",base\n0,0.0\n1,0.0\n2,25.0\n3,0.0\n4,0.0\n5,0.0\n6,0.0\n7,0.0\n")
    n = read(str(tmp_path))
    assert "stand_by_cost" not in n.table("Generator").static
    with pytest.raises(U.UnsupportedNetwork, match="stand_by_cost"):
        U.build(n)


def test_a_priced_attribute_is_refused_even_with_no_snapshots(tmp_path):
    """UnitCommitmentSuite.scala:321-344."""
    (tmp_path / "buses.csv").write_text("name,v_nom,carrier\nbus,110.0,AC\n")
    (tmp_path / "generators.csv").write_text("name,bus,p_nom,p_min_pu,marginal_cost,committable,stand_by_cost\n"
                                             "unit,bus,100.0,0.5,10.0,True,25.0\n")
    (tmp_path / "loads.csv").write_text("name,bus,p_set\nd,bus,50.0\n")
    (tmp_path / "snapshots.csv").write_text(",snapshot\n")
    n = read(str(tmp_path))
    assert len(n.snapshots) == 0
    with pytest.raises(U.UnsupportedNetwork, match="stand_by_cost"):
        U.build(n)
