"""Impedance named by a standard type (noaidi_b200/network/standard_types.py),
after the reference's StandardTypesSuite
(modules/network-model/src/test/scala/org/noaidi/network/StandardTypesSuite.scala):
the shipped library's own numbers, not transcriptions, drive the checks."""
import math

import pytest

from noaidi_b200.network import standard_types as S
from noaidi_b200.network.pypsa_csv import Network, Table

LINE_TYPE = "Al/St 240/40 4-bundle 380.0"   # 0.03 ohm/km, 0.246 ohm/km, 13.8 nF/km, 50 Hz
TRANSFORMER_TYPE = "160 MVA 380/110 kV"     # vsc 12.2 %, vscr 0.25 %, pfe 60 kW, i0 0.06 %


def _network(lines=None, transformers=None, own=None):
    tables = {"Bus": Table("Bus", ["A", "B"], {"v_nom": {"A": 380.0, "B": 110.0}})}
    if lines:
        ids = list(lines)
        cols = {a for v in lines.values() for a in v}
        tables["Line"] = Table("Line", ids, {a: {i: lines[i].get(a, math.nan) for i in ids} for a in cols})
    if transformers:
        ids = list(transformers)
        cols = {a for v in transformers.values() for a in v}
        tables["Transformer"] = Table("Transformer", ids, {a: {i: transformers[i].get(a, math.nan) for i in ids}
                                                           for a in cols})
    if own:
        tables.update(own)
    return Network("types", [0], {}, tables)


def _line(type_=LINE_TYPE, length=80.0, parallel=1.0, **kw):
    return {"bus0": "A", "bus1": "B", "type": type_, "length": length, "num_parallel": parallel, "s_nom": 1000.0, **kw}


def _library_row(component, name, attr):
    return float(S._shipped(component).value(attr, name))


def test_the_shipped_library_has_pypsas_rows():
    assert len(S.type_names("LineType")) == 59 and len(S.type_names("TransformerType")) == 14
    assert _library_row("LineType", LINE_TYPE, "x_per_length") == 0.246
    assert _library_row("TransformerType", TRANSFORMER_TYPE, "vsc") == 12.2


def test_a_line_takes_its_impedance_from_the_type():
    n = S.expand(_network(lines={"l": _line(parallel=2.0)}))
    lines = n.table("Line")
    assert float(lines.value("r", "l")) == pytest.approx(0.03 * 80.0 / 2.0, abs=1e-12)
    assert float(lines.value("x", "l")) == pytest.approx(0.246 * 80.0 / 2.0, abs=1e-12)
    assert float(lines.value("b", "l")) == pytest.approx(2.0 * math.pi * 1e-9 * 50.0 * 13.8 * 80.0 * 2.0, abs=1e-18)


def test_parallel_circuits_divide_the_series_impedance_and_multiply_the_shunt():
    n = S.expand(_network(lines={"one": _line(parallel=1.0), "four": _line(parallel=4.0)}))
    lines = n.table("Line")
    assert float(lines.value("x", "one")) / float(lines.value("x", "four")) == pytest.approx(4.0, abs=1e-12)
    assert float(lines.value("b", "four")) / float(lines.value("b", "one")) == pytest.approx(4.0, abs=1e-12)


def test_a_transformer_takes_impedance_and_rating_from_its_percentages():
    n = S.expand(_network(transformers={"t": {"bus0": "A", "bus1": "B", "type": TRANSFORMER_TYPE,
                                              "num_parallel": 2.0}}))
    t = n.table("Transformer")
    r = 0.25 / 100.0
    x = math.sqrt(0.122 * 0.122 - r * r)     # from the undivided r
    g = 60.0 / (1000.0 * 160.0)
    b = -math.sqrt(0.0006 * 0.0006 - g * g)
    assert float(t.value("r", "t")) == pytest.approx(r / 2.0, abs=1e-15)
    assert float(t.value("x", "t")) == pytest.approx(x / 2.0, abs=1e-15)
    assert float(t.value("g", "t")) == pytest.approx(g * 2.0, abs=1e-18)
    assert float(t.value("b", "t")) == pytest.approx(b * 2.0, abs=1e-18)
    assert float(t.value("s_nom", "t")) == 160.0  # the type's, not scaled by num_parallel
    assert float(t.value("tap_ratio", "t")) == 1.0


def test_the_tap_position_moves_the_ratio_by_the_types_step():
    n = S.expand(_network(transformers={"t": {"bus0": "A", "bus1": "B", "type": TRANSFORMER_TYPE,
                                              "tap_position": 2.0}}))
    step = _library_row("TransformerType", TRANSFORMER_TYPE, "tap_step")
    neutral = _library_row("TransformerType", TRANSFORMER_TYPE, "tap_neutral")
    assert float(n.table("Transformer").value("tap_ratio", "t")) == pytest.approx(1.0 + (2.0 - neutral) * step / 100.0)


def test_an_untyped_branch_keeps_its_own_impedance():
    plain = {"bus0": "A", "bus1": "B", "x": 0.4, "r": 0.05, "s_nom": 100.0}
    n = S.expand(_network(lines={"plain": plain, "typed": _line()}))
    lines = n.table("Line")
    assert float(lines.value("x", "plain")) == 0.4 and float(lines.value("r", "plain")) == 0.05
    assert float(lines.value("x", "typed")) == pytest.approx(0.246 * 80.0, abs=1e-12)


def test_a_type_the_network_defines_overrides_the_shipped_one():
    own = Table("LineType", [LINE_TYPE], {"f_nom": {LINE_TYPE: 50.0}, "r_per_length": {LINE_TYPE: 1.0},
                                          "x_per_length": {LINE_TYPE: 2.0}, "c_per_length": {LINE_TYPE: 0.0}})
    n = S.expand(_network(lines={"l": _line()}, own={"LineType": own}))
    assert float(n.table("Line").value("x", "l")) == pytest.approx(2.0 * 80.0, abs=1e-12)


def test_an_unknown_type_is_named_with_the_nearest_matches():
    with pytest.raises(S.UnknownType) as e:
        S.expand(_network(lines={"l": _line(type_="Al/St 240/40 4-bundle 381.0")}))
    assert "Al/St 240/40 4-bundle 381.0" in str(e.value) and LINE_TYPE in str(e.value)


def test_a_non_positive_parallel_count_is_refused():
    with pytest.raises(S.UnknownType, match="num_parallel"):
        S.expand(_network(lines={"l": _line(parallel=0.0)}))


def test_an_untyped_network_is_returned_untouched():
    n = _network(lines={"plain": {"bus0": "A", "bus1": "B", "x": 0.4, "s_nom": 100.0}})
    assert S.expand(n) is n


def test_expansion_is_idempotent():
    once = S.expand(_network(lines={"l": _line(parallel=3.0)},
                             transformers={"t": {"bus0": "A", "bus1": "B", "type": TRANSFORMER_TYPE}}))
    twice = S.expand(once)
    for comp, attrs in (("Line", ("r", "x", "b")), ("Transformer", ("r", "x", "g", "b", "s_nom", "tap_ratio"))):
        for a in attrs:
            assert once.table(comp).static[a] == twice.table(comp).static[a]
