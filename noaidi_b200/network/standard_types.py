"""Branch impedance named by a standard type: ``StandardTypes.expand``
(modules/network-model/src/main/scala/org/noaidi/network/StandardTypes.scala).

A line or transformer may set ``type`` instead of its impedance, naming a
row of PyPSA's standard type library; the impedance then exists nowhere in
the network's files.  The library ships beside this module
(``standard_types/line_types.csv``, ``transformer_types.csv``: PyPSA 1.2.4's,
which its CSV export omits), and a network's own ``line_types.csv`` or
``transformer_types.csv`` overrides it row by row.

Expansion happens on the way into a model, as PyPSA does it in
``calculate_dependent_values``, and returns a new network; values already in
the files are overridden by the type, as PyPSA does:

* line: r, x = per-length value x length / num_parallel;
  b = 2 pi 1e-9 f_nom c_per_length x length x num_parallel;
* transformer: r = vscr/100, x = sqrt(max(0, (vsc/100)^2 - r^2)),
  g = pfe / (1000 s_nom), b = -sqrt(max(0, (i0/100)^2 - g^2)), formed from
  the undivided r and g; then r, x / num_parallel and g, b x num_parallel;
  s_nom is the type's, not scaled; tap_ratio = 1 + (tap_position -
  tap_neutral) tap_step / 100; phase_shift and tap_side are the type's.
"""
from __future__ import annotations

import difflib
import math
import os
from dataclasses import replace
from functools import lru_cache

from .pypsa_csv import Network, Table, read_table

LIBRARY = os.path.join(os.path.dirname(os.path.abspath(__file__)), "standard_types")


class UnknownType(ValueError):
    """``StandardTypes.UnknownType``: a type in neither the network nor the library."""


@lru_cache(maxsize=None)
def _shipped(component: str) -> Table:
    stem = {"LineType": "line_types", "TransformerType": "transformer_types"}[component]
    table = read_table(os.path.join(LIBRARY, f"{stem}.csv"), component)
    if table is None:
        raise RuntimeError(f"the standard type library {stem}.csv is empty")
    return table


def type_names(component: str) -> list:
    """Names shipped with this package ("LineType" or "TransformerType")."""
    return list(_shipped(component).ids)


def _library(network: Network, component: str) -> dict:
    """type name -> table holding it: the shipped rows, then the network's own."""
    shipped = _shipped(component)
    merged = {name: shipped for name in shipped.ids}
    merged.update({name: network.table(component) for name in network.table(component).ids})
    return merged


def _type_name(tab: Table, entity: str) -> str:
    v = tab.static.get("type", {}).get(entity)
    return v.strip() if isinstance(v, str) else ""


def _typed(network: Network, component: str) -> bool:
    tab = network.table(component)
    return any(_type_name(tab, i) for i in tab.ids)


def _unknown(component: str, entity: str, name: str, known) -> UnknownType:
    nearest = difflib.get_close_matches(name, list(known), n=3, cutoff=0.0)
    return UnknownType(f"{component} '{entity}' has type '{name}', which is in neither the network's own types nor "
                       f"the {len(known)} shipped here; nearest are {', '.join(repr(x) for x in nearest)}")


def _num(tab: Table, attribute: str, entity: str) -> float:
    return float(tab.value(attribute, entity))


def _expand_lines(network: Network) -> Table:
    tab = network.table("Line")
    library = _library(network, "LineType")
    out = {a: dict(tab.static.get(a, {})) for a in ("r", "x", "b")}
    for i in tab.ids:
        name = _type_name(tab, i)
        if not name:
            for a in out:
                out[a][i] = _num(tab, a, i)
            continue
        if name not in library:
            raise _unknown("Line", i, name, library.keys())
        lt = library[name]
        length, parallel = _num(tab, "length", i), _num(tab, "num_parallel", i)
        if not parallel > 0.0:
            raise UnknownType(f"Line '{i}' has num_parallel = {parallel}, which its type's impedance is divided by")
        out["r"][i] = _num(lt, "r_per_length", name) * length / parallel
        out["x"][i] = _num(lt, "x_per_length", name) * length / parallel
        out["b"][i] = 2.0 * math.pi * 1e-9 * _num(lt, "f_nom", name) * _num(lt, "c_per_length", name) * length * parallel
    return replace(tab, static={**tab.static, **out})


def _expand_transformers(network: Network) -> Table:
    tab = network.table("Transformer")
    library = _library(network, "TransformerType")
    keys = ("r", "x", "g", "b", "s_nom", "tap_ratio", "phase_shift", "tap_side")
    out = {a: dict(tab.static.get(a, {})) for a in keys}
    for i in tab.ids:
        name = _type_name(tab, i)
        if not name:
            for a in keys:
                out[a][i] = _num(tab, a, i)
            continue
        if name not in library:
            raise _unknown("Transformer", i, name, library.keys())
        tt = library[name]
        parallel = _num(tab, "num_parallel", i)
        if not parallel > 0.0:
            raise UnknownType(f"Transformer '{i}' has num_parallel = {parallel}, which its type's impedance is "
                              "divided by")
        s_nom = _num(tt, "s_nom", name)
        if not s_nom > 0.0:
            raise UnknownType(f"transformer type '{name}' has s_nom = {s_nom}")
        r = _num(tt, "vscr", name) / 100.0
        vsc = _num(tt, "vsc", name) / 100.0
        x = math.sqrt(max(0.0, vsc * vsc - r * r))
        g = _num(tt, "pfe", name) / (1000.0 * s_nom)
        i0 = _num(tt, "i0", name) / 100.0
        b = -math.sqrt(max(0.0, i0 * i0 - g * g))
        out["r"][i], out["x"][i] = r / parallel, x / parallel
        out["g"][i], out["b"][i] = g * parallel, b * parallel
        out["s_nom"][i] = s_nom
        out["tap_ratio"][i] = 1.0 + (_num(tab, "tap_position", i) - _num(tt, "tap_neutral", name)) * \
            (_num(tt, "tap_step", name) / 100.0)
        out["phase_shift"][i] = _num(tt, "phase_shift", name)
        out["tap_side"][i] = _num(tt, "tap_side", name)
    return replace(tab, static={**tab.static, **out})


def expand(network: Network) -> Network:
    """The network with every typed branch's impedance filled in; the same
    object when no line or transformer names a type."""
    lines, transformers = _typed(network, "Line"), _typed(network, "Transformer")
    if not lines and not transformers:
        return network
    tables = dict(network.tables)
    if lines:
        tables["Line"] = _expand_lines(network)
    if transformers:
        tables["Transformer"] = _expand_transformers(replace(network, tables=tables))
    return replace(network, tables=tables)
