"""A PyPSA CSV network folder read into plain tables: the subset of the
reference's network model (modules/network-model/.../CsvReader.scala,
ComponentTable.scala) that the dispatch LOPF needs.

A folder holds ``<list>.csv`` per component (one row per entity, the first
column its name), ``<list>-<attribute>.csv`` for attributes that vary by
snapshot (one row per snapshot, one column per entity), and
``snapshots.csv`` with the weightings.  Attributes a file leaves out take
PyPSA's defaults (the schema's ``default`` entries for the attributes used
here); a varying attribute without a series file takes its static value.
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field

import numpy as np
import pandas as pd

# file stem of each component's tables (PyPSA's list names)
LIST_NAMES = {
    "Bus": "buses", "Carrier": "carriers", "Generator": "generators", "Load": "loads", "Line": "lines",
    "Link": "links", "Transformer": "transformers", "StorageUnit": "storage_units", "Store": "stores",
    "GlobalConstraint": "global_constraints", "SubNetwork": "sub_networks", "ShuntImpedance": "shunt_impedances",
    "LineType": "line_types", "TransformerType": "transformer_types", "Shape": "shapes", "Process": "processes",
}

# PyPSA's defaults for the attributes the dispatch LOPF reads
DEFAULTS = {
    "Bus": {"v_nom": 1.0, "carrier": "AC"},
    "Generator": {"p_nom": 0.0, "p_min_pu": 0.0, "p_max_pu": 1.0, "efficiency": 1.0, "marginal_cost": 0.0,
                  "p_nom_extendable": False, "committable": False, "carrier": "", "p_nom_min": 0.0,
                  "p_nom_max": math.inf, "capital_cost": 0.0, "fom_cost": 0.0, "start_up_cost": 0.0,
                  "shut_down_cost": 0.0, "min_up_time": 0.0, "min_down_time": 0.0, "up_time_before": 1.0,
                  "down_time_before": 0.0, "stand_by_cost": 0.0, "marginal_cost_quadratic": 0.0,
                  "ramp_limit_up": math.nan, "ramp_limit_down": math.nan, "ramp_limit_start_up": math.nan,
                  "ramp_limit_shut_down": math.nan},
    "Load": {"p_set": 0.0},
    "Line": {"x": 0.0, "r": 0.0, "b": 0.0, "g": 0.0, "s_nom": 0.0, "s_max_pu": 1.0, "s_nom_extendable": False,
             "s_nom_min": 0.0, "s_nom_max": math.inf, "capital_cost": 0.0, "fom_cost": 0.0, "length": 0.0,
             "num_parallel": 1.0},
    "Transformer": {"x": 0.0, "r": 0.0, "b": 0.0, "g": 0.0, "s_nom": 0.0, "s_max_pu": 1.0, "tap_ratio": 1.0,
                    "phase_shift": 0.0, "num_parallel": 1.0, "tap_position": 0.0, "tap_side": 0.0,
                    "s_nom_extendable": False, "s_nom_min": 0.0, "s_nom_max": math.inf, "capital_cost": 0.0,
                    "fom_cost": 0.0},
    "Link": {"p_nom": 0.0, "p_min_pu": 0.0, "p_max_pu": 1.0, "efficiency": 1.0, "marginal_cost": 0.0,
             "p_nom_extendable": False, "p_nom_min": 0.0, "p_nom_max": math.inf, "capital_cost": 0.0, "fom_cost": 0.0},
    "StorageUnit": {"p_nom": 0.0, "p_min_pu": -1.0, "p_max_pu": 1.0, "max_hours": 1.0, "efficiency_store": 1.0,
                    "efficiency_dispatch": 1.0, "standing_loss": 0.0, "inflow": 0.0, "state_of_charge_initial": 0.0,
                    "cyclic_state_of_charge": False, "marginal_cost": 0.0, "marginal_cost_storage": 0.0,
                    "spill_cost": 0.0, "state_of_charge_set": math.nan, "p_nom_extendable": False,
                    "p_nom_min": 0.0, "p_nom_max": math.inf, "capital_cost": 0.0, "fom_cost": 0.0},
    "Store": {"e_nom": 0.0, "e_min_pu": 0.0, "e_max_pu": 1.0, "e_initial": 0.0, "e_cyclic": False,
              "standing_loss": 0.0, "marginal_cost": 0.0, "marginal_cost_storage": 0.0, "marginal_cost_quadratic": 0.0,
              "p_set": math.nan, "e_set": math.nan, "e_nom_extendable": False, "e_nom_min": 0.0, "e_nom_max": math.inf,
              "capital_cost": 0.0, "fom_cost": 0.0},
    "GlobalConstraint": {"type": "primary_energy", "carrier_attribute": "co2_emissions", "sense": "=="},
    "Carrier": {"co2_emissions": 0.0},
}


class MalformedNetwork(ValueError):
    """``CsvReader.MalformedNetwork``: the files do not describe a network --
    a branch table without an endpoint column, an endpoint left blank or
    naming no bus."""


@dataclass
class Table:
    """One component's entities: static attributes and per-snapshot series."""
    component: str
    ids: list
    static: dict = field(default_factory=dict)   # attribute -> {id: value}
    series: dict = field(default_factory=dict)   # attribute -> array [snapshots, len(ids)]

    def __len__(self) -> int:
        return len(self.ids)

    def position(self, entity: str) -> int:
        """The entity's column in the series arrays (an index kept in step
        with ``ids``, which callers may append to)."""
        index = self.__dict__.get("_index")
        if index is None or len(index) != len(self.ids):
            index = {i: k for k, i in enumerate(self.ids)}
            self.__dict__["_index"] = index
        return index[entity]

    def has(self, attribute: str) -> bool:
        return attribute in self.static or attribute in self.series

    def endpoint(self, port: str, entity: str) -> str:
        """A bus reference as written: '' for an empty cell or an absent
        column (a port has no default, so a blank never names a bus)."""
        v = self.static.get(port, {}).get(entity)
        return "" if v is None else str(v)

    def value(self, attribute: str, entity: str):
        """A static attribute: PyPSA's default where the file omits the column
        or leaves the cell empty; an explicit NaN stays NaN."""
        if attribute in self.static:
            v = self.static[attribute].get(entity)
            if v is not None:
                return v
        return DEFAULTS.get(self.component, {}).get(attribute, math.nan)

    def at(self, attribute: str, entity: str, t: int) -> float:
        """A varying attribute at snapshot t: its series if there is one, else the static value."""
        if attribute in self.series:
            return float(self.series[attribute][t, self.position(entity)])
        return float(self.value(attribute, entity))


@dataclass
class Network:
    name: str
    snapshots: list
    weightings: dict          # column of snapshots.csv -> array [snapshots]
    tables: dict              # component -> Table

    def table(self, component: str) -> Table:
        return self.tables.get(component) or Table(component, [])

    def weighting(self, column: str, t: int) -> float:
        w = self.weightings.get(column)
        return 1.0 if w is None else float(w[t])


# Attributes that name other entities or labels: kept as text even when they
# read as numbers (bus "0" is a name, not a zero).
LABELS = frozenset({"bus", "bus0", "bus1", "bus2", "bus3", "carrier", "control", "type", "sub_network",
                    "generator", "country", "location", "unit", "sense", "investment_period", "mounting",
                    "references", "model"})


def _coerce(v, label: bool = False):
    """A cell: an empty one is absent (None: the attribute's default
    applies), the text nan an explicit NaN (CsvReader.scala:150-221)."""
    if v is None or (isinstance(v, float) and math.isnan(v)):
        return None
    if isinstance(v, str) and v.strip() == "":
        return None
    if label:
        return str(v)
    if isinstance(v, str):
        t = v.strip()
        if t.lower() in ("true", "false"):
            return t.lower() == "true"
        if t.lower() in ("nan", "na"):
            return math.nan
        try:
            return float(t)
        except ValueError:
            return v
    if isinstance(v, (bool, np.bool_)):
        return bool(v)
    return float(v)


def read_table(path: str, component: str):
    """One component list file (first column the names) as a Table of
    static attributes, or None when it has no rows."""
    df = pd.read_csv(path, dtype=str, keep_default_na=False)
    if df.empty:
        return None
    ids = [str(v) for v in df[df.columns[0]]]
    static = {col: {i: _coerce(v, col in LABELS or re.fullmatch(r"bus[0-9]+", col) is not None)
                    for i, v in zip(ids, df[col])} for col in df.columns[1:]}
    return Table(component, ids, static)


def read(folder: str, name: str = "") -> Network:
    snap = pd.read_csv(os.path.join(folder, "snapshots.csv"))
    label = "snapshot" if "snapshot" in snap.columns else snap.columns[0]
    snapshots = list(snap[label])
    weightings = {c: snap[c].to_numpy(dtype=np.float64) for c in ("objective", "stores", "generators")
                  if c in snap.columns}
    tables = {}
    files = set(os.listdir(folder))
    for component, stem in LIST_NAMES.items():
        if f"{stem}.csv" not in files:
            continue
        static_table = read_table(os.path.join(folder, f"{stem}.csv"), component)
        if static_table is None:
            continue
        ids, static = static_table.ids, static_table.static
        series = {}
        for f in files:
            if f.startswith(stem + "-") and f.endswith(".csv"):
                attr = f[len(stem) + 1:-4]
                s = pd.read_csv(os.path.join(folder, f), index_col=0)
                arr = np.full((len(snapshots), len(ids)), math.nan)
                for k, i in enumerate(ids):
                    if i in s.columns:
                        arr[:, k] = s[i].to_numpy(dtype=np.float64)
                    else:
                        arr[:, k] = float(Table(component, ids, static).value(attr, i))
                series[attr] = arr
        tables[component] = Table(component, ids, static, series)
    return Network(name or os.path.basename(folder.rstrip("/")), snapshots, weightings, tables)
