"""A PyPSA CSV network folder read into plain tables: the reference's
network model (modules/network-model/.../CsvReader.scala, Schema.scala,
ComponentTable.scala) as far as the LOPF builders read it.

A folder holds ``<list>.csv`` per component (one row per entity, the first
column its name), ``<list>-<attribute>.csv`` for attributes that vary by
snapshot (one row per snapshot, one column per entity that varies), and
``snapshots.csv`` with the weightings.  Every cell is typed by PyPSA's
component schema (``pypsa_schema.json``, generated from PyPSA 1.2.4's
registry): a float attribute's cell is a number or refused, a boolean's is
true only as ``true``, ``1`` or ``1.0``, an integer's is truncated, text is
trimmed, and a blank cell -- like an omitted column -- takes the schema
default.  A column the schema does not know is a custom attribute, typed
from its values.  A varying attribute without a series file, or an entity
its file does not cover, takes its static value.
"""
from __future__ import annotations

import json
import math
import os
import re
from dataclasses import dataclass, field

import numpy as np

SCHEMA_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pypsa_schema.json")
RESERVED = frozenset({"snapshots.csv", "network.csv", "investment_periods.csv"})  # not component tables


def _storage_type(pypsa_type: str) -> str:
    """``AttributeType.parse`` (Schema.scala:20-37): the varying shapes
    (``series``, ``static or series``, ``static``) are numbers."""
    t = pypsa_type.strip().lower()
    for kind, prefixes in (("float", ("float", "series", "static")), ("int", ("int",)), ("str", ("string",)),
                           ("bool", ("bool",)), ("geometry", ("geometry",))):
        if t.startswith(prefixes):
            return kind
    raise ValueError(f"unknown PyPSA attribute type '{pypsa_type}'")


def _default_text(v) -> str:
    """``Schema.renderDefault`` (Schema.scala:186-198): the schema tags
    non-finite defaults rather than writing invalid JSON."""
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, str):
        return v
    if v is None:
        return ""
    if isinstance(v, dict):
        return "nan" if "$nan" in v else ("-inf" if v.get("$inf") == "-" else "inf")
    if float(v) == math.floor(v) and abs(v) < 1e15:
        return str(int(v))
    return repr(float(v))


def _typed_default(kind: str, text: str):
    """A default as the column type stores it (CsvReader.scala:158-183,
    :206-210): a float default that is absent or not a number is NaN, an
    int's is 0, a boolean's false."""
    if kind == "float":
        if text in ("inf", "-inf", "nan"):
            return {"inf": math.inf, "-inf": -math.inf, "nan": math.nan}[text]
        v = _java_double(_java_trim(text)) if text else None
        return math.nan if v is None else v
    if kind == "int":
        return int(text) if re.fullmatch(r"[+-]?[0-9]+", text) else 0
    if kind == "bool":
        return text in ("true", "True")
    return text


def _load_schema():
    with open(SCHEMA_FILE) as f:
        raw = json.load(f)
    list_names, categories, attributes = {}, {}, {}
    for component, body in raw.items():
        list_names[component] = body["list_name"]
        categories[component] = body.get("category") or ""
        attributes[component] = {}
        for name, a in body["attributes"].items():
            kind = _storage_type(a["type"])
            default = _typed_default(kind, _default_text(a.get("default")))
            attributes[component][name] = (kind, default)
    return list_names, categories, attributes


# Java's String.trim and Double.parseDouble, which the reference's reader
# applies to every cell: trim drops the characters up to U+0020 at either end;
# the number grammar takes an optional sign, NaN, Infinity, decimal or
# hexadecimal significands and a trailing type letter.
_DECIMAL = re.compile(r"[+-]?(?:NaN|Infinity|(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?[fFdD]?)")
_HEX = re.compile(r"([+-]?)0[xX]((?:[0-9a-fA-F]+\.?[0-9a-fA-F]*|\.[0-9a-fA-F]+)[pP][+-]?[0-9]+)[fFdD]?")


def _java_trim(text: str) -> str:
    a, b = 0, len(text)
    while a < b and text[a] <= " ":
        a += 1
    while b > a and text[b - 1] <= " ":
        b -= 1
    return text[a:b]


def _java_double(text: str):
    """``Double.parseDouble`` of a trimmed cell, or None where it throws."""
    if _DECIMAL.fullmatch(text):
        body = text.rstrip("fFdD") if text[-1] in "fFdD" else text
        if body.lstrip("+-") == "NaN":
            return math.nan
        if body.lstrip("+-") == "Infinity":
            return -math.inf if body[0] == "-" else math.inf
        return float(body)
    m = _HEX.fullmatch(text)
    if m:
        v = float.fromhex("0x" + m.group(2))
        return -v if m.group(1) == "-" else v
    return None


# component -> list name; -> PyPSA category (passive_branch, controllable_one_port, ...); -> {attribute: (type, default)}
LIST_NAMES, CATEGORY, SCHEMA = _load_schema()
COMPONENT_OF = {stem: component for component, stem in LIST_NAMES.items()}
# the schema's defaults, which an omitted column or a blank cell resolves to
DEFAULTS = {component: {a: d for a, (_, d) in attrs.items()} for component, attrs in SCHEMA.items()}
PORT = re.compile(r"bus[0-9]+")  # Topology.PortColumn: a bus name even when it reads as a number


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


def split_line(line: str) -> list:
    """``CsvReader.splitLine`` (CsvReader.scala:273-294): commas separate
    fields, a double quote opens and closes a quoted stretch in which a
    doubled quote is one quote and commas are text."""
    if '"' not in line:
        return line.split(",")
    out, buf, quoted, i = [], [], False, 0
    while i < len(line):
        c = line[i]
        if quoted:
            if c == '"':
                if i + 1 < len(line) and line[i + 1] == '"':
                    buf.append('"')
                    i += 1
                else:
                    quoted = False
            else:
                buf.append(c)
        elif c == '"':
            quoted = True
        elif c == ",":
            out.append("".join(buf))
            buf = []
        else:
            buf.append(c)
        i += 1
    out.append("".join(buf))
    return out


def _rows(path: str) -> list:
    """The file's non-empty lines, split (CsvReader.parse, :263-271); a file
    that is not there has none."""
    if not os.path.exists(path):
        return []
    with open(path, encoding="utf-8", newline="") as f:  # lines end at LF, CR or CR LF only, as Java reads them
        return [split_line(line) for line in re.split(r"\r\n|\r|\n", f.read()) if line]


def _number(cell: str, where: str) -> float:
    """``CsvReader.parseFloat`` (CsvReader.scala:212-225): blank is NaN; a
    cell Java cannot parse may still be inf, +inf, infinity, -inf,
    -infinity, nan or na in any case; anything else is refused."""
    t = _java_trim(cell)
    if not t:
        return math.nan
    v = _java_double(t)
    if v is not None:
        return v
    low = t.lower()
    if low in ("inf", "+inf", "infinity"):
        return math.inf
    if low in ("-inf", "-infinity"):
        return -math.inf
    if low in ("nan", "na"):
        return math.nan
    raise MalformedNetwork(f"{where}: '{cell}' is not a number")


def _java_int(t: str, default) -> int:
    """``toIntOption``, else ``toDoubleOption`` cast to an Int (truncated,
    saturating at the 32-bit range, NaN to 0), else the default."""
    if re.fullmatch(r"[+-]?[0-9]+", t) and -2**31 <= int(t) < 2**31:
        return int(t)
    v = _java_double(t)
    if v is None:
        return default
    return 0 if math.isnan(v) else int(max(min(v, 2**31 - 1), -2**31))


def _schema_column(kind: str, default, cells: list, where: str) -> list:
    """A column the schema types (CsvReader.column, :146-183): a blank cell
    takes the default, as an omitted column does."""
    out = []
    for c in cells:
        t = _java_trim(c)
        if not t:
            out.append(default)
        elif kind == "float":
            out.append(_number(c, where))
        elif kind == "int":
            out.append(_java_int(t, default))
        elif kind == "bool":
            out.append(t.lower() in ("true", "1", "1.0"))
        else:
            out.append(t)
    return out


def _inferred_column(name: str, cells: list) -> list:
    """A custom column (CsvReader.inferColumn, :191-204): a port holds bus
    names; otherwise booleans if every present cell is True or False,
    numbers (blank NaN) if every one parses, else text."""
    trimmed = [_java_trim(c) for c in cells]
    present = [t for t in trimmed if t]
    if PORT.fullmatch(name):
        return trimmed
    if present and all(t in ("True", "False") for t in present):
        return [t == "True" for t in trimmed]
    if present:
        parsed = [_java_double(t) if t else math.nan for t in trimmed]
        if all(v is not None for v in parsed):
            return parsed
    return trimmed


def _table_from_rows(rows: list, component: str) -> Table:
    """``CsvReader.staticTable`` (:121-144): names in the first column."""
    if not rows or not rows[0]:
        return Table(component, [])
    header, body = rows[0], rows[1:]
    ids = [r[0] if r else "" for r in body]
    attributes = SCHEMA.get(component, {})
    list_name = LIST_NAMES.get(component, component)
    static = {}
    for k, name in enumerate(header[1:], start=1):
        cells = [r[k] if k < len(r) else "" for r in body]
        if name in attributes:
            kind, default = attributes[name]
            values = _schema_column(kind, default, cells, f"{list_name}.{name}")
        else:
            values = _inferred_column(name, cells)
        static[name] = dict(zip(ids, values))
    return Table(component, ids, static)


def read_table(path: str, component: str):
    """One component list file as a Table of static attributes, or None
    when it has no rows."""
    table = _table_from_rows(_rows(path), component)
    return table if len(table) else None


def _snapshots(path: str):
    """``CsvReader.readSnapshots`` (:87-107): labels from the column headed
    snapshot, else the second; every other named column a weighting, a cell
    that is not a number weighing 1."""
    rows = _rows(path)
    if not rows:
        return [], {}
    header, body = rows[0], rows[1:]
    at = header.index("snapshot") if "snapshot" in header else (1 if len(header) > 1 else 0)
    labels = [r[at] if at < len(r) else "" for r in body]
    weightings = {}
    for k, name in enumerate(header):
        if k == at or not name:
            continue
        w = [_java_double(_java_trim(r[k])) if k < len(r) else None for r in body]
        weightings[name] = np.array([1.0 if v is None else v for v in w], dtype=np.float64)
    return labels, weightings


_PLAIN = re.compile(r"[0-9eE+\-.,]*")  # cells Python and Java read alike


def _series(path: str, snapshots: int, where: str):
    """``CsvReader.readSeries`` (:227-261): the entities it covers and their
    values [snapshots, entities]; one row per snapshot or the file is
    refused."""
    rows = _rows(path)
    if not rows:
        return [], np.zeros((snapshots, 0))
    entities = [_java_trim(h) for h in rows[0][1:]]
    body = rows[1:]
    if len(body) != snapshots:
        raise MalformedNetwork(f"{where} has {len(body)} rows but the network has {snapshots} snapshots")
    values = np.empty((snapshots, len(entities)))
    for t, r in enumerate(body):
        cells = (r[1:] + [""] * len(entities))[:len(entities)]
        if all(c and _PLAIN.fullmatch(c) for c in cells):
            try:
                values[t] = np.array(cells, dtype=np.float64)
                continue
            except ValueError:
                pass  # a malformed number: the cell-by-cell path names it
        values[t] = [_number(c, where) for c in cells]
    return entities, values


def read(folder: str, name: str = "") -> Network:
    """``CsvReader.read`` (CsvReader.scala:34-75): the component tables the
    schema names, each with its series files."""
    if not os.path.isdir(folder):
        raise MalformedNetwork(f"{folder} is not a directory")
    csvs = sorted(f for f in os.listdir(folder) if f.endswith(".csv"))
    snapshots, weightings = _snapshots(os.path.join(folder, "snapshots.csv"))
    series_files: dict = {}
    for f in csvs:
        if "-" in f and f not in RESERVED:
            stem = f[:-4]
            series_files.setdefault(stem[:stem.index("-")], []).append(f)
    tables = {}
    for f in csvs:
        if "-" in f or f in RESERVED or f[:-4] not in COMPONENT_OF:
            continue
        component = COMPONENT_OF[f[:-4]]
        table = _table_from_rows(_rows(os.path.join(folder, f)), component)
        for sf in series_files.get(f[:-4], []):
            attribute = sf[:-4].split("-", 1)[1]
            entities, values = _series(os.path.join(folder, sf), len(snapshots), sf[:-4])
            column = {e: k for k, e in enumerate(entities)}
            arr = np.empty((len(snapshots), len(table.ids)))
            for k, i in enumerate(table.ids):  # an entity the file does not cover keeps its static value
                arr[:, k] = values[:, column[i]] if i in column else float(table.value(attribute, i))
            table.series[attribute] = arr
        if len(table):
            tables[component] = table
    return Network(name or os.path.basename(folder.rstrip("/")), snapshots, weightings, tables)
