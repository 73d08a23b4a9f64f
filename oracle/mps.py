"""A Python restatement of ``MpsReader``
(modules/prima-mps/src/main/scala/org/noaidi/prima/mps/MpsReader.scala).

TEST INFRASTRUCTURE ONLY: the oracle for the product's C++ reader
(``prima_mps_read`` in libprima_cuda.so, wrapped by noaidi_b200/prima/mps.py).
Imported by ``tests/`` only.

Lines end at LF, CR or CR LF (``Source.getLines``); a line is trimmed as
Java's ``String.trim`` does (every character at or below U+0020) and split on
Java's ``\\s+`` (space, tab, LF, VT, FF, CR); numbers follow
``java.lang.Double.parseDouble``'s grammar (``String.toDoubleOption``,
MpsReader.scala:284): NaN, Infinity, decimals, hex floats, an optional
f/F/d/D suffix -- and nothing else, so ``inf`` is not a number.

The conventions are the reference's, each of which changes the LP a file
means if done differently:

* whitespace-separated tokens, not fixed columns;
* the first ``N`` row is the objective, later ``N`` rows are free and dropped;
* an ``RHS`` entry on the objective row is the negated objective constant;
* ``MI`` sets only the lower bound to -infinity;
* a negative ``UP`` on a column whose lower bound is still the implicit zero
  also sends the lower bound to -infinity;
* ``RANGES``: ``G`` rows extend upwards, ``L`` rows downwards, ``E`` rows in
  the direction of the range value's sign;
* ``OBJSENSE MAX`` is refused rather than solved with the wrong sign;
* a ``BOUNDS`` line names its column by membership among the declared
  columns (the set name is optional and valueless kinds may carry an ignored
  value), and more than four fields is an error.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Iterable, Optional

import re

from noaidi_b200.prima.model import LpBuilder, LpProblem, RowTranslation

_TRIM = "".join(chr(i) for i in range(0x21))
_SPACE = re.compile(r"[ \t\n\x0b\f\r]+")
_DECIMAL = re.compile(r"[+-]?(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?[fFdD]?")
_HEX = re.compile(r"[+-]?0[xX](?:[0-9a-fA-F]+\.?[0-9a-fA-F]*|\.[0-9a-fA-F]+)[pP][+-]?[0-9]+[fFdD]?")


class MpsParseError(ValueError):
    """``MpsParseException``."""


@dataclass
class MpsInstance:
    """``MpsInstance`` (MpsReader.scala:14-32)."""
    name: str
    problem: LpProblem
    translation: RowTranslation
    row_names: list
    column_names: list
    integer_columns: frozenset

    @property
    def is_mixed_integer(self) -> bool:
        return bool(self.integer_columns)

    def column_index(self, name: str) -> Optional[int]:
        try:
            return self.column_names.index(name)
        except ValueError:
            return None


class _Row:
    __slots__ = ("name", "sense", "rhs", "range", "entries")

    def __init__(self, name: str, sense: str):
        self.name, self.sense, self.rhs, self.range, self.entries = name, sense, 0.0, None, []


class _Col:
    __slots__ = ("name", "index", "lower", "upper", "objective", "integer", "lower_explicit")

    def __init__(self, name: str, index: int):
        self.name, self.index = name, index
        self.lower, self.upper, self.objective = 0.0, math.inf, 0.0
        self.integer = self.lower_explicit = False


def _lines(content: str) -> list:
    return re.split(r"\r\n|\r|\n", content)


def read_file(path: str) -> MpsInstance:
    import os
    with open(path, "rb") as f:
        return read_lines(_lines(f.read().decode("utf-8", "surrogateescape")), os.path.basename(path))


def read_string(content: str, fallback_name: str = "inline") -> MpsInstance:
    return read_lines(_lines(content), fallback_name)


def java_double(token: str):
    """``String.toDoubleOption``: the value, or None outside Java's grammar."""
    t = token.strip(_TRIM)
    sign = t[:1] if t[:1] in ("+", "-") else ""
    body = t[len(sign):]
    if body == "NaN":
        return math.nan
    if body == "Infinity":
        return -math.inf if sign == "-" else math.inf
    core = t[:-1] if t[-1:] in ("f", "F", "d", "D") else t
    if _DECIMAL.fullmatch(t):
        return float(core)
    if _HEX.fullmatch(t):
        return float.fromhex(core)
    return None


def _number(token: str, line: str) -> float:
    v = java_double(token)
    if v is None:
        raise MpsParseError(f"'{token}' is not a number, in: '{line}'")
    return v


def _pairs(fields, line: str, section: str):
    if len(fields) % 2:
        raise MpsParseError(f"{section} entry has an unpaired field: '{line}'")
    return [(fields[i], _number(fields[i + 1], line)) for i in range(0, len(fields), 2)]


def _check_objsense(token: str) -> None:
    if token.upper().startswith("MAX"):
        raise MpsParseError("OBJSENSE MAX is not supported; the solver minimises")


def read_lines(lines: Iterable[str], fallback_name: str) -> MpsInstance:
    """``MpsReader.fromLines`` (:91-235)."""
    name, objective, obj_constant, section, integer_block = fallback_name, "", 0.0, "", False
    rows: dict[str, _Row] = {}
    cols: dict[str, _Col] = {}
    free: set = set()

    def column(cname: str) -> _Col:
        if cname not in cols:
            cols[cname] = _Col(cname, len(cols))
        return cols[cname]

    def row(rname: str, context: str) -> Optional[_Row]:
        if rname in free or rname == objective:
            return None
        if rname not in rows:
            raise MpsParseError(f"{context} refers to unknown row '{rname}'")
        return rows[rname]

    for raw in lines:
        line = raw.rstrip("\r\n").replace("\t", " ")
        trimmed = line.strip(_TRIM)
        if not trimmed or line.startswith("*"):
            continue
        tokens = _SPACE.split(trimmed)
        if not line.startswith(" "):
            section = tokens[0].upper()
            if section == "NAME" and len(tokens) > 1:
                name = tokens[1]
            elif section == "OBJSENSE" and len(tokens) > 1:
                _check_objsense(tokens[1])
            continue
        if section == "ROWS":
            if len(tokens) < 2:
                raise MpsParseError(f"malformed ROWS entry: '{line}'")
            kind, rname = tokens[0].upper(), tokens[1]
            if kind == "N":
                if not objective:
                    objective = rname
                else:
                    free.add(rname)
            elif kind in ("L", "G", "E"):
                rows[rname] = _Row(rname, kind)
            else:
                raise MpsParseError(f"unknown row type '{kind}' for row '{rname}'")
        elif section == "COLUMNS":
            if "'MARKER'" in tokens:
                if any(t.upper() == "'INTORG'" for t in tokens):
                    integer_block = True
                elif any(t.upper() == "'INTEND'" for t in tokens):
                    integer_block = False
                continue
            if len(tokens) < 3:
                raise MpsParseError(f"malformed COLUMNS entry: '{line}'")
            col = column(tokens[0])
            if integer_block:
                col.integer = True
            for rname, value in _pairs(tokens[1:], line, "COLUMNS"):
                if rname == objective:
                    col.objective += value
                elif rname not in free:
                    r = row(rname, "COLUMNS")
                    if r is not None:
                        r.entries.append((col.index, value))
        elif section in ("RHS", "RANGES"):
            fields = tokens[1:] if len(tokens) % 2 == 1 else tokens
            for rname, value in _pairs(fields, line, section):
                if section == "RHS":
                    if rname == objective:
                        obj_constant = -value
                    elif rname not in free:
                        r = row(rname, "RHS")
                        if r is not None:
                            r.rhs = value
                else:
                    r = row(rname, "RANGES")
                    if r is not None:
                        r.range = value
        elif section == "BOUNDS":
            if len(tokens) < 2:
                raise MpsParseError(f"malformed BOUNDS entry: '{line}'")
            kind = tokens[0].upper()
            valueless = kind in ("FR", "MI", "PL", "BV")
            candidates = tokens[1:] if valueless else tokens[1:max(2, len(tokens) - 1)]
            cname = next((t for t in candidates if t in cols), None)
            if cname is None:
                raise MpsParseError(f"BOUNDS names no column declared in COLUMNS (tried {', '.join(candidates)}) "
                                    f"in: '{line}'")
            if len(tokens) > 4:
                raise MpsParseError(f"BOUNDS entry carries more fields than one bound uses: '{line}'")
            col = cols[cname]
            if kind == "UP":
                value = _number(tokens[-1], line)
                col.upper = value
                if value < 0.0 and not col.lower_explicit:
                    col.lower = -math.inf
            elif kind == "LO":
                col.lower, col.lower_explicit = _number(tokens[-1], line), True
            elif kind == "FX":
                value = _number(tokens[-1], line)
                col.lower = col.upper = value
                col.lower_explicit = True
            elif kind == "FR":
                col.lower, col.upper, col.lower_explicit = -math.inf, math.inf, True
            elif kind == "MI":
                col.lower, col.lower_explicit = -math.inf, True
            elif kind == "PL":
                col.upper = math.inf
            elif kind == "BV":
                col.lower, col.upper, col.integer, col.lower_explicit = 0.0, 1.0, True, True
            elif kind == "LI":
                col.lower, col.integer, col.lower_explicit = _number(tokens[-1], line), True, True
            elif kind == "UI":
                col.upper, col.integer = _number(tokens[-1], line), True
            else:
                raise MpsParseError(f"unknown bound type '{kind}' on '{cname}'")
        elif section == "OBJSENSE":
            _check_objsense(tokens[0])
        elif section in ("ENDATA", ""):
            pass
        else:
            raise MpsParseError(f"unexpected data in section '{section}'")

    if not objective:
        raise MpsParseError("no objective row (an N row) was declared")
    return _build(name, obj_constant, list(rows.values()), list(cols.values()))


def _bracket(r: _Row) -> tuple[float, float]:
    """Row sense, right-hand side and optional range as two-sided bounds (:300-316)."""
    if r.range is None:
        return {"L": (-math.inf, r.rhs), "G": (r.rhs, math.inf), "E": (r.rhs, r.rhs)}[r.sense]
    width = abs(r.range)
    if r.sense == "G":
        return r.rhs, r.rhs + width
    if r.sense == "L":
        return r.rhs - width, r.rhs
    return (r.rhs, r.rhs + width) if r.range >= 0.0 else (r.rhs - width, r.rhs)


def _build(name: str, constant: float, rows: list, cols: list) -> MpsInstance:
    b = LpBuilder(len(cols))
    b.objective_offset(constant)
    for c in cols:
        b.objective_coefficient(c.index, c.objective)
        if c.lower > c.upper:
            raise MpsParseError(f"column '{c.name}' has empty bounds [{c.lower}, {c.upper}]")
        b.bounds(c.index, c.lower, c.upper)
    for r in rows:
        lo, hi = _bracket(r)
        b.constraint(r.entries, lo, hi)
    problem, translation = b.build()
    return MpsInstance(name, problem, translation, [r.name for r in rows], [c.name for c in cols],
                       frozenset(c.index for c in cols if c.integer))
