"""The MPS reader: ``MpsReader``
(modules/prima-mps/src/main/scala/org/noaidi/prima/mps/MpsReader.scala), the
on-disk format in front of the device solve, run by the C++ reader in
libprima_cuda.so (``prima_mps_read``, include/prima_model.h).

The conventions are the reference's, each of which changes the LP a file
means if done differently:

* whitespace-separated tokens, not fixed columns; lines end at LF, CR or
  CR LF; numbers follow ``java.lang.Double.parseDouble``'s grammar;
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

import ctypes as C
import os
from dataclasses import dataclass
from typing import Iterable, Optional

import numpy as np

from . import cuda
from .model import Direct, LpProblem, Negated, Range, RowTranslation


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


def _text(b: Optional[bytes]) -> str:
    return "" if b is None else b.decode("utf-8", "surrogateescape")


def _instance(lib, code: int, handle: C.c_void_p) -> MpsInstance:
    if code != cuda.OK:
        msg = lib.prima_last_error().decode("utf-8", "surrogateescape")
        if code == cuda.ERR_PARSE:
            raise MpsParseError(msg)
        if code == cuda.ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        raise cuda.PrimaError(code, msg)
    h = handle.value
    try:
        info = cuda.CMpsInfo()
        cuda._check(lib.prima_mps_get_info(h, C.byref(info)))
        view = cuda.CLp()
        cuda._check(lib.prima_mps_get_problem(h, C.byref(view)))
        problem = cuda.lp_from_view(view)
        k = info.num_rows
        kind, first, second = (np.zeros(k, np.int32) for _ in range(3))
        cuda._check(lib.prima_mps_get_translation(h, cuda._ip(kind), cuda._ip(first), cuda._ip(second)))
        rows = [Direct(int(a)) if t == 0 else Negated(int(a)) if t == 1 else Range(int(a), int(b))
                for t, a, b in zip(kind, first, second)]
        integers = np.zeros(info.num_integer_columns, np.int32)
        cuda._check(lib.prima_mps_get_integer_columns(h, cuda._ip(integers)))
        return MpsInstance(_text(lib.prima_mps_name(h)), problem, RowTranslation(rows),
                           [_text(lib.prima_mps_row_name(h, i)) for i in range(k)],
                           [_text(lib.prima_mps_column_name(h, j)) for j in range(info.num_variables)],
                           frozenset(int(j) for j in integers))
    finally:
        lib.prima_mps_free(h)


def read_string(content: str, fallback_name: str = "inline") -> MpsInstance:
    """``MpsReader.fromString``."""
    lib = cuda.library()
    data = content.encode("utf-8", "surrogateescape")
    h = C.c_void_p()
    code = lib.prima_mps_read(data, len(data), fallback_name.encode("utf-8", "surrogateescape"), C.byref(h))
    return _instance(lib, code, h)


def read_file(path: str) -> MpsInstance:
    """``MpsReader.read(path)``: the file's base name is the fallback name."""
    lib = cuda.library()
    h = C.c_void_p()
    code = lib.prima_mps_read_file(os.fsencode(path), C.byref(h))
    return _instance(lib, code, h)


def read_lines(lines: Iterable[str], fallback_name: str) -> MpsInstance:
    """``MpsReader.fromLines``."""
    return read_string("\n".join(line.rstrip("\r\n") for line in lines), fallback_name)
