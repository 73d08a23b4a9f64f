"""Linear-program data model: the input contract of the PDHG path.

Host-side mirror of prima-core's model types, with the same names, argument
meaning and error behaviour (``ValueError`` where the reference's ``require``
throws ``IllegalArgumentException``):

* :class:`SparseMatrix` -- canonical CSR (``SparseMatrix.scala:15-318``)
* :class:`LpProblem`    -- standard form, equalities first
  (``LpProblem.scala:22-104``)
* :class:`LpBuilder`    -- two-sided rows to standard form
  (``LpProblem.scala:209-248``), with :class:`RowTranslation` for duals
  (``LpProblem.scala:117-145``)

Arrays are numpy (``int32`` indices, ``float64`` values), laid out exactly as
the C ABI of ``libprima_cuda.so`` takes them, so handing a problem to the
device is a pointer pass, not a conversion.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Iterable, Sequence

import numpy as np


def _require(cond: bool, msg: str) -> None:
    if not cond:
        raise ValueError("requirement failed: " + msg)


class SparseMatrix:
    """Compressed sparse rows, canonical: column indices ascending within a
    row, duplicates summed, exact zeros dropped (``SparseMatrix.scala:5-14``).
    """

    __slots__ = ("rows", "cols", "row_ptr", "col_indices", "values", "_transpose")

    def __init__(self, rows: int, cols: int, row_ptr, col_indices, values):
        self.rows = int(rows)
        self.cols = int(cols)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.col_indices = np.ascontiguousarray(col_indices, dtype=np.int32)
        self.values = np.ascontiguousarray(values, dtype=np.float64)
        self._transpose = None

    # -- construction ------------------------------------------------------
    @staticmethod
    def from_triplets(rows: int, cols: int, r, c, v) -> "SparseMatrix":
        """``SparseMatrix.fromTriplets`` (``SparseMatrix.scala:204-260``):
        stable sort by (row, col), duplicates summed in order of appearance,
        exact zeros dropped, out-of-range and non-finite entries rejected."""
        _require(rows >= 0 and cols >= 0, f"matrix dimensions must be non-negative, got {rows} x {cols}")
        r = np.asarray(r, dtype=np.int64).ravel()
        c = np.asarray(c, dtype=np.int64).ravel()
        v = np.asarray(v, dtype=np.float64).ravel()
        _require(r.shape == c.shape == v.shape, "triplet arrays differ in length")
        if r.size:
            bad_r = np.flatnonzero((r < 0) | (r >= rows))
            _require(bad_r.size == 0, f"row index {int(r[bad_r[0]]) if bad_r.size else 0} out of range [0, {rows})")
            bad_c = np.flatnonzero((c < 0) | (c >= cols))
            _require(bad_c.size == 0, f"column index {int(c[bad_c[0]]) if bad_c.size else 0} out of range [0, {cols})")
            bad_v = np.flatnonzero(~np.isfinite(v))
            _require(bad_v.size == 0, f"entry at ({int(r[bad_v[0]]) if bad_v.size else 0}, "
                                      f"{int(c[bad_v[0]]) if bad_v.size else 0}) is not finite")
        order = np.lexsort((c, r))  # stable: equal keys keep input order
        r, c, v = r[order], c[order], v[order]
        if r.size:
            new_key = np.ones(r.size, dtype=bool)
            new_key[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
            starts = np.flatnonzero(new_key)
            vv = v[starts].copy()
            counts = np.diff(np.append(starts, r.size))
            for g in np.flatnonzero(counts > 1):  # sequential sums, rare
                s0 = starts[g]
                acc = v[s0]
                for k in range(s0 + 1, s0 + counts[g]):
                    acc = acc + v[k]
                vv[g] = acc
            rr, cc = r[starts], c[starts]
            keep = vv != 0.0
            rr, cc, vv = rr[keep], cc[keep], vv[keep]
        else:
            rr, cc, vv = r, c, v
        row_ptr = np.zeros(rows + 1, dtype=np.int64)
        np.add.at(row_ptr, rr + 1, 1)
        row_ptr = np.cumsum(row_ptr)
        _require(row_ptr[-1] < 2**31, "more than 2^31-1 stored entries")
        return SparseMatrix(rows, cols, row_ptr, cc, vv)

    @staticmethod
    def from_dense(data: Sequence[Sequence[float]], cols: int) -> "SparseMatrix":
        """``SparseMatrix.fromDense`` (``SparseMatrix.scala:263-269``)."""
        rr, cc, vv = [], [], []
        for i, row in enumerate(data):
            _require(len(row) == cols, f"row {i} has {len(row)} entries, expected {cols}")
            for j, x in enumerate(row):
                if x != 0.0:
                    rr.append(i), cc.append(j), vv.append(float(x))
        return SparseMatrix.from_triplets(len(data), cols, rr, cc, vv)

    @staticmethod
    def from_csr(rows: int, cols: int, row_ptr, col_indices, values) -> "SparseMatrix":
        """Wrap CSR arrays the caller guarantees canonical (the reference's
        ``fromCsrUnsafe``, ``SparseMatrix.scala:277-284``)."""
        return SparseMatrix(rows, cols, row_ptr, col_indices, values)

    @staticmethod
    def zeros(rows: int, cols: int) -> "SparseMatrix":
        return SparseMatrix(rows, cols, np.zeros(rows + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))

    @staticmethod
    def vstack(blocks: Sequence["SparseMatrix"]) -> "SparseMatrix":
        """``SparseMatrix.vstack`` (``SparseMatrix.scala:293-316``)."""
        _require(len(blocks) > 0, "vstack needs at least one block")
        cols = blocks[0].cols
        for b in blocks:
            _require(b.cols == cols, f"block has {b.cols} columns, expected {cols}")
        ptr = [np.zeros(1, np.int64)]
        base = 0
        for b in blocks:
            ptr.append(b.row_ptr[1:].astype(np.int64) + base)
            base += b.nnz
        return SparseMatrix(sum(b.rows for b in blocks), cols, np.concatenate(ptr),
                            np.concatenate([b.col_indices for b in blocks]),
                            np.concatenate([b.values for b in blocks]))

    # -- properties --------------------------------------------------------
    @property
    def nnz(self) -> int:
        return int(self.row_ptr[self.rows])

    @property
    def transpose(self) -> "SparseMatrix":
        """Materialised transpose (``SparseMatrix.scala:36-64``): a stable
        counting sort by column, so each transposed row stays sorted."""
        if self._transpose is None:
            rows_of = np.repeat(np.arange(self.rows, dtype=np.int32), np.diff(self.row_ptr))
            order = np.argsort(self.col_indices, kind="stable")
            t_ptr = np.zeros(self.cols + 1, dtype=np.int64)
            np.add.at(t_ptr, self.col_indices.astype(np.int64) + 1, 1)
            self._transpose = SparseMatrix(self.cols, self.rows, np.cumsum(t_ptr),
                                           rows_of[order], self.values[order])
            self._transpose._transpose = self
        return self._transpose

    def __call__(self, row: int, col: int) -> float:
        _require(0 <= row < self.rows, f"row {row} out of range [0, {self.rows})")
        _require(0 <= col < self.cols, f"col {col} out of range [0, {self.cols})")
        a, b = self.row_ptr[row], self.row_ptr[row + 1]
        k = np.searchsorted(self.col_indices[a:b], col)
        if k < b - a and self.col_indices[a + k] == col:
            return float(self.values[a + k])
        return 0.0

    def multiply(self, x) -> np.ndarray:
        """Index-order row sums (``SparseMatrix.multiplyInto``, ``:76-86``)."""
        x = np.asarray(x, dtype=np.float64)
        _require(x.shape[0] == self.cols, f"expected a vector of length {self.cols}, got {x.shape[0]}")
        prod = self.values * x[self.col_indices]
        out = np.zeros(self.rows)
        lens = np.diff(self.row_ptr)
        if self.nnz:
            nz = np.flatnonzero(lens > 0)
            out[nz] = np.add.reduceat(prod, self.row_ptr[:-1][nz])
        return out

    def row_abs_sums(self) -> np.ndarray:
        lens = np.diff(self.row_ptr)
        out = np.zeros(self.rows)
        if self.nnz:
            nz = np.flatnonzero(lens > 0)
            out[nz] = np.add.reduceat(np.abs(self.values), self.row_ptr[:-1][nz])
        return out

    @property
    def max_abs(self) -> float:
        return float(np.abs(self.values).max()) if self.nnz else 0.0

    @property
    def norm_inf(self) -> float:
        return float(self.row_abs_sums().max()) if self.rows else 0.0

    @property
    def norm1(self) -> float:
        return self.transpose.norm_inf

    @property
    def norm_frobenius(self) -> float:
        return float(math.sqrt(float(np.dot(self.values, self.values))))

    @property
    def spectral_norm_bound(self) -> float:
        """``sqrt(||K||_1 ||K||_inf)`` (``SparseMatrix.scala:181``)."""
        return math.sqrt(self.norm1 * self.norm_inf)

    def scaled_by(self, row_scale, col_scale) -> "SparseMatrix":
        """diag(row_scale) A diag(col_scale) on the same pattern, each entry
        (a * row) * col (``scaledBy``, SparseMatrix.scala:116-128)."""
        rs = np.asarray(row_scale, dtype=np.float64)
        cs = np.asarray(col_scale, dtype=np.float64)
        _require(rs.shape == (self.rows,) and cs.shape == (self.cols,),
                 f"scales have {rs.size} and {cs.size} entries for a {self.rows} x {self.cols} matrix")
        rows_of = np.repeat(np.arange(self.rows), np.diff(self.row_ptr))
        values = (self.values * rs[rows_of]) * cs[self.col_indices]
        return SparseMatrix(self.rows, self.cols, self.row_ptr, self.col_indices, values)

    def to_dense(self) -> np.ndarray:
        out = np.zeros((self.rows, self.cols))
        rows_of = np.repeat(np.arange(self.rows), np.diff(self.row_ptr))
        out[rows_of, self.col_indices] = self.values
        return out

    def __repr__(self) -> str:
        return f"SparseMatrix({self.rows} x {self.cols}, nnz={self.nnz})"


class LpProblem:
    """``minimise c'x + offset  s.t.  Kx = q (first num_equalities rows),
    Kx >= q (rest), l <= x <= u`` (``LpProblem.scala:7-20``)."""

    __slots__ = ("objective", "objective_offset", "constraint_matrix", "rhs",
                 "num_equalities", "variable_lower", "variable_upper")

    def __init__(self, objective, constraint_matrix: SparseMatrix, rhs, num_equalities: int,
                 variable_lower, variable_upper, objective_offset: float = 0.0):
        c = np.ascontiguousarray(objective, dtype=np.float64)
        q = np.ascontiguousarray(rhs, dtype=np.float64)
        lo = np.ascontiguousarray(variable_lower, dtype=np.float64)
        hi = np.ascontiguousarray(variable_upper, dtype=np.float64)
        n = c.shape[0]
        # LpProblem.apply, LpProblem.scala:62-104
        _require(constraint_matrix.cols == n, f"matrix has {constraint_matrix.cols} columns, expected {n}")
        _require(constraint_matrix.rows == q.shape[0],
                 f"matrix has {constraint_matrix.rows} rows but rhs has {q.shape[0]} entries")
        _require(0 <= num_equalities <= q.shape[0],
                 f"numEqualities {num_equalities} out of range [0, {q.shape[0]}]")
        _require(lo.shape[0] == n, f"lower bounds have {lo.shape[0]} entries, expected {n}")
        _require(hi.shape[0] == n, f"upper bounds have {hi.shape[0]} entries, expected {n}")
        bad = np.flatnonzero(~(lo <= hi))
        _require(bad.size == 0, f"variable {bad[0] if bad.size else 0} has empty bound interval")
        bad = np.flatnonzero(~np.isfinite(c))
        _require(bad.size == 0, f"objective coefficient {bad[0] if bad.size else 0} is not finite")
        bad = np.flatnonzero(~np.isfinite(q))
        _require(bad.size == 0, f"right-hand side {bad[0] if bad.size else 0} is not finite")
        self.objective = c
        self.objective_offset = float(objective_offset)
        self.constraint_matrix = constraint_matrix
        self.rhs = q
        self.num_equalities = int(num_equalities)
        self.variable_lower = lo
        self.variable_upper = hi

    @property
    def num_variables(self) -> int:
        return int(self.objective.shape[0])

    @property
    def num_constraints(self) -> int:
        return int(self.rhs.shape[0])

    @property
    def num_inequalities(self) -> int:
        return self.num_constraints - self.num_equalities

    def primal_objective(self, x) -> float:
        x = np.asarray(x, dtype=np.float64)
        _require(x.shape[0] == self.num_variables, f"expected {self.num_variables} variables, got {x.shape[0]}")
        s = self.objective_offset
        for a, b in zip(self.objective, x):
            s += a * b
        return s

    @staticmethod
    def builder(num_variables: int) -> "LpBuilder":
        return LpBuilder(num_variables)

    def __repr__(self) -> str:
        return (f"LpProblem(vars={self.num_variables}, eq={self.num_equalities}, "
                f"ineq={self.num_inequalities}, nnz={self.constraint_matrix.nnz})")


@dataclasses.dataclass(frozen=True)
class Direct:
    row: int


@dataclasses.dataclass(frozen=True)
class Negated:
    row: int


@dataclasses.dataclass(frozen=True)
class Range:
    lower_row: int
    upper_row: int


class RowTranslation:
    """Standard-form duals back to the caller's rows (``LpProblem.scala:128-145``)."""

    def __init__(self, expansions):
        self._expansions = list(expansions)

    @property
    def num_original_rows(self) -> int:
        return len(self._expansions)

    def expansion_of(self, original_row: int):
        return self._expansions[original_row]

    def original_duals(self, standard_duals) -> np.ndarray:
        d = np.asarray(standard_duals, dtype=np.float64)
        out = np.empty(len(self._expansions))
        for i, e in enumerate(self._expansions):
            if isinstance(e, Direct):
                out[i] = d[e.row]
            elif isinstance(e, Negated):
                out[i] = -d[e.row]
            else:
                out[i] = d[e.lower_row] - d[e.upper_row]
        return out


class LpBuilder:
    """Rows as ``lo <= a'x <= hi`` (``LpProblem.scala:152-248``)."""

    def __init__(self, num_variables: int):
        _require(num_variables >= 0, f"numVariables must be non-negative, got {num_variables}")
        self._n = int(num_variables)
        self._objective = np.zeros(self._n)
        self._lower = np.full(self._n, -np.inf)
        self._upper = np.full(self._n, np.inf)
        self._offset = 0.0
        self._rows: list[tuple[list, float, float]] = []

    def _check_variable(self, v: int) -> None:
        _require(0 <= v < self._n, f"variable index {v} out of range [0, {self._n})")

    def objective_coefficient(self, variable: int, value: float) -> "LpBuilder":
        self._check_variable(variable)
        self._objective[variable] = value
        return self

    def objective_offset(self, value: float) -> "LpBuilder":
        self._offset = float(value)
        return self

    def bounds(self, variable: int, lo: float, hi: float) -> "LpBuilder":
        self._check_variable(variable)
        _require(lo <= hi, f"variable {variable} has empty bound interval [{lo}, {hi}]")
        self._lower[variable] = lo
        self._upper[variable] = hi
        return self

    def constraint(self, coefficients: Iterable[tuple[int, float]], lo: float, hi: float) -> "LpBuilder":
        _require(lo <= hi, f"constraint has empty range [{lo}, {hi}]")
        _require(not (lo == -math.inf and hi == math.inf),
                 "constraint is unbounded on both sides and would have no effect")
        coefficients = [(int(j), float(a)) for j, a in coefficients]
        for j, _ in coefficients:
            self._check_variable(j)
        self._rows.append((coefficients, float(lo), float(hi)))
        return self

    def equality_constraint(self, coefficients, value: float) -> "LpBuilder":
        return self.constraint(coefficients, value, value)

    def greater_than(self, coefficients, lo: float) -> "LpBuilder":
        return self.constraint(coefficients, lo, math.inf)

    def less_than(self, coefficients, hi: float) -> "LpBuilder":
        return self.constraint(coefficients, -math.inf, hi)

    def build(self) -> tuple[LpProblem, RowTranslation]:
        """Equalities first (insertion order), then inequalities; ``<=`` rows
        negated; ranges split into ``a'x >= lo`` and ``-a'x >= -hi``
        (``LpProblem.scala:209-248``)."""
        er, ec, ev, rhs = [], [], [], []
        expansions: list = [None] * len(self._rows)

        def emit(coefficients, sign, value):
            r = len(rhs)
            for j, a in coefficients:
                er.append(r), ec.append(j), ev.append(sign * a)
            rhs.append(sign * value)
            return r

        for i, (co, lo, hi) in enumerate(self._rows):
            if lo == hi:
                expansions[i] = Direct(emit(co, 1.0, lo))
        num_eq = len(rhs)
        for i, (co, lo, hi) in enumerate(self._rows):
            if lo == hi:
                continue
            has_lo, has_hi = lo != -math.inf, hi != math.inf
            if has_lo and has_hi:
                expansions[i] = Range(emit(co, 1.0, lo), emit(co, -1.0, hi))
            elif has_lo:
                expansions[i] = Direct(emit(co, 1.0, lo))
            else:
                expansions[i] = Negated(emit(co, -1.0, hi))
        matrix = SparseMatrix.from_triplets(len(rhs), self._n, er, ec, ev)
        problem = LpProblem(self._objective.copy(), matrix, np.array(rhs, dtype=np.float64), num_eq,
                            self._lower.copy(), self._upper.copy(), self._offset)
        return problem, RowTranslation(expansions)
