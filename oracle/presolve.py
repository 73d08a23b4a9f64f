"""A Python restatement of ``Presolve``
(modules/prima-core/src/main/scala/org/noaidi/prima/Presolve.scala).

TEST INFRASTRUCTURE ONLY: the oracle for the product's C++ presolve
(``prima_presolve`` in libprima_cuda.so, wrapped by
noaidi_b200/prima/presolve.py).  Imported by ``tests/`` only.

Four rules, applied in passes until nothing changes (at most ``max_passes``),
because they feed one another:

* a column whose bounds coincide is fixed at that value (:237-242);
* a row with no live entries either holds -- relative to the magnitude of its
  right-hand side and of what fixed columns contributed -- or proves the
  problem infeasible (:252-267);
* a row with one live entry is a bound on that column in disguise, folded
  into the column's box; contradictory bounds prove infeasibility
  (:268-292);
* a column in no live row is decided by its cost alone; if that bound is
  infinite the problem is unbounded *if* the rest is feasible, a question the
  reduced solve settles (:294-323).

``PresolveResult.restore`` maps a solution of the reduced problem back,
duals included: a singleton row is priced only when its implied bound is the
one holding the column, by moving the column's reduced cost onto the row
(:146-160); fixed columns get c - K'y from the restored duals (:163-170).
"""
from __future__ import annotations

import math
from dataclasses import replace
from typing import Optional

import numpy as np

from noaidi_b200.prima.model import LpBuilder, LpProblem
from noaidi_b200.prima.presolve import Stats, kkt_evaluate
from noaidi_b200.prima.types import LpSolution, SolveStatus


# Undo records, newest first: ("fixed", j, value), ("empty_col", j, value,
# cost), ("empty_row", r), ("singleton", r, j, coefficient, bound).


class PresolveResult:
    """``Presolve.PresolveResult`` (:65-191)."""

    def __init__(self, original: LpProblem, reduced: Optional[LpProblem], stats: Stats, undo: list,
                 column_map: np.ndarray, row_map: np.ndarray, proven_infeasible: bool,
                 unbounded_if_feasible: bool):
        self.original = original
        self._reduced = reduced
        self.stats = stats
        self._undo = undo
        self.column_map = column_map
        self.row_map = row_map
        self.proven_infeasible = proven_infeasible
        self.unbounded_if_feasible = unbounded_if_feasible

    @property
    def proven_status(self) -> Optional[SolveStatus]:
        """Only infeasibility is ever proven by presolve (:85-101)."""
        return SolveStatus.PRIMAL_INFEASIBLE if self.proven_infeasible else None

    @property
    def reduced(self) -> LpProblem:
        if self.proven_status is not None:
            raise RuntimeError(f"presolve already established {self.proven_status.name}; there is nothing to solve")
        return self._reduced

    def restore(self, solution: LpSolution) -> LpSolution:
        if self.proven_status is not None:
            raise RuntimeError(f"presolve already established {self.proven_status.name}; "
                               "restoring a reduced solution would fabricate one")
        p = self.original
        n, m = p.num_variables, p.num_constraints
        primal, dual, rc = np.zeros(n), np.zeros(m), np.zeros(n)
        primal[self.column_map] = solution.primal
        rc[self.column_map] = solution.reduced_costs
        dual[self.row_map] = solution.dual
        for u in self._undo:
            kind = u[0]
            if kind == "fixed":
                primal[u[1]] = u[2]
                rc[u[1]] = math.nan  # recomputed from the restored duals below
            elif kind == "empty_col":
                primal[u[1]] = u[2]
                rc[u[1]] = u[3]
            elif kind == "empty_row":
                dual[u[1]] = 0.0
            else:
                _, r, j, a, bound = u
                on_bound = abs(primal[j] - bound) <= 1e-7 * max(1.0, abs(bound))
                if on_bound and a != 0.0 and not math.isnan(rc[j]) and rc[j] != 0.0:
                    price = rc[j] / a
                    dual[r] = price
                    rc[j] = rc[j] - a * price
                else:
                    dual[r] = 0.0
        aty = p.constraint_matrix.transpose.multiply(dual)
        nan = np.isnan(rc)
        rc[nan] = p.objective[nan] - aty[nan]
        status = solution.status
        if self.unbounded_if_feasible and status == SolveStatus.OPTIMAL:
            status = SolveStatus.DUAL_INFEASIBLE
        return replace(solution, status=status, primal=primal, dual=dual, reduced_costs=rc,
                       objective_value=p.primal_objective(primal), kkt=kkt_evaluate(p, primal, dual))


def presolve(problem: LpProblem, max_passes: int = 20) -> PresolveResult:
    """``Presolve.apply`` (:199-408)."""
    n, m, neq = problem.num_variables, problem.num_constraints, problem.num_equalities
    K = problem.constraint_matrix
    Kt = K.transpose
    col_alive = np.ones(n, dtype=bool)
    row_alive = np.ones(m, dtype=bool)
    lower = np.array(problem.variable_lower, dtype=np.float64)
    upper = np.array(problem.variable_upper, dtype=np.float64)
    rhs = np.array(problem.rhs, dtype=np.float64)
    c = problem.objective
    fixed_shift = np.zeros(m)
    fixed_value = np.zeros(n)
    undo: list = []
    counts = dict(fixed=0, empty_col=0, empty_row=0, singleton=0)
    infeasible = unbounded_if_feasible = False

    def row_entries(r):
        a, b = K.row_ptr[r], K.row_ptr[r + 1]
        return [(int(j), float(v)) for j, v in zip(K.col_indices[a:b], K.values[a:b]) if col_alive[j]]

    def col_has_live_row(j) -> bool:
        a, b = Kt.row_ptr[j], Kt.row_ptr[j + 1]
        return bool(np.any(row_alive[Kt.col_indices[a:b]]))

    def fix_column(j, value):
        col_alive[j] = False
        fixed_value[j] = value
        counts["fixed"] += 1
        undo.insert(0, ("fixed", j, value))
        a, b = Kt.row_ptr[j], Kt.row_ptr[j + 1]
        for r, v in zip(Kt.col_indices[a:b], Kt.values[a:b]):
            if row_alive[r]:
                fixed_shift[r] += v * value

    passes, changed = 0, True
    while changed and passes < max_passes and not infeasible:
        changed = False
        passes += 1
        for j in range(n):
            if col_alive[j] and lower[j] == upper[j] and math.isfinite(lower[j]):
                fix_column(j, float(lower[j]))
                changed = True
        for r in range(m):
            if infeasible:
                break
            if not row_alive[r]:
                continue
            entries = row_entries(r)
            adjusted = rhs[r] - fixed_shift[r]
            is_eq = r < neq
            if not entries:
                magnitude = max(abs(rhs[r]), abs(fixed_shift[r]))
                scale = 1e-9 * max(1.0, magnitude) if math.isfinite(magnitude) else 1e-9
                holds = abs(adjusted) <= scale if is_eq else adjusted <= scale
                if not holds:
                    infeasible = True
                else:
                    row_alive[r] = False
                    counts["empty_row"] += 1
                    undo.insert(0, ("empty_row", r))
                    changed = True
            elif len(entries) == 1:
                j, a = entries[0]
                bound = adjusted / a
                lo, hi = lower[j], upper[j]
                if is_eq:
                    lo, hi = max(lo, bound), min(hi, bound)
                elif a > 0.0:
                    lo = max(lo, bound)
                else:
                    hi = min(hi, bound)
                if not math.isfinite(lo) or not math.isfinite(hi):
                    contradictory = lo > hi
                else:
                    contradictory = lo > hi + 1e-9 * max(1.0, max(abs(lo), abs(hi)))
                if contradictory:
                    infeasible = True
                else:
                    lower[j] = lo
                    upper[j] = max(hi, lo)
                    row_alive[r] = False
                    counts["singleton"] += 1
                    undo.insert(0, ("singleton", r, j, a, bound))
                    changed = True
        if infeasible:
            break
        for j in range(n):
            if col_alive[j] and not col_has_live_row(j):
                cost = float(c[j])
                if cost > 0.0:
                    at = lower[j]
                elif cost < 0.0:
                    at = upper[j]
                elif math.isfinite(lower[j]):
                    at = lower[j]
                elif math.isfinite(upper[j]):
                    at = upper[j]
                else:
                    at = 0.0
                col_alive[j] = False
                counts["empty_col"] += 1
                if not math.isfinite(at):
                    unbounded_if_feasible = True
                    undo.insert(0, ("empty_col", j, 0.0, cost))
                else:
                    fixed_value[j] = at
                    undo.insert(0, ("empty_col", j, float(at), cost))
                changed = True

    stats = Stats(counts["fixed"], counts["empty_col"], counts["empty_row"], counts["singleton"])
    if infeasible:
        return PresolveResult(problem, None, stats, [], np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int64),
                              True, False)
    column_map = np.flatnonzero(col_alive)
    row_map = np.flatnonzero(row_alive)
    new_col = -np.ones(n, dtype=np.int64)
    new_col[column_map] = np.arange(column_map.size)
    b = LpBuilder(int(column_map.size))
    offset = problem.objective_offset
    for j in np.flatnonzero(~col_alive):
        offset += float(c[j]) * float(fixed_value[j])
    b.objective_offset(offset)
    for i, old in enumerate(column_map):
        b.objective_coefficient(i, float(c[old]))
        b.bounds(i, float(lower[old]), float(upper[old]))
    for old in row_map:
        entries = [(int(new_col[j]), a) for j, a in row_entries(old)]
        value = float(rhs[old] - fixed_shift[old])
        if old < neq:
            b.equality_constraint(entries, value)
        else:
            b.greater_than(entries, value)
    reduced, _ = b.build()
    return PresolveResult(problem, reduced, stats, undo, column_map, row_map, False, unbounded_if_feasible)
