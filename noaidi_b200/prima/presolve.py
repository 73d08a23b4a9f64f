"""Exact problem reductions before the device solve, undone after it:
``Presolve`` (modules/prima-core/src/main/scala/org/noaidi/prima/Presolve.scala),
run by the C++ presolve in libprima_cuda.so (``prima_presolve``,
include/prima_model.h).

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

import ctypes as C
import math
from dataclasses import dataclass, replace
from typing import Optional

import numpy as np

from .model import LpProblem
from .types import KktError, LpSolution, SolveStatus


def kkt_evaluate(problem: LpProblem, x, y) -> KktError:
    """``Kkt.evaluate`` (Kkt.scala:68-125) in the caller's units: primal
    residual over equality rows and the shortfall of >= rows, objectives, and
    the reduced cost that pushes against an infinite bound as dual residual."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    K = problem.constraint_matrix
    q, c = problem.rhs, problem.objective
    lo, hi = problem.variable_lower, problem.variable_upper
    neq = problem.num_equalities
    ax = K.multiply(x)
    eq = ax[:neq] - q[:neq]
    short = np.maximum(q[neq:] - ax[neq:], 0.0)
    primal_sq = float(np.dot(eq, eq) + np.dot(short, short))
    primal_obj = problem.objective_offset + float(np.dot(c, x))
    aty = K.transpose.multiply(y)
    reduced = c - aty
    dual_obj = problem.objective_offset + float(np.dot(q, y))
    pos, neg = reduced > 0.0, reduced < 0.0
    lo_inf, hi_inf = np.isneginf(lo), np.isposinf(hi)
    dual_sq = float(np.sum(reduced[pos & lo_inf] ** 2) + np.sum(reduced[neg & hi_inf] ** 2))
    dual_obj += float(np.sum(lo[pos & ~lo_inf] * reduced[pos & ~lo_inf]) +
                      np.sum(hi[neg & ~hi_inf] * reduced[neg & ~hi_inf]))
    return KktError(math.sqrt(primal_sq), math.sqrt(dual_sq), primal_obj, dual_obj)


@dataclass(frozen=True)
class Stats:
    """``Presolve.Stats`` (:50-62)."""
    fixed_columns: int
    empty_columns: int
    empty_rows: int
    singleton_rows: int

    @property
    def total(self) -> int:
        return self.fixed_columns + self.empty_columns + self.empty_rows + self.singleton_rows

    @property
    def is_empty(self) -> bool:
        return self.total == 0


class PresolveResult:
    """``Presolve.PresolveResult`` (:65-191) over the library's record of the
    reductions (freed with this object)."""

    def __init__(self, original: LpProblem, handle: int):
        from . import cuda
        self._lib = cuda.library()
        self._handle = handle
        self.original = original
        info = cuda.CPresolveInfo()
        cuda._check(self._lib.prima_presolve_get_info(handle, C.byref(info)))
        self.stats = Stats(info.fixed_columns, info.empty_columns, info.empty_rows, info.singleton_rows)
        self.passes = info.passes
        self.proven_infeasible = bool(info.proven_infeasible)
        self.unbounded_if_feasible = bool(info.unbounded_if_feasible)
        self.column_map = np.zeros(info.reduced_variables, np.int32)
        self.row_map = np.zeros(info.reduced_constraints, np.int32)
        self._reduced = None
        if not self.proven_infeasible:
            cuda._check(self._lib.prima_presolve_get_maps(handle, cuda._ip(self.column_map), cuda._ip(self.row_map)))
            view = cuda.CLp()
            cuda._check(self._lib.prima_presolve_get_reduced(handle, C.byref(view)))
            self._reduced = cuda.lp_from_view(view)

    def __del__(self):
        h, self._handle = getattr(self, "_handle", None), None
        if h:
            self._lib.prima_presolve_free(h)

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
        from . import cuda
        p = self.original
        primal, dual, rc = np.zeros(p.num_variables), np.zeros(p.num_constraints), np.zeros(p.num_variables)
        x = np.ascontiguousarray(solution.primal, dtype=np.float64)
        y = np.ascontiguousarray(solution.dual, dtype=np.float64)
        r = np.ascontiguousarray(solution.reduced_costs, dtype=np.float64)
        cuda._check(self._lib.prima_presolve_restore(self._handle, cuda._dp(x), cuda._dp(y), cuda._dp(r),
                                                     cuda._dp(primal), cuda._dp(dual), cuda._dp(rc)))
        status = solution.status
        if self.unbounded_if_feasible and status == SolveStatus.OPTIMAL:
            status = SolveStatus.DUAL_INFEASIBLE
        return replace(solution, status=status, primal=primal, dual=dual, reduced_costs=rc,
                       objective_value=p.primal_objective(primal), kkt=kkt_evaluate(p, primal, dual))


def presolve(problem: LpProblem, max_passes: int = 20) -> PresolveResult:
    """``Presolve.apply`` (:199-408)."""
    from . import cuda
    lib = cuda.library()
    view = cuda._LpView(problem)
    h = C.c_void_p()
    cuda._check(lib.prima_presolve(C.byref(view.c), int(max_passes), C.byref(h)))
    return PresolveResult(problem, h.value)
