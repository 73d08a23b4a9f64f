"""Parameters and results of the PDHG path.

Mirrors ``PdhgParams`` (``PdhgParams.scala:9-87``), ``ScalingParams``
(``Scaling.scala:11-24``), ``MixedPrecision.Params`` / ``Result``
(``MixedPrecision.scala:37-96``), ``SolveStatus`` / ``LpSolution``
(``SolveResult.scala:9-72``) and ``KktError`` / ``Convergence``
(``Kkt.scala:8-55``), with the same defaults and the same validation.
"""
from __future__ import annotations

import dataclasses
import enum
import math
from typing import Optional

import numpy as np


def _require(cond: bool, msg: str) -> None:
    if not cond:
        raise ValueError("requirement failed: " + msg)


class SolveStatus(enum.IntEnum):
    """Ordinals match the reference enum order (``SolveResult.scala:9-18``)
    and the C ABI's ``PRIMA_STATUS_*`` values."""
    OPTIMAL = 0
    PRIMAL_INFEASIBLE = 1
    DUAL_INFEASIBLE = 2
    ITERATION_LIMIT = 3
    TIME_LIMIT = 4
    NUMERICAL_ERROR = 5
    INTERRUPTED = 6

    @property
    def is_success(self) -> bool:
        return self is SolveStatus.OPTIMAL

    @property
    def is_conclusive(self) -> bool:
        return self in (SolveStatus.OPTIMAL, SolveStatus.PRIMAL_INFEASIBLE, SolveStatus.DUAL_INFEASIBLE)


@dataclasses.dataclass(frozen=True)
class ScalingParams:
    ruiz_iterations: int = 10
    apply_pock_chambolle: bool = True
    pock_chambolle_alpha: float = 1.0

    def __post_init__(self):
        _require(self.ruiz_iterations >= 0, f"ruizIterations must be non-negative, got {self.ruiz_iterations}")
        _require(0.0 <= self.pock_chambolle_alpha <= 2.0,
                 f"pockChambolleAlpha must lie in [0, 2], got {self.pock_chambolle_alpha}")

    @staticmethod
    def none() -> "ScalingParams":
        return ScalingParams(ruiz_iterations=0, apply_pock_chambolle=False)


@dataclasses.dataclass(frozen=True)
class PdhgParams:
    eps_abs: float = 1e-8
    eps_rel: float = 1e-8
    max_iterations: int = 100_000
    time_limit_millis: Optional[int] = None
    evaluation_frequency: int = 64
    scaling: ScalingParams = ScalingParams()
    infeasibility_tolerance: float = 1e-8
    restart_sufficient_reduction: float = 0.2
    restart_necessary_reduction: float = 0.8
    restart_artificial_fraction: float = 0.36
    primal_weight_smoothing: float = 0.5

    def __post_init__(self):
        # PdhgParams.scala:55-79
        _require(self.eps_abs >= 0.0, f"epsAbs must be non-negative, got {self.eps_abs}")
        _require(self.eps_rel >= 0.0, f"epsRel must be non-negative, got {self.eps_rel}")
        _require(self.max_iterations > 0, f"maxIterations must be positive, got {self.max_iterations}")
        _require(self.evaluation_frequency > 0,
                 f"evaluationFrequency must be positive, got {self.evaluation_frequency}")
        _require(0.0 <= self.primal_weight_smoothing <= 1.0,
                 f"primalWeightSmoothing must lie in [0, 1], got {self.primal_weight_smoothing}")
        _require(0.0 < self.restart_sufficient_reduction <= self.restart_necessary_reduction,
                 "restartSufficientReduction must be positive and no greater than restartNecessaryReduction")
        _require(0.0 < self.restart_artificial_fraction <= 1.0,
                 f"restartArtificialFraction must lie in (0, 1], got {self.restart_artificial_fraction}")
        _require(self.infeasibility_tolerance >= 0.0,
                 f"infeasibilityTolerance must be non-negative, got {self.infeasibility_tolerance}")

    def copy(self, **kw) -> "PdhgParams":
        return dataclasses.replace(self, **kw)

    @staticmethod
    def loose() -> "PdhgParams":
        return PdhgParams(eps_abs=1e-6, eps_rel=1e-6)


@dataclasses.dataclass(frozen=True)
class MixedPrecisionParams:
    """``MixedPrecision.Params`` (``MixedPrecision.scala:37-79``)."""
    reduced_tolerance: float = 1e-5
    reduced_max_iterations: int = 20_000
    always_refine: bool = False
    reduced_time_share: float = 0.5

    def __post_init__(self):
        _require(self.reduced_tolerance > 0.0, f"reducedTolerance must be positive, got {self.reduced_tolerance}")
        _require(self.reduced_max_iterations > 0,
                 f"reducedMaxIterations must be positive, got {self.reduced_max_iterations}")
        _require(0.0 < self.reduced_time_share < 1.0,
                 f"reducedTimeShare must lie in (0, 1), got {self.reduced_time_share}")


@dataclasses.dataclass(frozen=True)
class KktError:
    primal_residual_norm: float
    dual_residual_norm: float
    primal_objective: float
    dual_objective: float

    @property
    def duality_gap(self) -> float:
        return self.primal_objective - self.dual_objective

    @property
    def absolute_gap(self) -> float:
        return abs(self.duality_gap)

    @property
    def is_finite(self) -> bool:
        return all(math.isfinite(v) for v in (self.primal_residual_norm, self.dual_residual_norm,
                                              self.primal_objective, self.dual_objective))

    def weighted(self, primal_weight: float) -> float:
        """``KktError.weighted`` (``Kkt.scala:28-33``)."""
        p, d, g = self.primal_residual_norm, self.dual_residual_norm, self.duality_gap
        return math.sqrt(primal_weight * p * p + (d * d) / primal_weight + g * g)


@dataclasses.dataclass(frozen=True)
class Convergence:
    error: KktError
    primal_tolerance: float
    dual_tolerance: float
    gap_tolerance: float

    @property
    def converged(self) -> bool:
        e = self.error
        return (e.is_finite and e.primal_residual_norm <= self.primal_tolerance
                and e.dual_residual_norm <= self.dual_tolerance and e.absolute_gap <= self.gap_tolerance)

    @property
    def relative_error(self) -> float:
        e = self.error
        return max(e.primal_residual_norm / self.primal_tolerance,
                   max(e.dual_residual_norm / self.dual_tolerance, e.absolute_gap / self.gap_tolerance))


def convergence(error: KktError, rhs_norm: float, objective_norm: float, eps_abs: float,
                eps_rel: float) -> Convergence:
    """``Kkt.convergence`` (``Kkt.scala:130-143``)."""
    return Convergence(error, eps_abs + eps_rel * rhs_norm, eps_abs + eps_rel * objective_norm,
                       eps_abs + eps_rel * (abs(error.primal_objective) + abs(error.dual_objective)))


@dataclasses.dataclass
class LpSolution:
    """``LpSolution`` (``SolveResult.scala:33-72``)."""
    status: SolveStatus
    primal: np.ndarray
    dual: np.ndarray
    reduced_costs: np.ndarray
    objective_value: float
    dual_objective_value: float
    iterations: int
    restarts: int
    solve_time_millis: int
    kkt: KktError
    final_step_size: float = math.nan
    final_primal_weight: float = math.nan

    @property
    def duality_gap(self) -> float:
        return self.kkt.absolute_gap

    def __repr__(self) -> str:
        return (f"LpSolution({self.status.name}, obj={self.objective_value:.10g}, gap={self.kkt.absolute_gap:.3e}, "
                f"pRes={self.kkt.primal_residual_norm:.3e}, dRes={self.kkt.dual_residual_norm:.3e}, "
                f"iters={self.iterations}, restarts={self.restarts}, {self.solve_time_millis}ms)")


@dataclasses.dataclass
class MixedPrecisionResult:
    """``MixedPrecision.Result`` (``MixedPrecision.scala:82-96``), plus the
    outer-refinement round count of the device scheme."""
    solution: LpSolution
    reduced_iterations: int
    reduced_restarts: int
    reduced_millis: int
    refinement_iterations: int
    refinement_millis: int
    refined: bool
    refinement_rounds: int = 0

    @property
    def total_iterations(self) -> int:
        return self.reduced_iterations + self.refinement_iterations


@dataclasses.dataclass
class WarmStart:
    """``Pdhg.WarmStart`` (``Pdhg.scala:72-105``): a point in the caller's
    coordinates plus the adaptive state (equilibrated space)."""
    primal: np.ndarray
    dual: np.ndarray
    step_size: Optional[float] = None
    primal_weight: Optional[float] = None

    @staticmethod
    def from_solution(solution: LpSolution) -> "WarmStart":
        _require(bool(np.all(np.isfinite(solution.primal))),
                 "warm start rejected: the source solution's primal vector is not finite")
        _require(bool(np.all(np.isfinite(solution.dual))),
                 "warm start rejected: the source solution has no usable dual vector "
                 "(this backend reports duals it cannot vouch for as NaN)")
        s, w = solution.final_step_size, solution.final_primal_weight
        return WarmStart(np.array(solution.primal, dtype=np.float64), np.array(solution.dual, dtype=np.float64),
                         s if (math.isfinite(s) and s > 0.0) else None,
                         w if (math.isfinite(w) and w > 0.0) else None)

    def save(self, path: str) -> None:
        """The four-tuple to disk (numpy .npz), exactly: a solve resumed from
        ``load(path)`` is the one resumed from this object.  The file lands
        at ``path`` exactly (through a file handle, so numpy adds no
        ``.npz`` suffix)."""
        with open(path, "wb") as f:
            np.savez(f, primal=self.primal, dual=self.dual,
                     step_size=np.float64(math.nan if self.step_size is None else self.step_size),
                     primal_weight=np.float64(math.nan if self.primal_weight is None else self.primal_weight))

    @staticmethod
    def load(path: str) -> "WarmStart":
        with np.load(path) as f:
            s, w = float(f["step_size"]), float(f["primal_weight"])
            return WarmStart(np.array(f["primal"], dtype=np.float64), np.array(f["dual"], dtype=np.float64),
                             None if math.isnan(s) else s, None if math.isnan(w) else w)
