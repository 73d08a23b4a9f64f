"""ctypes loader for the C restatement of Prima's PDHG path.

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg, and there only as the oracle results
are compared with, or as the timed CPU reference.  The product (``noaidi_b200``) never imports this.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

from noaidi_b200.prima.types import (KktError, LpSolution, MixedPrecisionParams, MixedPrecisionResult,
                                     PdhgParams, SolveStatus)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

FP64 = 0  # ScalaKernels
FP32 = 1  # Float32Kernels


class OrcParams(C.Structure):
    _fields_ = [("eps_abs", C.c_double), ("eps_rel", C.c_double), ("max_iterations", C.c_int32),
                ("evaluation_frequency", C.c_int32), ("time_limit_ms", C.c_double),
                ("ruiz_iterations", C.c_int32), ("apply_pock_chambolle", C.c_int32),
                ("pock_chambolle_alpha", C.c_double), ("infeasibility_tolerance", C.c_double),
                ("restart_sufficient_reduction", C.c_double), ("restart_necessary_reduction", C.c_double),
                ("restart_artificial_fraction", C.c_double), ("primal_weight_smoothing", C.c_double)]


class OrcResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32),
                ("pad", C.c_int32), ("solve_ms", C.c_int64), ("objective", C.c_double),
                ("dual_objective", C.c_double), ("primal_residual", C.c_double),
                ("dual_residual", C.c_double), ("final_step_size", C.c_double),
                ("final_primal_weight", C.c_double)]


class OrcMixedParams(C.Structure):
    _fields_ = [("reduced_tolerance", C.c_double), ("reduced_max_iterations", C.c_int32),
                ("always_refine", C.c_int32), ("reduced_time_share", C.c_double)]


class OrcMixedInfo(C.Structure):
    _fields_ = [("reduced_iterations", C.c_int32), ("reduced_restarts", C.c_int32),
                ("reduced_ms", C.c_int64), ("refinement_iterations", C.c_int32),
                ("refined", C.c_int32), ("refinement_ms", C.c_int64)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.orc_csr_from_triplets.restype = C.c_int64
        for f in ("orc_csr_norm_inf", "orc_csr_spectral_norm_bound", "orc_k_dot", "orc_k_squared_norm"):
            getattr(_lib, f).restype = C.c_double
    return _lib


def _p(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _d(a):
    return _p(a, C.c_double)


def _i(a):
    return _p(a, C.c_int32)


def to_c_params(p: PdhgParams) -> OrcParams:
    return OrcParams(p.eps_abs, p.eps_rel, p.max_iterations, p.evaluation_frequency,
                     -1.0 if p.time_limit_millis is None else float(p.time_limit_millis),
                     p.scaling.ruiz_iterations, int(p.scaling.apply_pock_chambolle),
                     p.scaling.pock_chambolle_alpha, p.infeasibility_tolerance,
                     p.restart_sufficient_reduction, p.restart_necessary_reduction,
                     p.restart_artificial_fraction, p.primal_weight_smoothing)


def _arrays(problem):
    K = problem.constraint_matrix
    return (problem.num_variables, problem.num_constraints, problem.num_equalities, K.row_ptr,
            K.col_indices, K.values, problem.objective, problem.rhs, problem.variable_lower,
            problem.variable_upper, problem.objective_offset)


def _solution(res: OrcResult, x, y, rc) -> LpSolution:
    return LpSolution(SolveStatus(res.status), x, y, rc, res.objective, res.dual_objective,
                      res.iterations, res.restarts, int(res.solve_ms),
                      KktError(res.primal_residual, res.dual_residual, res.objective, res.dual_objective),
                      res.final_step_size, res.final_primal_weight)


def solve(problem, params: PdhgParams = PdhgParams(), mode: int = FP64, warm_start=None,
          cancel=None) -> LpSolution:
    """``Pdhg.solveWith(problem, params, ScalaKernels|Float32Kernels, ...)``."""
    n, m, neq, rp, ci, v, c, q, lo, hi, off = _arrays(problem)
    x, y, rc = np.zeros(n), np.zeros(m), np.zeros(n)
    res = OrcResult()
    wx = wy = None
    ws = ww = math.nan
    if warm_start is not None:
        if len(warm_start.primal) != n:
            raise ValueError(f"requirement failed: warm start has {len(warm_start.primal)} primal entries, expected {n}")
        if len(warm_start.dual) != m:
            raise ValueError(f"requirement failed: warm start has {len(warm_start.dual)} dual entries, expected {m}")
        wx = np.ascontiguousarray(warm_start.primal, dtype=np.float64)
        wy = np.ascontiguousarray(warm_start.dual, dtype=np.float64)
        ws = math.nan if warm_start.step_size is None else warm_start.step_size
        ww = math.nan if warm_start.primal_weight is None else warm_start.primal_weight
    cp = to_c_params(params)
    flag = None if cancel is None else C.byref(cancel)
    rc_ = lib().orc_pdhg_solve(n, m, neq, _i(rp), _i(ci), _d(v), _d(c), _d(q), _d(lo), _d(hi),
                               C.c_double(off), C.byref(cp), mode, _d(wx), _d(wy), C.c_double(ws),
                               C.c_double(ww), flag, _d(x), _d(y), _d(rc), C.byref(res))
    if rc_ != 0:
        raise ValueError("requirement failed: invalid argument to the oracle solve")
    return _solution(res, x, y, rc)


def mixed_solve(problem, params: PdhgParams = PdhgParams(),
                mixed: MixedPrecisionParams = MixedPrecisionParams(), cancel=None) -> MixedPrecisionResult:
    """``MixedPrecision.solve(problem, params, Float32Kernels, mixed)``."""
    n, m, neq, rp, ci, v, c, q, lo, hi, off = _arrays(problem)
    x, y, rc = np.zeros(n), np.zeros(m), np.zeros(n)
    res, info = OrcResult(), OrcMixedInfo()
    mp = OrcMixedParams(mixed.reduced_tolerance, mixed.reduced_max_iterations, int(mixed.always_refine),
                        mixed.reduced_time_share)
    cp = to_c_params(params)
    flag = None if cancel is None else C.byref(cancel)
    rc_ = lib().orc_mixed_solve(n, m, neq, _i(rp), _i(ci), _d(v), _d(c), _d(q), _d(lo), _d(hi),
                                C.c_double(off), C.byref(cp), C.byref(mp), flag, _d(x), _d(y), _d(rc),
                                C.byref(res), C.byref(info))
    if rc_ != 0:
        raise ValueError("requirement failed: invalid argument to the oracle mixed solve")
    return MixedPrecisionResult(_solution(res, x, y, rc), info.reduced_iterations, info.reduced_restarts,
                                int(info.reduced_ms), info.refinement_iterations, int(info.refinement_ms),
                                bool(info.refined))


def kkt_evaluate(problem, x, y, kx=None, kty=None) -> KktError:
    n, m, neq, rp, ci, v, c, q, lo, hi, off = _arrays(problem)
    out = np.zeros(4)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    kx = None if kx is None else np.ascontiguousarray(kx, dtype=np.float64)
    kty = None if kty is None else np.ascontiguousarray(kty, dtype=np.float64)
    lib().orc_kkt_evaluate(n, m, neq, _i(rp), _i(ci), _d(v), _d(c), _d(q), _d(lo), _d(hi),
                           C.c_double(off), _d(x), _d(y), _d(kx), _d(kty), _d(out))
    return KktError(*[float(t) for t in out])


def primal_infeasibility(problem, y, kty=None):
    n, m, neq, rp, ci, v, c, q, lo, hi, off = _arrays(problem)
    y = np.ascontiguousarray(y, dtype=np.float64)
    kty = None if kty is None else np.ascontiguousarray(kty, dtype=np.float64)
    out = C.c_double()
    ok = lib().orc_primal_infeasibility(n, m, neq, _i(rp), _i(ci), _d(v), _d(q), _d(lo), _d(hi), _d(y),
                                        _d(kty), C.byref(out))
    return out.value if ok else None


def dual_infeasibility(problem, d, kd=None):
    n, m, neq, rp, ci, v, c, q, lo, hi, off = _arrays(problem)
    d = np.ascontiguousarray(d, dtype=np.float64)
    kd = None if kd is None else np.ascontiguousarray(kd, dtype=np.float64)
    out = C.c_double()
    ok = lib().orc_dual_infeasibility(n, m, neq, _i(rp), _i(ci), _d(v), _d(c), _d(lo), _d(hi), _d(d),
                                      _d(kd), C.byref(out))
    return out.value if ok else None


def classify(problem, x, y, tolerance, kx=None, kty=None):
    n, m, neq, rp, ci, v, c, q, lo, hi, off = _arrays(problem)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    kx = None if kx is None else np.ascontiguousarray(kx, dtype=np.float64)
    kty = None if kty is None else np.ascontiguousarray(kty, dtype=np.float64)
    s = lib().orc_classify(n, m, neq, _i(rp), _i(ci), _d(v), _d(c), _d(q), _d(lo), _d(hi), _d(x), _d(y),
                           C.c_double(tolerance), _d(kx), _d(kty))
    return None if s < 0 else SolveStatus(s)


def scale(problem, ruiz_iterations=10, apply_pc=True, alpha=1.0):
    """``Scaling.apply``: returns (scaled values, c, q, l, u, rowScale, colScale)."""
    n, m, neq, rp, ci, v, c, q, lo, hi, off = _arrays(problem)
    sv, sc, sq, sl, su = np.zeros(len(v)), np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)
    rs, cs = np.zeros(m), np.zeros(n)
    lib().orc_scale(n, m, _i(rp), _i(ci), _d(v), _d(c), _d(q), _d(lo), _d(hi), ruiz_iterations,
                    int(apply_pc), C.c_double(alpha), _d(sv), _d(sc), _d(sq), _d(sl), _d(su), _d(rs), _d(cs))
    return sv, sc, sq, sl, su, rs, cs


def csr_from_triplets(rows, cols, r, c, v):
    r = np.ascontiguousarray(r, dtype=np.int32)
    c = np.ascontiguousarray(c, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.float64)
    rp = np.zeros(rows + 1, dtype=np.int32)
    ci = np.zeros(max(len(r), 1), dtype=np.int32)
    vv = np.zeros(max(len(r), 1))
    nnz = lib().orc_csr_from_triplets(rows, cols, len(r), _i(r), _i(c), _d(v), _i(rp), _i(ci), _d(vv))
    if nnz < 0:
        raise ValueError("requirement failed: bad triplet")
    return rp, ci[:nnz].copy(), vv[:nnz].copy()


def csr_transpose(rows, cols, rp, ci, v):
    trp = np.zeros(cols + 1, dtype=np.int32)
    tci = np.zeros(max(len(ci), 1), dtype=np.int32)
    tv = np.zeros(max(len(ci), 1))
    lib().orc_csr_transpose(rows, cols, _i(rp), _i(ci), _d(v), _i(trp), _i(tci), _d(tv))
    return trp, tci[:len(ci)].copy(), tv[:len(ci)].copy()


def spectral_norm_bound(matrix) -> float:
    return lib().orc_csr_spectral_norm_bound(matrix.rows, matrix.cols, _i(matrix.row_ptr),
                                             _i(matrix.col_indices), _d(matrix.values))


class Ops:
    """The eight kernel-seam operations of ScalaKernels (FP64) or
    Float32Kernels (FP32) on host arrays (``Kernels.scala:42-125``)."""

    def __init__(self, mode: int):
        self.mode = mode

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        out = np.zeros(len(a))
        lib().orc_k_upload(self.mode, len(a), _d(a), _d(out))
        return out

    def spmv(self, matrix, x):
        vals = self.upload(matrix.values) if self.mode == FP32 else matrix.values
        out = np.zeros(matrix.rows)
        lib().orc_k_spmv(self.mode, matrix.rows, _i(matrix.row_ptr), _i(matrix.col_indices), _d(vals),
                         _d(np.ascontiguousarray(x, dtype=np.float64)), _d(out))
        return out

    def axpby(self, alpha, x, beta, y):
        out = np.zeros(len(x))
        lib().orc_k_axpby(self.mode, len(x), C.c_double(alpha), _d(np.ascontiguousarray(x)), C.c_double(beta),
                          _d(np.ascontiguousarray(y)), _d(out))
        return out

    def scale(self, alpha, x):
        out = np.zeros(len(x))
        lib().orc_k_scale(self.mode, len(x), C.c_double(alpha), _d(np.ascontiguousarray(x)), _d(out))
        return out

    def dot(self, x, y):
        return lib().orc_k_dot(self.mode, len(x), _d(np.ascontiguousarray(x)), _d(np.ascontiguousarray(y)))

    def squared_norm(self, x):
        return lib().orc_k_squared_norm(self.mode, len(x), _d(np.ascontiguousarray(x)))

    def primal_step(self, x, kty, c, l, u, tau):
        out = np.zeros(len(x))
        arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, kty, c, l, u)]
        lib().orc_k_primal_step(self.mode, len(x), *[_d(a) for a in arr], C.c_double(tau), _d(out))
        return out

    def dual_step(self, y, kxbar, q, sigma, neq):
        out = np.zeros(len(y))
        arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (y, kxbar, q)]
        lib().orc_k_dual_step(self.mode, len(y), *[_d(a) for a in arr], C.c_double(sigma), neq, _d(out))
        return out
