"""ctypes binding of ``libprima_cuda.so`` (declared in ``include/prima_cuda.h``).

* :class:`CudaKernels` -- the ``Kernels`` seam (``Kernels.scala:42-125``) on a
  B200: the eight numeric operations over device-resident vectors.
* :func:`solve` -- ``Pdhg.solveWith`` (``Pdhg.scala:48-55``) with the whole
  iteration on the device (one persistent launch).
* :func:`mixed_solve` -- ``MixedPrecision.solve`` (``MixedPrecision.scala:104-199``)
  with both passes on the device.
* :func:`solve_batch` -- ``PrimaZio.solveAll``'s shape in one launch, and
  :func:`solve_labelled` -- ``solveLabelled``'s.

There is no CPU fallback: if the library is missing or no sm_100 device is
present these raise.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import threading
from typing import Optional, Sequence

import numpy as np

from .model import LpProblem, SparseMatrix
from .types import (KktError, LpSolution, MixedPrecisionParams, MixedPrecisionResult, PdhgParams, SolveStatus,
                    WarmStart)

# The in-tree build; PRIMA_CUDA_LIBRARY names another build of the same ABI
# (a differently tuned compile of the same sources, say).
LIB_PATH = os.environ.get("PRIMA_CUDA_LIBRARY") or \
    os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "libprima_cuda.so")

OK, ERR_INVALID_ARGUMENT, ERR_OUT_OF_MEMORY, ERR_CUDA, ERR_TIMEOUT, ERR_CLOSED, ERR_NO_DEVICE, ERR_PARSE = range(8)
MIXED_TWO_PASS, MIXED_REFINEMENT = 0, 1


class PrimaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Capabilities(C.Structure):
    _fields_ = [("name", C.c_char * 64), ("device", C.c_char * 128), ("supports_float64", C.c_int32),
                ("precision_bits", C.c_int32)]


class CLp(C.Structure):
    _fields_ = [("num_variables", C.c_int32), ("num_constraints", C.c_int32), ("num_equalities", C.c_int32),
                ("pad", C.c_int32), ("row_ptr", C.POINTER(C.c_int32)), ("col_idx", C.POINTER(C.c_int32)),
                ("values", C.POINTER(C.c_double)), ("objective", C.POINTER(C.c_double)),
                ("rhs", C.POINTER(C.c_double)), ("lower", C.POINTER(C.c_double)),
                ("upper", C.POINTER(C.c_double)), ("objective_offset", C.c_double)]


class CParams(C.Structure):
    _fields_ = [("eps_abs", C.c_double), ("eps_rel", C.c_double), ("max_iterations", C.c_int32),
                ("evaluation_frequency", C.c_int32), ("time_limit_ms", C.c_double),
                ("ruiz_iterations", C.c_int32), ("apply_pock_chambolle", C.c_int32),
                ("pock_chambolle_alpha", C.c_double), ("infeasibility_tolerance", C.c_double),
                ("restart_sufficient_reduction", C.c_double), ("restart_necessary_reduction", C.c_double),
                ("restart_artificial_fraction", C.c_double), ("primal_weight_smoothing", C.c_double)]


class CWarm(C.Structure):
    _fields_ = [("primal", C.POINTER(C.c_double)), ("dual", C.POINTER(C.c_double)), ("step_size", C.c_double),
                ("primal_weight", C.c_double)]


class CInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32),
                ("device_error", C.c_int32), ("solve_ms", C.c_int64), ("objective", C.c_double),
                ("dual_objective", C.c_double), ("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("final_step_size", C.c_double), ("final_primal_weight", C.c_double), ("device_ms", C.c_double),
                ("setup_ms", C.c_double), ("trials", C.c_int64), ("span_ms", C.c_double), ("blocks", C.c_int32),
                ("tile_rows", C.c_int32)]


class CMixedParams(C.Structure):
    _fields_ = [("reduced_tolerance", C.c_double), ("reduced_max_iterations", C.c_int32),
                ("always_refine", C.c_int32), ("reduced_time_share", C.c_double), ("scheme", C.c_int32),
                ("pad", C.c_int32), ("round_reduction", C.c_double)]


class CMixedInfo(C.Structure):
    _fields_ = [("reduced_iterations", C.c_int32), ("reduced_restarts", C.c_int32), ("reduced_ms", C.c_int64),
                ("refinement_iterations", C.c_int32), ("refined", C.c_int32), ("refinement_ms", C.c_int64),
                ("refinement_rounds", C.c_int32), ("pad", C.c_int32)]


class CMpsInfo(C.Structure):
    _fields_ = [("num_variables", C.c_int32), ("num_constraints", C.c_int32), ("num_equalities", C.c_int32),
                ("num_rows", C.c_int32), ("nnz", C.c_int64), ("num_integer_columns", C.c_int32), ("pad", C.c_int32)]


class CPresolveInfo(C.Structure):
    _fields_ = [("fixed_columns", C.c_int32), ("empty_columns", C.c_int32), ("empty_rows", C.c_int32),
                ("singleton_rows", C.c_int32), ("proven_infeasible", C.c_int32),
                ("unbounded_if_feasible", C.c_int32), ("passes", C.c_int32), ("reduced_variables", C.c_int32),
                ("reduced_constraints", C.c_int32), ("reduced_equalities", C.c_int32), ("reduced_nnz", C.c_int64)]


# Every exported symbol with its ctypes signature; the ABI test checks this
# list against include/*.h.
_H = C.c_int64
_HP = C.POINTER(C.c_int64)
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)
SIGNATURES = {
    "prima_last_error": (C.c_char_p, []),
    "prima_open": (C.c_int32, [C.c_int32, C.c_int32, _HP]),
    "prima_close": (C.c_int32, [_H]),
    "prima_capabilities_get": (C.c_int32, [_H, C.POINTER(Capabilities)]),
    "prima_set_device_wait_limit": (C.c_int32, [_H, C.c_int64]),
    "prima_set_solver_layout": (C.c_int32, [_H, C.c_int32, C.c_int32]),
    "prima_vec_alloc": (C.c_int32, [_H, C.c_int64, _HP]),
    "prima_vec_upload": (C.c_int32, [_H, _DP, C.c_int64, _HP]),
    "prima_vec_download": (C.c_int32, [_H, _H, _DP, C.c_int64]),
    "prima_vec_length": (C.c_int32, [_H, _H, C.POINTER(C.c_int64)]),
    "prima_vec_free": (C.c_int32, [_H, _H]),
    "prima_mat_upload_csr": (C.c_int32, [_H, C.c_int32, C.c_int32, _IP, _IP, _DP, _HP]),
    "prima_spmv": (C.c_int32, [_H, _H, _H, _H]),
    "prima_axpby": (C.c_int32, [_H, C.c_double, _H, C.c_double, _H, _H]),
    "prima_scale": (C.c_int32, [_H, C.c_double, _H, _H]),
    "prima_copy": (C.c_int32, [_H, _H, _H]),
    "prima_dot": (C.c_int32, [_H, _H, _H, _DP]),
    "prima_squared_norm": (C.c_int32, [_H, _H, _DP]),
    "prima_dot_no_alloc": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]),
    "prima_primal_step": (C.c_int32, [_H, _H, _H, _H, _H, _H, C.c_double, _H]),
    "prima_dual_step": (C.c_int32, [_H, _H, _H, _H, C.c_double, C.c_int32, _H]),
    "prima_params_default": (None, [C.POINTER(CParams)]),
    "prima_mixed_params_default": (None, [C.POINTER(CMixedParams)]),
    "prima_pdhg_solve": (C.c_int32, [_H, C.POINTER(CLp), C.POINTER(CParams), C.POINTER(CWarm), _IP, _DP, _DP,
                                     _DP, C.POINTER(CInfo)]),
    "prima_mixed_solve": (C.c_int32, [_H, C.POINTER(CLp), C.POINTER(CParams), C.POINTER(CMixedParams), _IP,
                                      _DP, _DP, _DP, C.POINTER(CInfo), C.POINTER(CMixedInfo)]),
    "prima_pdhg_solve_batch": (C.c_int32, [_H, C.c_int32, C.POINTER(CLp), C.POINTER(CParams), _IP,
                                           C.POINTER(_DP), C.POINTER(_DP), C.POINTER(_DP), C.POINTER(CInfo)]),
    "prima_mixed_solve_batch": (C.c_int32, [_H, C.c_int32, C.POINTER(CLp), C.POINTER(CParams),
                                            C.POINTER(CMixedParams), _IP, C.POINTER(_DP), C.POINTER(_DP),
                                            C.POINTER(_DP), C.POINTER(CInfo), C.POINTER(CMixedInfo)]),
    "prima_problem_create": (C.c_int32, [_H, C.POINTER(CLp), C.POINTER(CParams), _HP]),
    "prima_problem_free": (C.c_int32, [_H, _H]),
    "prima_problem_set_bounds": (C.c_int32, [_H, _H, _DP, _DP]),
    "prima_problem_scaled": (C.c_int32, [_H, _H, _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
    "prima_problem_solve": (C.c_int32, [_H, _H, C.POINTER(CParams), C.POINTER(CWarm), _IP, _DP, _DP, _DP,
                                        C.POINTER(CInfo)]),
    "prima_problem_mixed_solve": (C.c_int32, [_H, _H, C.POINTER(CParams), C.POINTER(CMixedParams), _IP, _DP, _DP,
                                              _DP, C.POINTER(CInfo), C.POINTER(CMixedInfo)]),
    # the host model layer (include/prima_model.h)
    "prima_mps_read": (C.c_int32, [C.c_char_p, C.c_int64, C.c_char_p, C.POINTER(C.c_void_p)]),
    "prima_mps_read_file": (C.c_int32, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "prima_mps_free": (None, [C.c_void_p]),
    "prima_mps_get_info": (C.c_int32, [C.c_void_p, C.POINTER(CMpsInfo)]),
    "prima_mps_get_problem": (C.c_int32, [C.c_void_p, C.POINTER(CLp)]),
    "prima_mps_get_translation": (C.c_int32, [C.c_void_p, _IP, _IP, _IP]),
    "prima_mps_name": (C.c_char_p, [C.c_void_p]),
    "prima_mps_row_name": (C.c_char_p, [C.c_void_p, C.c_int32]),
    "prima_mps_column_name": (C.c_char_p, [C.c_void_p, C.c_int32]),
    "prima_mps_get_integer_columns": (C.c_int32, [C.c_void_p, _IP]),
    "prima_presolve": (C.c_int32, [C.POINTER(CLp), C.c_int32, C.POINTER(C.c_void_p)]),
    "prima_presolve_free": (None, [C.c_void_p]),
    "prima_presolve_get_info": (C.c_int32, [C.c_void_p, C.POINTER(CPresolveInfo)]),
    "prima_presolve_get_reduced": (C.c_int32, [C.c_void_p, C.POINTER(CLp)]),
    "prima_presolve_get_maps": (C.c_int32, [C.c_void_p, _IP, _IP]),
    "prima_presolve_restore": (C.c_int32, [C.c_void_p, _DP, _DP, _DP, _DP, _DP, _DP]),
}

_lib = None
_lib_lock = threading.Lock()


def library():
    """Load ``libprima_cuda.so`` (never a fallback: a missing library raises)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise PrimaError(ERR_NO_DEVICE, f"{LIB_PATH} is missing; build it with `python -m noaidi_b200.build`")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def _check(code: int) -> None:
    if code != OK:
        msg = library().prima_last_error().decode()
        if code == ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        raise PrimaError(code, msg)


def _dp(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_DP)


def _ip(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_IP)


def to_c_params(p: PdhgParams) -> CParams:
    return CParams(p.eps_abs, p.eps_rel, p.max_iterations, p.evaluation_frequency,
                   -1.0 if p.time_limit_millis is None else float(p.time_limit_millis),
                   p.scaling.ruiz_iterations, int(p.scaling.apply_pock_chambolle), p.scaling.pock_chambolle_alpha,
                   p.infeasibility_tolerance, p.restart_sufficient_reduction, p.restart_necessary_reduction,
                   p.restart_artificial_fraction, p.primal_weight_smoothing)


def lp_from_view(v: CLp) -> LpProblem:
    """An LpProblem copied out of a prima_lp view the library owns."""
    n, m = v.num_variables, v.num_constraints

    def arr(ptr, k, dtype):
        return np.ctypeslib.as_array(ptr, shape=(k,)).astype(dtype, copy=True) if k else np.zeros(0, dtype)

    rp = arr(v.row_ptr, m + 1, np.int32)
    nnz = int(rp[-1])
    K = SparseMatrix(m, n, rp, arr(v.col_idx, nnz, np.int32), arr(v.values, nnz, np.float64))
    return LpProblem(arr(v.objective, n, np.float64), K, arr(v.rhs, m, np.float64), v.num_equalities,
                     arr(v.lower, n, np.float64), arr(v.upper, n, np.float64), v.objective_offset)


class _LpView:
    """A prima_lp over a problem's arrays (kept alive by this object)."""

    def __init__(self, problem: LpProblem):
        K = problem.constraint_matrix
        self._keep = (np.ascontiguousarray(K.row_ptr, np.int32), np.ascontiguousarray(K.col_indices, np.int32),
                      np.ascontiguousarray(K.values, np.float64), np.ascontiguousarray(problem.objective),
                      np.ascontiguousarray(problem.rhs), np.ascontiguousarray(problem.variable_lower),
                      np.ascontiguousarray(problem.variable_upper))
        rp, ci, v, c, q, lo, hi = self._keep
        self.c = CLp(problem.num_variables, problem.num_constraints, problem.num_equalities, 0, _ip(rp), _ip(ci),
                     _dp(v), _dp(c), _dp(q), _dp(lo), _dp(hi), problem.objective_offset)


class Context:
    """An open ``libprima_cuda`` context (a ``Kernels`` instance's device state)."""

    def __init__(self, device: int = 0, precision: int = 64):
        self.lib = library()
        h = C.c_int64()
        _check(self.lib.prima_open(device, precision, C.byref(h)))
        self.handle = h.value
        self.precision = precision
        self._closed = False

    def close(self) -> None:
        if not self._closed:
            _check(self.lib.prima_close(self.handle))
            self._closed = True

    def set_solver_layout(self, blocks_per_sm: int = 0, tile_rows: int = 0) -> None:
        """Pin the persistent solver's layout (``prima_set_solver_layout``);
        (0, 0) restores the choice by timing."""
        _check(self.lib.prima_set_solver_layout(self.handle, blocks_per_sm, tile_rows))

    def set_device_wait_limit(self, polls: int) -> None:
        """Team-barrier polls before a block of a solve gives up
        (``prima_set_device_wait_limit``); 0 restores the default."""
        _check(self.lib.prima_set_device_wait_limit(self.handle, polls))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CudaKernels:
    """``Kernels`` on a B200 (``Kernels.scala:42-125``).  ``precision=64`` has
    ScalaKernels semantics, ``precision=32`` Float32Kernels semantics.
    Vectors and matrices are integer handles owned by the context."""

    def __init__(self, device: int = 0, precision: int = 64):
        self.ctx = Context(device, precision)
        self.lib = self.ctx.lib
        self.h = self.ctx.handle

    # capabilities ------------------------------------------------------------
    @property
    def capabilities(self):
        caps = Capabilities()
        _check(self.lib.prima_capabilities_get(self.h, C.byref(caps)))
        return _Caps(caps.name.decode(), caps.device.decode(), bool(caps.supports_float64))

    # memory --------------------------------------------------------------------
    def allocate(self, n: int) -> int:
        v = C.c_int64()
        _check(self.lib.prima_vec_alloc(self.h, n, C.byref(v)))
        return v.value

    def upload(self, data) -> int:
        a = np.ascontiguousarray(data, dtype=np.float64)
        v = C.c_int64()
        _check(self.lib.prima_vec_upload(self.h, _dp(a), a.shape[0], C.byref(v)))
        return v.value

    def download(self, v: int, into: np.ndarray) -> None:
        if into.dtype != np.float64 or not into.flags.c_contiguous:
            raise ValueError("download target must be a contiguous float64 array")
        _check(self.lib.prima_vec_download(self.h, v, _dp(into), into.shape[0]))

    def upload_matrix(self, m: SparseMatrix) -> int:
        h = C.c_int64()
        rp = np.ascontiguousarray(m.row_ptr, np.int32)
        ci = np.ascontiguousarray(m.col_indices, np.int32)
        vv = np.ascontiguousarray(m.values, np.float64)
        _check(self.lib.prima_mat_upload_csr(self.h, m.rows, m.cols, _ip(rp), _ip(ci), _dp(vv), C.byref(h)))
        return h.value

    def length(self, v: int) -> int:
        n = C.c_int64()
        _check(self.lib.prima_vec_length(self.h, v, C.byref(n)))
        return n.value

    def close(self) -> None:
        self.ctx.close()

    # numerics ------------------------------------------------------------------
    def spmv(self, a: int, x: int, out: int) -> None:
        _check(self.lib.prima_spmv(self.h, a, x, out))

    def axpby(self, alpha: float, x: int, beta: float, y: int, out: int) -> None:
        _check(self.lib.prima_axpby(self.h, alpha, x, beta, y, out))

    def scale(self, alpha: float, x: int, out: int) -> None:
        _check(self.lib.prima_scale(self.h, alpha, x, out))

    def copy(self, src: int, dst: int) -> None:
        _check(self.lib.prima_copy(self.h, src, dst))

    def dot(self, x: int, y: int) -> float:
        out = C.c_double()
        _check(self.lib.prima_dot(self.h, x, y, C.byref(out)))
        return out.value

    def squared_norm(self, x: int) -> float:
        out = C.c_double()
        _check(self.lib.prima_squared_norm(self.h, x, C.byref(out)))
        return out.value

    def primal_step(self, x: int, kty: int, cost: int, lower: int, upper: int, tau: float, out: int) -> None:
        _check(self.lib.prima_primal_step(self.h, x, kty, cost, lower, upper, tau, out))

    def dual_step(self, y: int, kxbar: int, rhs: int, sigma: float, num_equalities: int, out: int) -> None:
        _check(self.lib.prima_dual_step(self.h, y, kxbar, rhs, sigma, num_equalities, out))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class _Caps:
    def __init__(self, name: str, device: str, supports_float64: bool):
        self.name, self.device, self.supports_float64 = name, device, supports_float64

    @property
    def requires_double_precision_refinement(self) -> bool:
        return not self.supports_float64


def _solution(info: CInfo, x, y, rc) -> LpSolution:
    sol = LpSolution(SolveStatus(info.status), x, y, rc, info.objective, info.dual_objective, info.iterations,
                     info.restarts, int(info.solve_ms),
                     KktError(info.primal_residual, info.dual_residual, info.objective, info.dual_objective),
                     info.final_step_size, info.final_primal_weight)
    sol.device_ms = info.device_ms
    sol.setup_ms = info.setup_ms
    sol.trials = info.trials
    sol.span_ms = info.span_ms
    sol.blocks = info.blocks
    sol.tile_rows = info.tile_rows
    return sol


def _warm(problem: LpProblem, ws: Optional[WarmStart]):
    if ws is None:
        return None, None
    n, m = problem.num_variables, problem.num_constraints
    if len(ws.primal) != n:
        raise ValueError(f"requirement failed: warm start has {len(ws.primal)} primal entries, expected {n}")
    if len(ws.dual) != m:
        raise ValueError(f"requirement failed: warm start has {len(ws.dual)} dual entries, expected {m}")
    px = np.ascontiguousarray(ws.primal, dtype=np.float64)
    py = np.ascontiguousarray(ws.dual, dtype=np.float64)
    w = CWarm(_dp(px), _dp(py), math.nan if ws.step_size is None else ws.step_size,
              math.nan if ws.primal_weight is None else ws.primal_weight)
    return w, (px, py)


_ctx_cache: dict = {}
_ctx_lock = threading.Lock()


def context(device: int = 0, precision: int = 64) -> Context:
    """A per-thread cached context (contexts are not thread-safe)."""
    key = (threading.get_ident(), device, precision)
    with _ctx_lock:
        ctx = _ctx_cache.get(key)
        if ctx is None or ctx._closed:
            ctx = Context(device, precision)
            _ctx_cache[key] = ctx
    return ctx


def solve(problem: LpProblem, params: PdhgParams = PdhgParams(), precision: int = 64,
          warm_start: Optional[WarmStart] = None, cancel: Optional[C.c_int32] = None, device: int = 0,
          ctx: Optional[Context] = None) -> LpSolution:
    """``Pdhg.solveWith`` with the iteration resident on the GPU."""
    ctx = ctx or context(device, precision)
    lpv = _LpView(problem)
    n, m = problem.num_variables, problem.num_constraints
    x, y, rc = np.zeros(n), np.zeros(m), np.zeros(n)
    warm, keep = _warm(problem, warm_start)
    info = CInfo()
    cp = to_c_params(params)
    _check(ctx.lib.prima_pdhg_solve(ctx.handle, C.byref(lpv.c), C.byref(cp), None if warm is None else C.byref(warm),
                                    None if cancel is None else C.cast(C.byref(cancel), _IP), _dp(x), _dp(y),
                                    _dp(rc), C.byref(info)))
    return _solution(info, x, y, rc)


def to_c_mixed(mixed: MixedPrecisionParams, scheme: int = MIXED_REFINEMENT, round_reduction: float = 0.0) -> CMixedParams:
    return CMixedParams(mixed.reduced_tolerance, mixed.reduced_max_iterations, int(mixed.always_refine),
                        mixed.reduced_time_share, scheme, 0, round_reduction)


DEFAULT_SCHEME = MIXED_REFINEMENT


def mixed_solve(problem: LpProblem, params: PdhgParams = PdhgParams(),
                mixed: MixedPrecisionParams = MixedPrecisionParams(), scheme: int = None,
                cancel: Optional[C.c_int32] = None, device: int = 0, round_reduction: float = 0.0,
                ctx: Optional[Context] = None) -> MixedPrecisionResult:
    """``MixedPrecision.solve`` with both passes on the GPU."""
    scheme = DEFAULT_SCHEME if scheme is None else scheme
    ctx = ctx or context(device, 32)
    lpv = _LpView(problem)
    n, m = problem.num_variables, problem.num_constraints
    x, y, rc = np.zeros(n), np.zeros(m), np.zeros(n)
    info, minfo = CInfo(), CMixedInfo()
    cp = to_c_params(params)
    mp = to_c_mixed(mixed, scheme, round_reduction)
    _check(ctx.lib.prima_mixed_solve(ctx.handle, C.byref(lpv.c), C.byref(cp), C.byref(mp),
                                     None if cancel is None else C.cast(C.byref(cancel), _IP), _dp(x), _dp(y),
                                     _dp(rc), C.byref(info), C.byref(minfo)))
    res = MixedPrecisionResult(_solution(info, x, y, rc), minfo.reduced_iterations, minfo.reduced_restarts,
                               int(minfo.reduced_ms), minfo.refinement_iterations, int(minfo.refinement_ms),
                               bool(minfo.refined), minfo.refinement_rounds)
    return res


def mixed_solve_batch(problems: Sequence[LpProblem], params: PdhgParams = PdhgParams(),
                      mixed: MixedPrecisionParams = MixedPrecisionParams(), scheme: int = None,
                      round_reduction: float = 0.0, cancel: Optional[C.c_int32] = None, device: int = 0,
                      ctx: Optional[Context] = None) -> list[MixedPrecisionResult]:
    """``mixed_solve`` for many independent LPs, each pass one device launch
    for all of them."""
    scheme = DEFAULT_SCHEME if scheme is None else scheme
    ctx = ctx or context(device, 32)
    k = len(problems)
    views = [_LpView(p) for p in problems]
    arr = (CLp * k)(*[v.c for v in views])
    xs = [np.zeros(p.num_variables) for p in problems]
    ys = [np.zeros(p.num_constraints) for p in problems]
    rcs = [np.zeros(p.num_variables) for p in problems]
    px = (_DP * k)(*[_dp(a) for a in xs])
    py = (_DP * k)(*[_dp(a) for a in ys])
    prc = (_DP * k)(*[_dp(a) for a in rcs])
    infos, minfos = (CInfo * k)(), (CMixedInfo * k)()
    cp = to_c_params(params)
    mp = to_c_mixed(mixed, scheme, round_reduction)
    _check(ctx.lib.prima_mixed_solve_batch(ctx.handle, k, arr, C.byref(cp), C.byref(mp),
                                           None if cancel is None else C.cast(C.byref(cancel), _IP), px, py, prc,
                                           infos, minfos))
    out = []
    for i in range(k):
        mi = minfos[i]
        out.append(MixedPrecisionResult(_solution(infos[i], xs[i], ys[i], rcs[i]), mi.reduced_iterations,
                                        mi.reduced_restarts, int(mi.reduced_ms), mi.refinement_iterations,
                                        int(mi.refinement_ms), bool(mi.refined), mi.refinement_rounds))
    return out


class DeviceProblem:
    """An LP uploaded and equilibrated once on the device (``prima_problem_*``),
    then solved any number of times.  ``solve``/``mixed_solve`` with
    ``want_solution=False`` leave the solution vectors on the device and
    return only the scalars (status, objective, KKT, iterations)."""

    def __init__(self, problem: LpProblem, params: PdhgParams = PdhgParams(), ctx: Optional[Context] = None,
                 device: int = 0, precision: int = 64):
        self.ctx = ctx or context(device, precision)
        self.problem = problem
        lpv = _LpView(problem)
        h = C.c_int64()
        _check(self.ctx.lib.prima_problem_create(self.ctx.handle, C.byref(lpv.c), C.byref(to_c_params(params)),
                                                 C.byref(h)))
        self.handle = h.value

    def _outs(self, want):
        n, m = self.problem.num_variables, self.problem.num_constraints
        if want:
            return np.zeros(n), np.zeros(m), np.zeros(n)
        return None, None, None

    def solve(self, params: PdhgParams = PdhgParams(), warm_start: Optional[WarmStart] = None,
              cancel: Optional[C.c_int32] = None, want_solution: bool = True) -> LpSolution:
        x, y, rc = self._outs(want_solution)
        warm, keep = _warm(self.problem, warm_start)
        info = CInfo()
        _check(self.ctx.lib.prima_problem_solve(self.ctx.handle, self.handle, C.byref(to_c_params(params)),
                                                None if warm is None else C.byref(warm),
                                                None if cancel is None else C.cast(C.byref(cancel), _IP), _dp(x),
                                                _dp(y), _dp(rc), C.byref(info)))
        return _solution(info, x, y, rc)

    def set_bounds(self, lower, upper) -> None:
        """New variable bounds for the resident problem (``prima_problem_set_bounds``);
        the upload and the equilibration are kept."""
        lo = np.ascontiguousarray(lower, dtype=np.float64)
        hi = np.ascontiguousarray(upper, dtype=np.float64)
        n = self.problem.num_variables
        if lo.shape != (n,) or hi.shape != (n,):
            raise ValueError(f"requirement failed: bounds must have {n} entries")
        _check(self.ctx.lib.prima_problem_set_bounds(self.ctx.handle, self.handle, _dp(lo), _dp(hi)))
        p = self.problem
        self.problem = LpProblem(p.objective, p.constraint_matrix, p.rhs, p.num_equalities, lo, hi,
                                 p.objective_offset)

    def mixed_solve(self, params: PdhgParams = PdhgParams(), mixed: MixedPrecisionParams = MixedPrecisionParams(),
                    scheme: int = None, cancel: Optional[C.c_int32] = None, want_solution: bool = True,
                    round_reduction: float = 0.0) -> MixedPrecisionResult:
        scheme = DEFAULT_SCHEME if scheme is None else scheme
        x, y, rc = self._outs(want_solution)
        info, minfo = CInfo(), CMixedInfo()
        mp = to_c_mixed(mixed, scheme, round_reduction)
        _check(self.ctx.lib.prima_problem_mixed_solve(self.ctx.handle, self.handle, C.byref(to_c_params(params)),
                                                      C.byref(mp),
                                                      None if cancel is None else C.cast(C.byref(cancel), _IP),
                                                      _dp(x), _dp(y), _dp(rc), C.byref(info), C.byref(minfo)))
        return MixedPrecisionResult(_solution(info, x, y, rc), minfo.reduced_iterations, minfo.reduced_restarts,
                                    int(minfo.reduced_ms), minfo.refinement_iterations, int(minfo.refinement_ms),
                                    bool(minfo.refined), minfo.refinement_rounds)

    def scaled(self):
        """The device's equilibration of this problem (``prima_problem_scaled``):
        (values in CSR order, objective, rhs, lower, upper, row scale, column
        scale), all float64."""
        p = self.problem
        n, m, nnz = p.num_variables, p.num_constraints, p.constraint_matrix.nnz
        out = (np.zeros(nnz), np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n), np.zeros(m), np.zeros(n))
        _check(self.ctx.lib.prima_problem_scaled(self.ctx.handle, self.handle, *[_dp(a) for a in out]))
        return out

    def free(self) -> None:
        if self.handle is not None and not self.ctx._closed:
            _check(self.ctx.lib.prima_problem_free(self.ctx.handle, self.handle))
        self.handle = None


def solve_labelled(labelled: Sequence[tuple], params: PdhgParams = PdhgParams(), **kw) -> list[tuple]:
    """``PrimaZio.solveLabelled`` (PrimaZio.scala:68-76): every (label,
    problem) solved in one device launch, each result kept with its label,
    in order."""
    labels = [label for label, _ in labelled]
    return list(zip(labels, solve_batch([p for _, p in labelled], params, **kw)))


def solve_batch(problems: Sequence[LpProblem], params: PdhgParams = PdhgParams(), precision: int = 64,
                cancel: Optional[C.c_int32] = None, device: int = 0,
                ctx: Optional[Context] = None) -> list[LpSolution]:
    """``PrimaZio.solveAll``'s shape: every problem in one device launch."""
    ctx = ctx or context(device, precision)
    views = [_LpView(p) for p in problems]
    arr = (CLp * len(problems))(*[v.c for v in views])
    xs = [np.zeros(p.num_variables) for p in problems]
    ys = [np.zeros(p.num_constraints) for p in problems]
    rcs = [np.zeros(p.num_variables) for p in problems]
    px = (_DP * len(problems))(*[_dp(a) for a in xs])
    py = (_DP * len(problems))(*[_dp(a) for a in ys])
    prc = (_DP * len(problems))(*[_dp(a) for a in rcs])
    infos = (CInfo * len(problems))()
    cp = to_c_params(params)
    _check(ctx.lib.prima_pdhg_solve_batch(ctx.handle, len(problems), arr, C.byref(cp),
                                          None if cancel is None else C.cast(C.byref(cancel), _IP), px, py, prc,
                                          infos))
    return [_solution(infos[i], xs[i], ys[i], rcs[i]) for i in range(len(problems))]
