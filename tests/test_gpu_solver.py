"""The device-resident solve (prima_pdhg_solve through the C ABI) against the
oracle on the same seeded inputs: PdhgSuite (core/src/test/.../PdhgSuite.scala)
and the validation ladder, in FP64 (ScalaKernels semantics) and FP32
(Float32Kernels semantics).

Tolerances: status identical; objective within 1e-8 relative of the oracle's
FP64 answer at eps = 1e-9 (the ladder's worst-gap bound).  Iteration counts:
the device reduces in a fixed tree and evaluates pow/exp/log with CUDA's
libm, so its trajectory can differ from the oracle's in the last bit.  The
tiny fixtures, where neither can change a bit, must match exactly.  The
others are chaotic in the last bit -- the oracle itself moves by up to
several times when one objective coefficient moves by one ulp -- so their
count must lie within that spread (tests/golden/ladder_envelope.json, made by
make_ladder_envelope.py), widened by a quarter."""
import ctypes
import json
import math
import os

import numpy as np
import pytest

from noaidi_b200.prima import LpProblem, PdhgParams, ScalingParams, SolveStatus, WarmStart
from noaidi_b200.prima import generators as G
from oracle import oracle as O
from tests import lp_fixtures as F

pytestmark = pytest.mark.gpu

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))
ENVELOPE = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ladder_envelope.json")))
P9 = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=500_000)
LADDER = F.ladder()
EXACT = {"tiny-lower-bound", "product-mix", "equality-split", "degenerate", "free-sign", "range-row",
         "economic-dispatch", "unbounded"}


def gpu_solve(problem, params=P9, precision=64, **kw):
    from noaidi_b200.prima import cuda
    return cuda.solve(problem, params, precision=precision, **kw)


@pytest.mark.parametrize("entry", LADDER, ids=lambda e: e.name)
def test_ladder_fp64_matches_oracle(entry):
    ref = O.solve(entry.problem, P9)
    got = gpu_solve(entry.problem)
    assert got.status == ref.status == entry.expected
    if ref.status == SolveStatus.OPTIMAL:
        assert F.relative_gap(got.objective_value, ref.objective_value) <= 1e-8
        assert np.allclose(got.primal, ref.primal, atol=1e-5 * max(1.0, np.abs(ref.primal).max()))
    if entry.name in EXACT:
        assert (got.iterations, got.restarts) == (ref.iterations, ref.restarts)
    else:
        env = ENVELOPE[entry.name]
        lo, hi = min(env["perturbed"] + [ref.iterations]), max(env["perturbed"] + [ref.iterations])
        assert lo / 1.25 - 128 <= got.iterations <= hi * 1.25 + 128, (got.iterations, lo, hi)


@pytest.mark.parametrize("entry", LADDER[:10], ids=lambda e: e.name)
def test_ladder_fp32_matches_float32_oracle(entry):
    p = PdhgParams(eps_abs=1e-5, eps_rel=1e-5, max_iterations=200_000, infeasibility_tolerance=1e-5)
    ref = O.solve(entry.problem, p, mode=O.FP32)
    got = gpu_solve(entry.problem, p, precision=32)
    assert got.status == ref.status
    if ref.status == SolveStatus.OPTIMAL:
        assert F.relative_gap(got.objective_value, ref.objective_value) <= 1e-4


def test_known_optima_and_congestion_prices():
    for inst in F.optimal():
        s = gpu_solve(inst.problem)
        assert s.status == SolveStatus.OPTIMAL
        assert s.objective_value == pytest.approx(inst.expected_objective, abs=1e-6 * max(1.0, abs(inst.expected_objective)))
        for v, e in zip(s.primal, inst.expected_primal):
            assert v == pytest.approx(e, abs=1e-5)
        assert s.objective_value == pytest.approx(s.dual_objective_value, abs=1e-5 * max(1.0, abs(s.objective_value)))
    s = gpu_solve(F.economic_dispatch().problem)
    pin = PINS["fixtures"]["economic_dispatch_prices"]
    assert s.dual[0] == pytest.approx(s.dual[1], abs=1e-4)
    assert s.dual[2] == pytest.approx(pin["A2"], abs=pin["tolerance"])
    assert s.dual[3] == pytest.approx(pin["B2"], abs=pin["tolerance"])


def test_limits_trivial_and_statuses():
    capped = gpu_solve(F.economic_dispatch().problem, PdhgParams(eps_abs=1e-14, eps_rel=1e-14, max_iterations=3))
    assert capped.status == SolveStatus.ITERATION_LIMIT and capped.iterations == 3
    ref = O.solve(F.economic_dispatch().problem, PdhgParams(eps_abs=1e-14, eps_rel=1e-14, max_iterations=3))
    assert capped.objective_value == pytest.approx(ref.objective_value, rel=1e-12)
    b = LpProblem.builder(2)
    b.bounds(0, 0.0, 1.0).bounds(1, 0.0, 1.0)
    triv = gpu_solve(b.build()[0])
    assert triv.status == SolveStatus.OPTIMAL and triv.iterations == 0
    timed = PdhgParams(eps_abs=1e-16, eps_rel=1e-16, max_iterations=50_000_000, time_limit_millis=50)
    s = gpu_solve(F.random_feasible(5, 200, 40, 80), timed)
    assert s.status == SolveStatus.TIME_LIMIT and s.iterations < 50_000_000


def test_cancel_flag_is_polled_at_evaluation_points():
    flag = ctypes.c_int32(1)
    s = gpu_solve(F.random_feasible(5, 200, 40, 80), PdhgParams(eps_abs=1e-16, eps_rel=1e-16), cancel=flag)
    assert s.status == SolveStatus.INTERRUPTED and s.iterations == 64


def test_scaling_off_and_stability_bound():
    unscaled = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, scaling=ScalingParams.none())
    for inst in F.optimal():
        a, b = O.solve(inst.problem, unscaled), gpu_solve(inst.problem, unscaled)
        assert a.status == b.status == SolveStatus.OPTIMAL
        assert F.relative_gap(b.objective_value, a.objective_value) <= 1e-8
    b = LpProblem.builder(1)
    b.objective_coefficient(0, 1.0).bounds(0, 0.0, 10.0)
    for _ in range(100):
        b.greater_than([(0, 1.0)], 3.0)
    s = gpu_solve(b.build()[0])
    assert s.status == SolveStatus.OPTIMAL and s.objective_value == pytest.approx(3.0, abs=1e-6)


def test_warm_starts():
    p = F.economic_dispatch().problem
    cold = gpu_solve(p)
    warm = gpu_solve(p, warm_start=WarmStart.from_solution(cold))
    assert warm.status == SolveStatus.OPTIMAL and warm.iterations < cold.iterations
    ref = O.solve(p, P9, warm_start=WarmStart.from_solution(cold))
    assert (warm.iterations, warm.restarts) == (ref.iterations, ref.restarts)
    wild = WarmStart(np.array([1e6, -1e6]), np.array([-5.0]))
    s = gpu_solve(F.equality_split().problem, warm_start=wild)
    assert s.status == SolveStatus.OPTIMAL and s.objective_value == pytest.approx(24.0, abs=1e-6)
    with pytest.raises(ValueError):
        gpu_solve(F.equality_split().problem, warm_start=WarmStart(np.array([1.0]), np.array([0.0])))
    with pytest.raises(ValueError):
        gpu_solve(F.equality_split().problem, warm_start=WarmStart(np.array([math.nan, 1.0]), np.array([0.0])))


def test_invalid_arguments_are_rejected():
    """The C ABI re-validates everything (PdhgParams.scala:55-79,
    LpProblem.scala:62-104) and answers PRIMA_ERR_INVALID_ARGUMENT."""
    from noaidi_b200.prima import cuda
    ctx = cuda.context(0, 64)
    lpv = cuda._LpView(F.economic_dispatch().problem)
    info = cuda.CInfo()
    for field, bad in (("restart_artificial_fraction", 0.0), ("infeasibility_tolerance", -1e-9),
                       ("max_iterations", 0), ("primal_weight_smoothing", 1.5)):
        cp = cuda.to_c_params(P9)
        setattr(cp, field, bad)
        rc = ctx.lib.prima_pdhg_solve(ctx.handle, ctypes.byref(lpv.c), ctypes.byref(cp), None, None, None, None,
                                      None, ctypes.byref(info))
        assert rc == cuda.ERR_INVALID_ARGUMENT, field
    lpv.c.num_equalities = 99
    rc = ctx.lib.prima_pdhg_solve(ctx.handle, ctypes.byref(lpv.c), ctypes.byref(cuda.to_c_params(P9)), None, None,
                                  None, None, None, ctypes.byref(info))
    assert rc == cuda.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("precision,eps", [(64, 1e-8), (32, 1e-5)], ids=["fp64", "fp32"])
def test_lopf_matches_oracle(precision, eps):
    P = G.dc_lopf(seed=3, buses=120, lines=180, generators=60, snapshots=6)
    p = PdhgParams(eps_abs=eps, eps_rel=eps, max_iterations=400_000)
    ref = O.solve(P, p, mode=O.FP64 if precision == 64 else O.FP32)
    got = gpu_solve(P, p, precision=precision)
    assert got.status == ref.status == SolveStatus.OPTIMAL
    assert F.relative_gap(got.objective_value, ref.objective_value) <= (1e-8 if precision == 64 else 1e-4)
    assert got.kkt.primal_residual_norm <= eps + eps * np.linalg.norm(P.rhs)
    assert got.kkt.dual_residual_norm <= eps + eps * np.linalg.norm(P.objective)


def test_random_sparse_lp_600_columns():
    P = G.random_sparse_lp(0)
    p = PdhgParams(eps_abs=1e-6, eps_rel=1e-6, max_iterations=400_000)
    ref, got = O.solve(P, p), gpu_solve(P, p)
    assert got.status == ref.status == SolveStatus.OPTIMAL
    assert F.relative_gap(got.objective_value, ref.objective_value) <= 1e-5


def test_long_rows_take_the_warp_path_and_match_the_oracle():
    """A row and a column far denser than a tile stage holds (a budget row over
    every variable, a variable in every row) go through the warp-per-row path;
    the sums stay in index order, so the solve matches the oracle as any other."""
    rng = np.random.default_rng(8)
    n, m = 3000, 2600
    rows, cols, vals = [], [], []
    for r in range(m - 1):  # sparse rows, plus column 0 in every row
        cs = np.unique(np.concatenate([[0], rng.choice(n, 4, replace=False)]))
        rows += [r] * len(cs)
        cols += cs.tolist()
        vals += rng.uniform(0.5, 1.5, len(cs)).tolist()
    rows += [m - 1] * n  # the dense budget row
    cols += list(range(n))
    vals += [1.0] * n
    from noaidi_b200.prima import SparseMatrix
    K = SparseMatrix.from_triplets(m, n, rows, cols, vals)
    x0 = rng.uniform(0.0, 1.0, n)
    q = K.multiply(x0) - rng.uniform(0.0, 0.5, m)
    c = rng.uniform(-1.0, 1.0, n)
    P = LpProblem(c, K, q, 0, np.zeros(n), np.full(n, 2.0))
    p = PdhgParams(eps_abs=1e-7, eps_rel=1e-7, max_iterations=200_000)
    ref = O.solve(P, p)
    for prec in (64, 32):
        got = gpu_solve(P, p, precision=prec)
        assert got.status == ref.status == SolveStatus.OPTIMAL
        assert F.relative_gap(got.objective_value, ref.objective_value) <= (1e-6 if prec == 64 else 1e-4)


def test_an_allocation_the_device_cannot_hold_fails_cleanly():
    """Fault injection on the host side: a 1 TiB vector cannot be allocated,
    which answers PRIMA_ERR_OUT_OF_MEMORY, and the context stays usable --
    the next operations and a whole solve succeed."""
    from noaidi_b200.prima import cuda
    ctx = cuda.Context(0, 64)
    try:
        h = ctypes.c_int64()
        assert ctx.lib.prima_vec_alloc(ctx.handle, 1 << 37, ctypes.byref(h)) == cuda.ERR_OUT_OF_MEMORY
        assert b"cudaMalloc" in ctx.lib.prima_last_error()
        ok = ctypes.c_int64()
        assert ctx.lib.prima_vec_alloc(ctx.handle, 1000, ctypes.byref(ok)) == cuda.OK
        p = F.economic_dispatch().problem
        s = cuda.solve(p, P9, ctx=ctx)
        assert s.status == SolveStatus.OPTIMAL and s.objective_value == pytest.approx(3700.0, rel=1e-8)
    finally:
        ctx.close()
