"""prima_pdhg_solve_batch: PrimaZio.solveAll's shape (modules/prima-zio/.../
PrimaZio.scala:61-66) -- many independent LPs -- in one persistent launch.

Each instance must come out as its own solve would: a batch of small LPs
(one block per team, as a single solve of each uses) reproduces every single
solve bit for bit; a batch of uneven LOPF instances matches the oracle's
statuses and objectives within 1e-8 relative at eps = 1e-9, like single
solves do."""
import numpy as np
import pytest

from noaidi_b200.prima import PdhgParams, SolveStatus
from noaidi_b200.prima import generators as G
from oracle import oracle as O
from tests import lp_fixtures as F

pytestmark = pytest.mark.gpu

P9 = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=200_000)


def cuda():
    from noaidi_b200.prima import cuda as C
    return C


@pytest.mark.parametrize("precision", [64, 32])
def test_small_batch_reproduces_single_solves(precision):
    insts = [i.problem for i in F.conclusive()] + [F.random_feasible(1, 60, 10, 20, 0.25)]
    batch = cuda().solve_batch(insts, P9, precision=precision)
    for p, got in zip(insts, batch):
        one = cuda().solve(p, P9, precision=precision)
        assert got.status == one.status
        assert (got.iterations, got.restarts) == (one.iterations, one.restarts)
        assert got.objective_value == one.objective_value or (np.isnan(got.objective_value) and np.isnan(one.objective_value))
        np.testing.assert_array_equal(got.primal, one.primal)
        np.testing.assert_array_equal(got.dual, one.dual)


def test_uneven_lopf_batch_matches_oracle():
    p = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=400_000)
    rng = np.random.default_rng(3)
    insts = []
    for k in range(6):
        b = int(rng.integers(40, 160))
        insts.append(G.dc_lopf(seed=10 + k, buses=b, lines=3 * b // 2, generators=b // 2,
                               snapshots=int(rng.integers(2, 6)), load_scale=float(rng.uniform(0.6, 0.95))))
    insts += [F.infeasible().problem, F.unbounded().problem, F.product_mix().problem]
    batch = cuda().solve_batch(insts, p)
    for prob, got in zip(insts, batch):
        ref = O.solve(prob, p)
        assert got.status == ref.status
        if ref.status == SolveStatus.OPTIMAL:
            assert F.relative_gap(got.objective_value, ref.objective_value) <= 1e-8
            assert got.kkt.primal_residual_norm <= 1e-9 * (1 + np.linalg.norm(prob.rhs)) * 1.01


def test_empty_batch():
    assert cuda().solve_batch([], P9) == []


@pytest.mark.parametrize("scheme", [0, 1], ids=["two-pass", "refinement"])
def test_mixed_batch_matches_single_mixed_solves(scheme):
    """Each instance of a mixed batch takes the same path as its own
    prima_mixed_solve: same statuses and refinement decisions, objectives at
    the FP64-validated tolerance."""
    from noaidi_b200.prima import convergence
    insts = [i.problem for i in F.optimal()] + [F.infeasible().problem, F.unbounded().problem,
                                                G.dc_lopf(seed=5, buses=150, lines=225, generators=75, snapshots=4)]
    batch = cuda().mixed_solve_batch(insts, P9, scheme=scheme)
    for prob, got in zip(insts, batch):
        one = cuda().mixed_solve(prob, P9, scheme=scheme)
        assert got.solution.status == one.solution.status
        assert got.refined == one.refined
        if one.solution.status == SolveStatus.OPTIMAL:
            assert F.relative_gap(got.solution.objective_value, one.solution.objective_value) <= 1e-8
            conv = convergence(got.solution.kkt, float(np.linalg.norm(prob.rhs)),
                               float(np.linalg.norm(prob.objective)), 1e-9, 1e-9)
            assert conv.converged


def test_labelled_results_keep_their_labels():
    """PrimaZioSuite.scala:73-80: solveLabelled returns each result with its
    label, in the order given."""
    items = [("dispatch", F.economic_dispatch().problem), ("mix", F.product_mix().problem)]
    got = cuda().solve_labelled(items, P9)
    assert [label for label, _ in got] == ["dispatch", "mix"]
    for (label, sol), (_, p) in zip(got, items):
        ref = O.solve(p, P9)
        assert sol.status == SolveStatus.OPTIMAL
        assert sol.objective_value == pytest.approx(ref.objective_value, rel=1e-8)


def test_a_raised_cancel_flag_interrupts_every_instance():
    """PrimaZioSuite.scala:40-58: an interrupted sweep stops at the next
    evaluation point of every instance, reporting Interrupted."""
    import ctypes
    flag = ctypes.c_int32(1)
    insts = [F.random_feasible(5 + k, 200, 40, 80) for k in range(3)]
    got = cuda().solve_batch(insts, PdhgParams(eps_abs=1e-16, eps_rel=1e-16), cancel=flag)
    assert all(s.status == SolveStatus.INTERRUPTED and s.iterations == 64 for s in got), got
