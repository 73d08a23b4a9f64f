"""A warm start saved to disk and read back resumes a solve exactly as the
in-memory one does (the oracle solving): the Pdhg.WarmStart four-tuple
(Pdhg.scala:72-105) is the checkpoint."""
import numpy as np

from noaidi_b200.prima import PdhgParams
from noaidi_b200.prima.types import WarmStart
from tests import lp_fixtures as F


def test_a_saved_warm_start_resumes_identically(tmp_path):
    from oracle import oracle as O
    p = F.economic_dispatch().problem
    partial = O.solve(p, PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=128))
    warm = WarmStart.from_solution(partial)
    path = str(tmp_path / "checkpoint.npz")
    warm.save(path)
    back = WarmStart.load(path)
    assert np.array_equal(back.primal, warm.primal) and np.array_equal(back.dual, warm.dual)
    assert (back.step_size, back.primal_weight) == (warm.step_size, warm.primal_weight)
    params = PdhgParams(eps_abs=1e-9, eps_rel=1e-9)
    a, b = O.solve(p, params, warm_start=warm), O.solve(p, params, warm_start=back)
    assert (a.status, a.iterations, a.restarts, a.objective_value) == (b.status, b.iterations, b.restarts,
                                                                        b.objective_value)


def test_a_point_without_adaptive_state_round_trips(tmp_path):
    warm = WarmStart(np.array([1.0, 2.0]), np.array([0.5]))
    path = str(tmp_path / "point.npz")
    warm.save(path)
    back = WarmStart.load(path)
    assert back.step_size is None and back.primal_weight is None
    assert np.array_equal(back.primal, warm.primal)


def test_a_path_without_extension_is_written_and_read_at_that_path(tmp_path):
    warm = WarmStart(np.array([3.0, -1.0]), np.array([0.25, 4.0]), 0.5, 2.0)
    path = str(tmp_path / "ckpt")
    warm.save(path)
    assert (tmp_path / "ckpt").exists() and not (tmp_path / "ckpt.npz").exists()
    back = WarmStart.load(path)
    assert np.array_equal(back.primal, warm.primal) and np.array_equal(back.dual, warm.dual)
    assert (back.step_size, back.primal_weight) == (0.5, 2.0)
