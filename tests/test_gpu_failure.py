"""The bounded waits of the persistent solver, made to run out on purpose.

Every wait in the kernel is bounded: a block waiting at a team barrier for
the other blocks gives up after a number of polls, raises the team's abort
flag, and every block leaves; the call returns PRIMA_ERR_TIMEOUT and the
context stays usable.  The reference has no such wait (its loop,
``Pdhg.scala:206-246``, runs on one thread); these tests make the wait run
out by setting the poll limit so low that no multi-block team can meet it,
and check the error, then that the same context solves normally again.
Nothing here faults, traps or hangs the GPU: the wait ends by its own bound.
"""
import pytest

from noaidi_b200.prima import PdhgParams, SolveStatus
from tests import multiblock_cases as M

pytestmark = pytest.mark.gpu

P6 = PdhgParams(eps_abs=1e-6, eps_rel=1e-6, max_iterations=200_000)


@pytest.mark.parametrize("precision", [64, 32])
def test_a_team_barrier_gives_up_and_the_context_recovers(precision):
    from noaidi_b200.prima import cuda
    p = M.lopf_300x24()
    ctx = cuda.Context(0, precision)
    try:
        ctx.set_device_wait_limit(1)
        with pytest.raises(cuda.PrimaError) as err:
            cuda.solve(p, P6, ctx=ctx)
        assert err.value.code == cuda.ERR_TIMEOUT
        # again: the abort state does not leak into the next launch
        with pytest.raises(cuda.PrimaError) as err:
            cuda.solve(p, P6, ctx=ctx)
        assert err.value.code == cuda.ERR_TIMEOUT
        ctx.set_device_wait_limit(0)  # the default bound
        s = cuda.solve(p, P6, ctx=ctx)
        assert s.status == SolveStatus.OPTIMAL and s.blocks > 1
    finally:
        ctx.close()


def test_a_one_block_solve_never_waits_on_another_block():
    """A problem of up to 4,096 rows and columns runs as one block, whose
    barriers are __syncthreads: the poll limit does not apply."""
    from noaidi_b200.prima import cuda
    from tests import lp_fixtures as F
    ctx = cuda.Context(0, 64)
    try:
        ctx.set_device_wait_limit(1)
        s = cuda.solve(F.economic_dispatch().problem, PdhgParams(eps_abs=1e-9, eps_rel=1e-9), ctx=ctx)
        assert s.status == SolveStatus.OPTIMAL and s.blocks == 1
    finally:
        ctx.close()


def test_the_limit_must_be_non_negative():
    from noaidi_b200.prima import cuda
    ctx = cuda.Context(0, 64)
    try:
        with pytest.raises(ValueError):
            ctx.set_device_wait_limit(-1)
    finally:
        ctx.close()
