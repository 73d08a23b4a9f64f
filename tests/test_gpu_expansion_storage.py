"""The capacity-expansion LOPF with storage on the device, FP64 and the FP32
refinement scheme, against the oracle on the same small year slice."""
import pytest

from noaidi_b200.network import synthetic as S
from noaidi_b200.prima import PdhgParams

pytestmark = pytest.mark.gpu

P = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=1_000_000)


@pytest.mark.parametrize("mixed", [False, True])
def test_a_year_slice_matches_the_oracle_on_the_device(mixed):
    from noaidi_b200.prima import cuda
    from oracle import oracle as O
    p = S.expansion_storage(0, 12, 18, 20, 4, 48)
    want = O.solve(p, P)
    got = cuda.mixed_solve(p, P).solution if mixed else cuda.solve(p, P, precision=64)
    assert got.status == want.status
    assert got.objective_value == pytest.approx(want.objective_value, rel=1e-8)
