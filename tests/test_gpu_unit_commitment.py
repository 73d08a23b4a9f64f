"""Unit commitment with every branch-and-bound node relaxation solved on the
device (FP64, the matrix resident, bounds moved per node), against PyPSA."""
import pytest

from noaidi_b200.network import unit_commitment as U
from tests import uc_cases as X

pytestmark = pytest.mark.gpu


def test_unit_commitment_matches_pypsa_on_the_device():
    res = X.check_against_pypsa(lambda n: U.solve(n))
    assert res.nodes_explored >= 1


def test_the_horizon_head_residual_on_the_device(tmp_path):
    X.check_residual(lambda n: U.solve(n), str(tmp_path / "residual"))
