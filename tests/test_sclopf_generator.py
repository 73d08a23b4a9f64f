"""The N-1 security-constrained generator (generators.sclopf_n1)
on CPU: LODF against explicit post-outage power flows, and small instances
solved by the oracle meet every security row."""
import numpy as np
import pytest

from noaidi_b200.prima import PdhgParams, SolveStatus
from noaidi_b200.prima import generators as G


def dc_flows(net, inj, drop=None):
    keep = np.ones(net.lines, dtype=bool)
    if drop is not None:
        keep[drop] = False
    A = np.zeros((net.lines, net.buses))
    A[np.arange(net.lines), net.line_from] += 1.0
    A[np.arange(net.lines), net.line_to] -= 1.0
    y = np.where(keep, 1.0 / net.reactance, 0.0)
    Bm = A.T @ (y[:, None] * A)
    theta = np.zeros(net.buses)
    theta[1:] = np.linalg.solve(Bm[1:, 1:], inj[1:])
    return y * (A @ theta)


def test_lodf_predicts_post_outage_flows():
    rng = np.random.default_rng(4)
    net = G.random_network(rng, 12, 20, 4)
    lodf, ok = G.lodf_matrix(net)
    inj = rng.normal(size=net.buses)
    inj -= inj.mean()
    before = dc_flows(net, inj)
    for o in np.flatnonzero(ok):
        after = dc_flows(net, inj, drop=o)
        predicted = before + lodf[:, o] * before[o]
        predicted[o] = 0.0
        assert np.allclose(after, predicted, atol=1e-9)


def test_small_sclopf_meets_every_security_row():
    from oracle import oracle as O
    P = G.sclopf_n1(seed=1, buses=20, lines=30, generators=8, snapshots=2, outages=6)
    plain = G.dc_lopf(seed=1, buses=20, lines=30, generators=8, snapshots=2)
    p = PdhgParams(eps_abs=1e-7, eps_rel=1e-7, max_iterations=200_000)
    s = O.solve(P, p)
    assert s.status == SolveStatus.OPTIMAL
    kx = P.constraint_matrix.multiply(s.primal)
    neq = P.num_equalities
    assert np.all(kx[neq:] >= P.rhs[neq:] - 1e-5 * (1 + np.abs(P.rhs[neq:])))
    base = O.solve(plain, p)
    assert s.objective_value >= base.objective_value - 1e-6 * abs(base.objective_value)


def test_config4_sizes():
    P = G.sclopf_n1()
    assert P.num_variables == 24 * (300 + 2 * 500 + 750)
    assert 7.0e6 <= P.num_constraints - P.num_equalities <= 7.2e6
    assert 14.0e6 <= P.constraint_matrix.nnz <= 14.5e6
