"""UnitCommitmentSuite's checks (modules/network-lopf/src/test/scala/org/noaidi/
lopf/UnitCommitmentSuite.scala:43-305) on PyPSA's unit-commitment network: the
MILP built by noaidi_b200.network.unit_commitment, its node relaxations
solved by a node solver passed in (the oracle on CPU, the device on GPU),
against PyPSA's optimum of 17,000 and its schedule."""
import os

import pytest

from noaidi_b200.network import unit_commitment as U
from noaidi_b200.network.pypsa_csv import read
from noaidi_b200.prima.bnb import MilpStatus
from tests import lopf_cases as X

HERE = X.HERE


def network():
    return X.network("unit-commitment")


def check_against_pypsa(solve):
    """solve(network) -> UcResult."""
    n, exp = network(), X.expected("unit-commitment")
    res = solve(n)
    assert res.status == MilpStatus.OPTIMAL, res.solution
    assert res.objective == pytest.approx(exp["objective"], abs=1e-6 * 17000.0)
    gens, loads = n.table("Generator"), n.table("Load")
    T = len(n.snapshots)
    off = 0
    for t in range(T):
        for g in gens.ids:
            if U._committable(gens, g):  # the schedule (:53-80); a non-committable unit decides nothing
                theirs = X.frame_value(exp["generator_status"], t, g) > 0.5
                assert res.committed(g, t) == theirs, (g, t)
                off += not theirs
            assert res.output(g, t) == pytest.approx(X.frame_value(exp["generator_p"], t, g), abs=1e-4), (g, t)
            if U._committable(gens, g):  # minimum output when on, nothing when off (:95-117)
                floor = float(gens.value("p_nom", g)) * gens.at("p_min_pu", g, t)
                if res.committed(g, t):
                    assert res.output(g, t) >= floor - 1e-4
                else:
                    assert res.output(g, t) == pytest.approx(0.0, abs=1e-4)
        supplied = sum(res.output(g, t) for g in gens.ids)
        assert supplied == pytest.approx(sum(loads.at("p_set", d, t) for d in loads.ids), abs=1e-4)
    assert off >= 3
    for g in gens.ids:  # minimum down time holds, and it is what makes this cost 17000 (:132-157)
        if not U._committable(gens, g):
            continue
        min_down = int(float(gens.value("min_down_time", g)))
        run_start = None
        for t in range(T + 1):
            on = t == T or res.committed(g, t)
            if not on and run_start is None:
                run_start = t
            elif on and run_start is not None:
                if t < T:
                    assert t - run_start >= min_down, (g, run_start, t)
                run_start = None
    return res


def residual_network(tmp):
    """One expensive committable unit serving its minimum up time at the
    horizon head beside ample cheap capacity (:229-288): PyPSA holds it at its
    50 MW minimum for two snapshots and releases it, for 57,000."""
    os.makedirs(tmp, exist_ok=True)
    files = {
        "buses.csv": "name,v_nom,carrier\nbus,110.0,AC\n",
        "generators.csv": "name,bus,p_nom,p_min_pu,marginal_cost,committable,min_up_time,min_down_time\n"
                          "unit,bus,100.0,0.5,500.0,True,3,1\ncheap,bus,500.0,0.0,10.0,False,0,0\n",
        "loads.csv": "name,bus,p_set\nd,bus,200.0\n",
        "snapshots.csv": ",snapshot\n0,0\n1,1\n2,2\n3,3\n",
    }
    for name, text in files.items():
        with open(os.path.join(tmp, name), "w") as f:
            f.write(text)
    return read(tmp, "uc-residual")


def check_residual(solve, tmp):
    res = solve(residual_network(tmp))
    assert res.status == MilpStatus.OPTIMAL
    for t in range(2):
        assert res.committed("unit", t) and res.output("unit", t) == pytest.approx(50.0, abs=1e-4)
    for t in range(2, 4):
        assert not res.committed("unit", t)
    assert res.objective == pytest.approx(57000.0, abs=1e-3)
