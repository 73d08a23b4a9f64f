"""Unit commitment: ``UnitCommitment.solve``
(modules/network-lopf/src/main/scala/org/noaidi/lopf/UnitCommitment.scala:116-300),
which thermal units run as well as how much they produce, solved by the
branch-and-bound of noaidi_b200.prima.bnb with every node relaxation on the
GPU -- the LP matrix stays resident and each node only moves bounds.

Per committable generator g and snapshot t: a binary status u, and
continuous start-up and shut-down indicators su, sd (driven to 0 or 1 by
the rows below whenever u is integral, and costed non-negatively, so the
search branches on u alone):

    p_min_pu p_nom u <= p <= p_max_pu p_nom u
    su - sd = u[t] - u[t-1]      (u[-1] from up_time_before)
    sum of su over the last min_up_time snapshots   <= u[t]
    sum of sd over the last min_down_time snapshots <= 1 - u[t]

and, at the head of the horizon, u pinned for the residual of a minimum up
or down time the unit was already serving (min_up_time - up_time_before).
Bus balance has generators and loads only: the model is a single bus, so a
network with branches, storage, global constraints, ramp limits, stand-by or
quadratic costs, or extendable generators is refused rather than solved as a
cheaper problem.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

from ..prima.bnb import BnbParams, MilpSolution, MilpStatus, NodeSolver, device_node_solver, solve_with
from ..prima.model import LpBuilder, LpProblem
from ..prima.types import PdhgParams
from . import standard_types
from .pypsa_csv import Network

HANDLED = {"Generator", "Load", "Bus", "Carrier", "SubNetwork", "LineType", "TransformerType", "Shape"}


class UnsupportedNetwork(ValueError):
    """``UnitCommitment.UnsupportedNetwork``."""


@dataclass
class UcResult:
    """``UcResult`` (UnitCommitment.scala:7-38)."""
    status: MilpStatus
    objective: float
    best_bound: float
    nodes_explored: int
    solution: MilpSolution
    _dispatch: dict
    _commitment: dict

    def output(self, generator: str, snapshot: int) -> float:
        """Output in MW."""
        return self._dispatch[(generator, snapshot)]

    def committed(self, generator: str, snapshot: int) -> bool:
        """A non-committable generator has no status variable and reports True."""
        return self._commitment[(generator, snapshot)]


@dataclass
class UcModel:
    problem: LpProblem
    columns: dict        # (kind, generator, t) -> column; kind in p, u, su, sd
    integers: set
    committable: dict    # generator -> bool


def _committable(gens, g) -> bool:
    return "committable" in gens.static and bool(gens.value("committable", g)) is True


def _int(gens, attr, g) -> int:
    return int(float(gens.value(attr, g)))


def _reject(network: Network) -> None:
    """``UnitCommitment.reject`` (UnitCommitment.scala:316-425)."""
    gc = network.table("GlobalConstraint")
    if len(gc):
        raise UnsupportedNetwork(f"network has {len(gc)} global constraint(s); emissions and primary-energy caps are "
                                 "not modelled here, and dropping one would price the schedule below the truth")
    unhandled = [f"{c} ({len(t)})" for c, t in network.tables.items() if len(t) and c not in HANDLED]
    if unhandled:
        raise UnsupportedNetwork("unit commitment is formulated without branch flows, so it models a single bus; "
                                 "this network carries " + ", ".join(unhandled))
    buses = set(network.table("Bus").ids)
    for comp in ("Generator", "Load"):
        tab = network.table(comp)
        for i in tab.ids:
            if str(tab.value("bus", i)) not in buses:
                raise UnsupportedNetwork(f"{comp} '{i}' references unknown bus '{tab.value('bus', i)}' via bus")
    gens = network.table("Generator")
    for attr in ("stand_by_cost", "marginal_cost_quadratic"):
        if attr in gens.static or attr in gens.series:
            for g in gens.ids:
                values = [("statically", float(gens.value(attr, g)))] + \
                    [(f"at snapshot {t}", gens.at(attr, g, t)) for t in range(len(network.snapshots))]
                for where, v in values:
                    if math.isfinite(v) and v != 0.0:
                        raise UnsupportedNetwork(f"generator '{g}' has {attr} = {v} {where}; it enters PyPSA's "
                                                 "objective and not this one, so ignoring it would price the "
                                                 "schedule below the truth")
    for attr in ("ramp_limit_up", "ramp_limit_down", "ramp_limit_start_up", "ramp_limit_shut_down"):
        if attr in gens.static:
            for g in gens.ids:
                v = float(gens.value(attr, g))
                if math.isfinite(v):
                    raise UnsupportedNetwork(f"generator '{g}' has {attr} = {v}; ramp limits are not modelled, and "
                                             "ignoring one yields a schedule the network cannot actually follow")
    for g in gens.ids:
        if "p_nom_extendable" in gens.static and bool(gens.value("p_nom_extendable", g)) is True:
            raise UnsupportedNetwork(f"generator '{g}' is extendable; commitment takes capacity as given")


def build(network: Network) -> UcModel:
    """The commitment MILP's relaxation, with its integer columns."""
    network = standard_types.expand(network)
    _reject(network)
    T = len(network.snapshots)
    if T == 0:
        raise UnsupportedNetwork("network has no snapshots")
    gens, loads = network.table("Generator"), network.table("Load")
    buses = network.table("Bus").ids
    committable = {g: _committable(gens, g) for g in gens.ids}
    units = [g for g in gens.ids if committable[g]]
    limits = {}
    for t in range(T):
        for g in gens.ids:
            p_nom = float(gens.value("p_nom", g))
            limits[(g, t)] = (p_nom * gens.at("p_min_pu", g, t), p_nom * gens.at("p_max_pu", g, t))
    columns, bounds, costs = {}, [], []

    def declare(kind, g, t, lo, hi, cost):
        columns[(kind, g, t)] = len(bounds)
        bounds.append((lo, hi))
        costs.append(cost)

    for t in range(T):
        w = network.weighting("objective", t)
        for g in gens.ids:
            lo, hi = limits[(g, t)]
            cost = gens.at("marginal_cost", g, t) * w
            if committable[g]:  # the floor is enforced through u: zero is allowed too
                declare("p", g, t, 0.0, max(hi, 0.0), cost)
            else:
                declare("p", g, t, min(lo, hi), max(lo, hi), cost)
        for g in units:
            declare("u", g, t, 0.0, 1.0, 0.0)
            declare("su", g, t, 0.0, 1.0, float(gens.value("start_up_cost", g)))
            declare("sd", g, t, 0.0, 1.0, float(gens.value("shut_down_cost", g)))

    b = LpBuilder(len(bounds))
    for j, (lo, hi) in enumerate(bounds):
        b.bounds(j, lo, hi)
    for j, c in enumerate(costs):
        b.objective_coefficient(j, c)
    at_bus = {bus: [g for g in gens.ids if str(gens.value("bus", g)) == bus] for bus in buses}
    loads_at = {bus: [d for d in loads.ids if str(loads.value("bus", d)) == bus] for bus in buses}
    for t in range(T):
        for bus in buses:
            terms = [(columns[("p", g, t)], 1.0) for g in at_bus[bus]]
            demand = sum(loads.at("p_set", d, t) for d in loads_at[bus])
            if terms or demand != 0.0:
                b.equality_constraint(terms, demand)
    for t in range(T):
        for g in units:
            p, on, su, sd = (columns[(k, g, t)] for k in ("p", "u", "su", "sd"))
            lo, hi = limits[(g, t)]
            b.less_than([(p, 1.0), (on, -hi)], 0.0)
            b.greater_than([(p, 1.0), (on, -lo)], 0.0)
            up_before, down_before = _int(gens, "up_time_before", g), _int(gens, "down_time_before", g)
            initially_up = up_before > 0
            if t > 0:
                b.equality_constraint([(su, 1.0), (sd, -1.0), (on, -1.0), (columns[("u", g, t - 1)], 1.0)], 0.0)
            else:
                b.equality_constraint([(su, 1.0), (sd, -1.0), (on, -1.0)], -(1.0 if initially_up else 0.0))
            min_up, min_down = _int(gens, "min_up_time", g), _int(gens, "min_down_time", g)
            forced = max(min_up - up_before, 0) if initially_up else max(min_down - down_before, 0)
            if t < forced:  # the residual of a minimum time served before the horizon
                b.equality_constraint([(on, 1.0)], 1.0 if initially_up else 0.0)
            if min_up > 1:
                window = [(columns[("su", g, i)], 1.0) for i in range(max(0, t - min_up + 1), t + 1)]
                b.less_than(window + [(on, -1.0)], 0.0)
            if min_down > 1:
                window = [(columns[("sd", g, i)], 1.0) for i in range(max(0, t - min_down + 1), t + 1)]
                b.less_than(window + [(on, 1.0)], 1.0)
    problem, _ = b.build()
    integers = {j for (k, _, _), j in columns.items() if k == "u"}
    return UcModel(problem, columns, integers, committable)


DEFAULT_PARAMS = BnbParams(lp=PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=200_000), max_nodes=20_000)


def solve(network: Network, params: BnbParams = DEFAULT_PARAMS, node_solver: Optional[NodeSolver] = None,
          precision: int = 64, device: int = 0) -> UcResult:
    """``UnitCommitment.solve``: the MILP by branch-and-bound, node
    relaxations on the GPU unless a node solver is given."""
    model = build(network)
    resident = None
    if node_solver is None:
        node_solver = device_node_solver(model.problem, params, precision=precision, device=device)
        resident = node_solver.resident
    try:
        milp = solve_with(model.problem, model.integers, params, node_solver)
    finally:
        if resident is not None:
            resident.free()
    dispatch, commitment = {}, {}
    if milp.primal.size:
        gens = network.table("Generator")
        for t in range(len(network.snapshots)):
            for g in gens.ids:
                dispatch[(g, t)] = float(milp.primal[model.columns[("p", g, t)]])
                commitment[(g, t)] = bool(milp.primal[model.columns[("u", g, t)]] > 0.5) if model.committable[g] \
                    else True
    return UcResult(milp.status, milp.objective_value, milp.best_bound, milp.nodes_explored, milp, dispatch,
                    commitment)
