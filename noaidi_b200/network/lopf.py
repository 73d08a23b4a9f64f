"""Dispatch LOPF: a PyPSA network as an LP for the device solve, and the
answer mapped back onto component names.  The dispatch subset of ``Lopf``
(modules/network-lopf/src/main/scala/org/noaidi/lopf/Lopf.scala:69-561)
with its conventions, since equivalence is judged against PyPSA's output:

* columns per snapshot: each generator's output in p_nom x [p_min_pu,
  p_max_pu], each passive branch's flow p0 in +-s_nom x s_max_pu, each link's
  p0 in p_nom x [p_min_pu, p_max_pu]; costs are marginal_cost x the
  snapshot's objective weighting (:148-196);
* bus balance per snapshot and bus: generators inject, a branch takes p0 out
  at bus0 and delivers efficiency x p0 at bus1 (1 for a line), and a
  multi-port link efficiencyN x p0 at each further busN it names
  (Topology.scala:175-227), loads on the right-hand side (:281-333);
* Kirchhoff's voltage law over a cycle basis of the passive branches, one
  row per cycle per snapshot: sum(orientation x impedance x p0) = 0, with
  reactance in AC sub-networks and resistance in DC ones, referred to
  v_nom squared (:397-433; Cycles.scala);
* primary-energy global constraints (<=): per generator, carrier intensity /
  efficiency x the snapshot's generators weighting (:503-559).

* storage units (Lopf.scala:200-240, :336-395; Storage.scala): discharge,
  charge, state of charge and spill per snapshot; discharge and charge at
  the bus; the state of charge carried between snapshots through the
  efficiencies, the standing loss raised to the elapsed hours (the
  snapshot's stores weighting), inflow and spill, from the previous snapshot,
  the last one when cyclic, or the initial state; set points pin it.

* stores (Stores.scala; Lopf.scala:242-265, :440-467): an energy level in
  e_nom x [e_min_pu, e_max_pu] and one signed power with no rating, positive
  into the bus; e(t) = (1 - standing_loss)^eh e(t-1) - eh p(t), wrapping to
  the last snapshot when cyclic, else starting from e_initial.

* capacity expansion (Expansion.scala; Lopf.scala:124-146, :453-478): one
  capacity column per extendable entity over the horizon, bounded by
  ``<nom>_min``/``<nom>_max`` and costed at capital plus fixed O&M cost; the
  entity's operational columns become unbounded and two rows per snapshot
  tie them to min_pu and max_pu times the capacity; the objective is the
  cost of the change, so the existing capacity's cost is subtracted.

* standard types (noaidi_b200.network.standard_types): a typed line's or
  transformer's impedance and a typed transformer's rating come from the
  type library, expanded before anything is built.

* transformers: passive branches like lines, rated by s_nom x s_max_pu and
  referred to their own base in Kirchhoff rows, z tap_ratio / s_nom
  (Cycles.scala:154-193); the phase shift moves angles, not the optimised
  flows, and is not read.  The security-constrained model monitors and
  outages lines and transformers alike.

Components the dispatch model does not build (processes, shunts), committable generators, generator, storage or store set points, and
annuitised or modular capacities are refused rather than
dropped: a dropped component leaves a feasible LP for a different network.
"""
from __future__ import annotations

import math
import re
from collections import deque
from dataclasses import dataclass
from typing import Optional

import numpy as np

from ..prima.model import LpBuilder, LpProblem, Negated, RowTranslation
from ..prima.types import LpSolution, PdhgParams, SolveStatus
from . import standard_types
from .pypsa_csv import CATEGORY, LIST_NAMES, MalformedNetwork, Network

HANDLED = {"Bus", "Carrier", "Generator", "Load", "Line", "Transformer", "Link", "GlobalConstraint", "SubNetwork",
           "LineType", "TransformerType", "Shape", "StorageUnit", "Store"}


def _role(*categories) -> tuple:
    """Components by PyPSA's own category (``Role.of``, Topology.scala:31-49),
    in the order of their list names, as the reference reads the files."""
    return tuple(sorted((c for c, k in CATEGORY.items() if k in categories), key=LIST_NAMES.get))


PASSIVE = _role("passive_branch")  # Line, Transformer: branches whose flow follows from impedance
BRANCHES = _role("passive_branch", "controllable_branch")  # with Link and Process
ONE_PORTS = _role("controllable_one_port", "passive_one_port")  # attached at one bus


class UnsupportedNetwork(ValueError):
    """``Lopf.UnsupportedNetwork``."""


@dataclass
class Cycle:
    carrier: str
    terms: list  # (component, id, orientation)


@dataclass
class Model:
    problem: LpProblem
    translation: RowTranslation
    columns: dict      # (component, id, t) -> column
    balance_rows: dict  # (bus, t) -> row of the builder's constraints (before standard form)
    cycles: list
    objective_constant: float = 0.0  # cost of the capacity the network came with, extendables only
    network: Optional[Network] = None  # what the LP was built from: standard types expanded


@dataclass
class LopfResult:
    network: Network
    model: Model
    solution: LpSolution

    @property
    def status(self) -> SolveStatus:
        return self.solution.status

    @property
    def objective(self) -> float:
        return self.solution.objective_value

    @property
    def total_system_cost(self) -> float:
        """PyPSA's objective plus its ``objective_constant``: the cost of the
        whole optimal capacity rather than of the change."""
        return self.objective + self.model.objective_constant

    def dispatch(self, component: str, entity: str, t: int) -> float:
        """A column's value; for a StorageUnit the net injection p_dispatch -
        p_store (PyPSA's storage_units_t.p), for a Store its signed power."""
        if component == "StorageUnit":
            return self.discharging(entity, t) - self.charging(entity, t)
        if component == "Store":
            return self._col("Store-p", entity, t)
        return self._col(component, entity, t)

    def _col(self, key: str, entity: str, t: int) -> float:
        return float(self.solution.primal[self.model.columns[(key, entity, t)]])

    def energy(self, entity: str, t: int) -> float:
        """A store's energy at the end of snapshot t."""
        return self._col("Store-e", entity, t)

    def state_of_charge(self, entity: str, t: int) -> float:
        """A storage unit's state of charge at the end of snapshot t."""
        return self._col("StorageUnit-state_of_charge", entity, t)

    def charging(self, entity: str, t: int) -> float:
        return self._col("StorageUnit-p_store", entity, t)

    def discharging(self, entity: str, t: int) -> float:
        return self._col("StorageUnit-p_dispatch", entity, t)

    def spill(self, entity: str, t: int) -> float:
        return self._col("StorageUnit-spill", entity, t)

    def marginal_price(self, bus: str, t: int) -> float:
        """The dual of the bus's balance row at snapshot t, through the row
        translation (so the sign is the constraint's as written), per unit of
        the snapshot's objective weighting (``LopfResult.marginalPrice``,
        Lopf.scala:692-706)."""
        if (bus, t) not in self.model.balance_rows:
            raise KeyError(f"no balance row for bus '{bus}' at snapshot {t}")
        duals = self.__dict__.get("_duals")
        if duals is None:
            duals = self.model.translation.original_duals(self.solution.dual)
            self.__dict__["_duals"] = duals
        return float(duals[self.model.balance_rows[(bus, t)]]) / (self.model.network or self.network).weighting(
            "objective", t)

    def capacity(self, component: str, entity: str) -> float:
        """The chosen capacity of an extendable entity, else its given one
        (``LopfResult.capacity``)."""
        nom = NOMINAL[component]
        col = self.model.columns.get((f"{component}-{nom}", entity, -1))
        if col is None:
            return float((self.model.network or self.network).table(component).value(nom, entity))
        return float(self.solution.primal[col])


def _reject(network: Network) -> None:
    unhandled = [f"{c} ({len(t)})" for c, t in network.tables.items() if len(t) and c not in HANDLED]
    if unhandled:
        raise UnsupportedNetwork("network contains unmodelled component(s): " + ", ".join(unhandled))
    for comp, nom in NOMINAL.items():  # Expansion.reject (Expansion.scala:133-190)
        tab = network.table(comp)
        for i in tab.ids:
            if not extendable(tab, i):
                continue
            if "overnight_cost" in tab.static and math.isfinite(float(tab.value("overnight_cost", i))):
                raise UnsupportedNetwork(f"{comp} '{i}' sets overnight_cost; only capital_cost is modelled")
            mod = float(tab.value(f"{nom}_mod", i)) if f"{nom}_mod" in tab.static else math.nan
            if math.isfinite(mod) and mod > 0.0:
                raise UnsupportedNetwork(f"{comp} '{i}' sets {nom}_mod: a modular capacity is mixed-integer")
            lo, hi = float(tab.value(f"{nom}_min", i)), float(tab.value(f"{nom}_max", i))
            if lo > hi:
                raise UnsupportedNetwork(f"{comp} '{i}' has {nom}_min = {lo} above {nom}_max = {hi}")
            if not lo >= 0.0:
                raise UnsupportedNetwork(f"{comp} '{i}' has {nom}_min = {lo}, which is not a capacity")
    gens = network.table("Generator")
    for g in gens.ids:
        if bool(gens.value("committable", g)) is True:
            raise UnsupportedNetwork(f"Generator '{g}' is committable; unit commitment is not a dispatch LP "
                                     "(noaidi_b200.network.unit_commitment solves it as a MILP)")
    if "p_set" in gens.series and np.isfinite(gens.series["p_set"]).any():
        raise UnsupportedNetwork("a generator has a p_set, which fixes its dispatch; the dispatch model does not")
    su = network.table("StorageUnit")
    for attr in ("p_set", "p_dispatch_set", "p_store_set"):  # Storage.reject (Storage.scala:26-39)
        if (attr in su.series and np.isfinite(su.series[attr]).any()) or any(
                math.isfinite(float(su.value(attr, i))) for i in su.ids if attr in su.static):
            raise UnsupportedNetwork(f"a StorageUnit sets {attr}, which pins its dispatch; not built here")
    for i in su.ids:
        if not float(su.value("max_hours", i)) > 0.0:
            raise UnsupportedNetwork(f"StorageUnit '{i}' has max_hours = {su.value('max_hours', i)}, so it can store nothing")
    _reject_standing_loss(network, su)
    st = network.table("Store")
    for attr, what in (("e_set", "its energy"), ("p_set", "its power")):  # Stores.reject (Stores.scala:48-90)
        pinned = [i for i in st.ids if attr in st.static and math.isfinite(float(st.value(attr, i)))]
        if attr in st.series and np.isfinite(st.series[attr]).any():
            pinned.append("(series)")
        if pinned:
            raise UnsupportedNetwork(f"Store '{pinned[0]}' sets {attr}, which pins {what}; that constraint is "
                                     "not built here")
    for attr in ("e_cyclic_per_period", "e_initial_per_period"):
        if any(attr in st.static and bool(st.value(attr, i)) is True for i in st.ids):
            raise UnsupportedNetwork(f"a Store sets {attr}, a multi-period concept; this model has one horizon")
    if any(float(st.value("marginal_cost_quadratic", i)) != 0.0 for i in st.ids) or \
            ("marginal_cost_quadratic" in st.series and np.any(st.series["marginal_cost_quadratic"] != 0.0)):
        raise UnsupportedNetwork("a Store has a non-zero marginal_cost_quadratic; the objective here is linear")
    _reject_standing_loss(network, st)
    dangling = dangling_bus_references(network)  # Lopf.rejectDanglingBuses (Lopf.scala:593-606)
    if dangling:
        comp, i, port, bus = dangling[0]
        raise UnsupportedNetwork(f"{comp} '{i}' references unknown bus '{bus}' via {port}")




def _ports(network: Network, component: str) -> list:
    """``Topology.portsOf`` (Topology.scala:212-232): a branch table's bus
    columns in port order; one without bus0 or bus1 is malformed."""
    tab = network.table(component)
    if not len(tab):
        return []
    for required in ("bus0", "bus1"):
        if required not in tab.static:
            raise MalformedNetwork(f"{LIST_NAMES[component]} has no '{required}' column; a branch needs both "
                                   "endpoints")
    return link_ports(tab)


def dangling_references(network: Network, components=BRANCHES) -> list:
    """``Topology.danglingReferences`` (Topology.scala:277-326): every
    (component, id, port, bus) of a branch naming no bus.  A blank bus0 or
    bus1 is dangling; a blank further port (a two-port link in a table with
    a bus2 column) is not connected, and not an error."""
    known = set(network.table("Bus").ids)
    out = []
    for comp in components:
        tab = network.table(comp)
        for port in _ports(network, comp):
            for i in tab.ids:
                bus = tab.endpoint(port, i)
                if (bus not in known) if bus else port in ("bus0", "bus1"):
                    out.append((comp, i, port, bus))
    return out


def dangling_bus_references(network: Network) -> list:
    """``Topology.danglingBusReferences`` (Topology.scala:293-307): the
    branches' dangling references, then every one-port component whose bus
    names no bus (a stale load would simply vanish from the balance)."""
    known = set(network.table("Bus").ids)
    out = dangling_references(network)
    for comp in ONE_PORTS:
        tab = network.table(comp)
        out += [(comp, i, "bus", tab.endpoint("bus", i)) for i in tab.ids if tab.endpoint("bus", i) not in known]
    return out


def _pairs(network: Network, components) -> list:
    """``Topology.branchesWhere`` (Topology.scala:234-252): every pair of a
    branch's non-blank ports, so a multi-port link connects all of them."""
    out = []
    for comp in components:
        tab = network.table(comp)
        ports = _ports(network, comp)
        for i in tab.ids:
            ends = [b for b in (tab.endpoint(p, i) for p in ports) if b]
            out += [(a, b) for k, a in enumerate(ends) for b in ends[k + 1:]]
    return out


def controllable_branches(network: Network) -> list:
    """Endpoint pairs of the links and processes
    (``Topology.controllableBranches``)."""
    return _pairs(network, _role("controllable_branch"))


def isolated_buses(network: Network) -> list:
    """Buses no branch of any kind reaches (``Topology.isolatedBuses``,
    Topology.scala:335-344): a load there makes the network infeasible."""
    connected = {b for pair in _pairs(network, BRANCHES) for b in pair}
    return [b for b in network.table("Bus").ids if b not in connected]


def attached_to(network: Network, bus: str) -> list:
    """(component, id) of the one-ports at a bus (``Topology.attachedTo``);
    branches are not attached, they have bus0 and bus1."""
    return [(comp, i) for comp in ONE_PORTS for i in network.table(comp).ids
            if network.table(comp).endpoint("bus", i) == bus]


def link_ports(links) -> list:
    """``Topology.portsOf``: bus0, bus1 and any further busN columns of a
    branch table, in port order (a multi-port link, PyPSA's ``bus2``...)."""
    ports = [c for c in links.static if re.fullmatch(r"bus[0-9]+", c)]
    return sorted(set(ports) | {"bus0", "bus1"}, key=lambda c: int(c[3:]))


def port_efficiency(links, entity: str, port: str, t: int) -> float:
    """``Topology.portEfficiency``: ``efficiency`` for bus1, ``efficiencyN``
    for busN, a series over the static value; a missing or non-finite value
    is lossless."""
    attr = "efficiency" if port == "bus1" else f"efficiency{port[3:]}"
    if attr not in links.series and attr not in links.static and attr != "efficiency":
        return 1.0
    v = links.at(attr, entity, t)
    return v if math.isfinite(v) else 1.0


NOMINAL = {"Generator": "p_nom", "Line": "s_nom", "Transformer": "s_nom", "Link": "p_nom", "StorageUnit": "p_nom",
           "Store": "e_nom"}
EXPANSION_ORDER = ("Line", "Transformer", "Link", "Generator", "StorageUnit", "Store")


def passive_branches(network: Network) -> list:
    """(component, id, bus0, bus1) of every line and transformer, lines first."""
    out = []
    for c in PASSIVE:
        tab = network.table(c)
        out += [(c, i, str(tab.value("bus0", i)), str(tab.value("bus1", i))) for i in tab.ids]
    return out


def extendable(tab, entity: str) -> bool:
    """``Expansion.isExtendable``: the ``<nom>_extendable`` flag."""
    nom = NOMINAL.get(tab.component)
    return nom is not None and f"{nom}_extendable" in tab.static and bool(tab.value(f"{nom}_extendable", entity))


def periodized_cost(tab, entity: str) -> float:
    """``Expansion.periodizedCost``: capital cost plus fixed O&M cost."""
    total = 0.0
    for attr in ("capital_cost", "fom_cost"):
        v = float(tab.value(attr, entity))
        if math.isfinite(v):
            total += v
    return total


def _reject_standing_loss(network: Network, tab) -> None:
    """``Losses.rejectStandingLoss``: a standing loss outside [0, 1) at any
    snapshot the energy balance reads is a gain, not a loss."""
    for i in tab.ids:
        for t in range(len(network.snapshots)):
            loss = tab.at("standing_loss", i, t)
            if not (0.0 <= loss < 1.0):
                raise UnsupportedNetwork(f"{tab.component} '{i}' has standing_loss = {loss} at snapshot {t}, "
                                         "not a fraction below 1")


def cycle_basis(network: Network) -> list:
    """A cycle basis of the passive branches: per connected component a
    breadth-first spanning tree and one cycle per non-tree edge (circuit rank
    edges - nodes + components).  orientation +1 where the cycle runs bus0 to
    bus1.  Any basis spans the same constraints."""
    edges = passive_branches(network)
    adjacency: dict = {}
    for e in edges:
        adjacency.setdefault(e[2], []).append(e)
        adjacency.setdefault(e[3], []).append(e)
    bus_tab = network.table("Bus")
    # the island's label, read off its first sorted bus rather than this walk's
    # root, so that a mixed-carrier island picks x or r as Cycles.scala:43-53 does
    carrier_of = {b: sub.carrier for sub in sub_networks(network) for b in sub.buses}
    visited, cycles = set(), []
    for root in bus_tab.ids:
        if root in visited or root not in adjacency:
            continue
        carrier = carrier_of[root]
        parent, depth = {}, {root: 0}
        tree = set()
        visited.add(root)
        order = deque([root])
        while order:
            b = order.popleft()
            for e in adjacency[b]:
                nxt = e[3] if e[2] == b else e[2]
                if nxt not in visited:
                    visited.add(nxt)
                    parent[nxt] = e
                    depth[nxt] = depth[b] + 1
                    tree.add((e[0], e[1]))
                    order.append(nxt)
        seen = set()
        for b in sorted(depth):
            for e in adjacency[b]:
                key = (e[0], e[1])
                if key in tree or key in seen:
                    continue
                seen.add(key)
                # walk both ends up to their common ancestor: bus1 -> ... -> bus0 closes the cycle
                terms = [(e[0], e[1], 1.0)]
                a, c = e[3], e[2]
                up_a, up_c = [], []
                while depth[a] > depth[c]:
                    p = parent[a]
                    up_a.append((p[0], p[1], 1.0 if p[2] == a else -1.0))
                    a = p[3] if p[2] == a else p[2]
                while depth[c] > depth[a]:
                    p = parent[c]
                    up_c.append((p[0], p[1], 1.0 if p[3] == c else -1.0))
                    c = p[3] if p[2] == c else p[2]
                while a != c:
                    p = parent[a]
                    up_a.append((p[0], p[1], 1.0 if p[2] == a else -1.0))
                    a = p[3] if p[2] == a else p[2]
                    p = parent[c]
                    up_c.append((p[0], p[1], 1.0 if p[3] == c else -1.0))
                    c = p[3] if p[2] == c else p[2]
                cycles.append(Cycle(carrier, terms + up_a + up_c))
    return cycles


def tap_ratio(tab, entity: str) -> float:
    """``Branches.tapRatio``: a missing, non-finite or non-positive tap is 1."""
    if "tap_ratio" not in tab.static:
        return 1.0
    v = float(tab.value("tap_ratio", entity))
    return v if math.isfinite(v) and v > 0.0 else 1.0


def impedance(network: Network, component: str, entity: str, carrier: str) -> float:
    """Per-unit impedance in a Kirchhoff row (``Cycles.impedance``,
    Cycles.scala:154-193): reactance in an AC sub-network, resistance in a DC
    one; a line's is referred to v_nom^2 of bus0, a transformer's to its own
    rating and tap, z tap_ratio / s_nom.  The phase shift is not read: it
    moves angles, not the optimised flows."""
    tab = network.table(component)
    raw = float(tab.value("r" if carrier == "DC" else "x", entity))
    if component == "Line":
        v = float(network.table("Bus").value("v_nom", str(tab.value("bus0", entity))))
        return raw / (v * v) if v > 0.0 else raw
    if component == "Transformer":
        s_nom = float(tab.value("s_nom", entity))
        if not s_nom > 0.0:
            raise UnsupportedNetwork(f"Transformer '{entity}' has s_nom = {s_nom}, which is its per-unit base")
        return raw * tap_ratio(tab, entity) / s_nom
    raise UnsupportedNetwork(f"{component} '{entity}' is a passive branch whose per-unit base is not known here")


def susceptance(network: Network, component: str, entity: str, carrier: str) -> float:
    """Per-unit susceptance of a branch in the outage factors
    (``Branches.susceptance``, modules/network-pf/.../Branches.scala:67-106):
    the reciprocal of the Kirchhoff-row impedance, but strict where that one
    is lenient -- a reactance (resistance in DC) that is not positive, or a
    line whose bus0 has no positive v_nom, has no susceptance and is
    refused."""
    tab = network.table(component)
    name = "r" if carrier == "DC" else "x"
    z = float(tab.value(name, entity))
    if not z > 0.0:
        raise UnsupportedNetwork(f"{component} '{entity}' has {name} = {z} in a {carrier} sub-network, so it has "
                                 "no susceptance")
    if component == "Line":
        bus0 = str(tab.value("bus0", entity))
        v = float(network.table("Bus").value("v_nom", bus0))
        if not v > 0.0:
            raise UnsupportedNetwork(f"bus '{bus0}' has v_nom = {v}, so Line '{entity}' has no per-unit base; "
                                     "every branch in a sub-network must share one")
        return v * v / z
    return 1.0 / impedance(network, component, entity, carrier)


def build(network: Network) -> Model:
    network = standard_types.expand(network)  # impedance named by type (Lopf.scala:73)
    _reject(network)
    T = len(network.snapshots)
    if T == 0:
        raise UnsupportedNetwork("network has no snapshots")
    buses = network.table("Bus").ids
    if not buses:
        raise UnsupportedNetwork("network has no buses")
    gens, lines, links, loads = (network.table(c) for c in ("Generator", "Line", "Link", "Load"))
    units, stores = network.table("StorageUnit"), network.table("Store")
    columns, bounds, costs = {}, [], []

    def declare(component, entity, t, lo, hi, cost):
        columns[(component, entity, t)] = len(bounds)
        bounds.append((lo, hi))
        costs.append(cost)

    # capacity columns first, one per extendable entity over the horizon
    expandable = [(c, network.table(c), [i for i in network.table(c).ids if extendable(network.table(c), i)])
                  for c in EXPANSION_ORDER]
    expandable = [(c, tab, ids) for c, tab, ids in expandable if ids]
    for c, tab, ids in expandable:
        nom = NOMINAL[c]
        for i in ids:
            declare(f"{c}-{nom}", i, -1, float(tab.value(f"{nom}_min", i)), float(tab.value(f"{nom}_max", i)),
                    periodized_cost(tab, i))

    for t in range(T):
        w = network.weighting("objective", t)
        for g in gens.ids:
            if extendable(gens, g):
                declare("Generator", g, t, -math.inf, math.inf, gens.at("marginal_cost", g, t) * w)
                continue
            pn = float(gens.value("p_nom", g))
            lo, hi = pn * gens.at("p_min_pu", g, t), pn * gens.at("p_max_pu", g, t)
            declare("Generator", g, t, min(lo, hi), max(lo, hi), gens.at("marginal_cost", g, t) * w)
        for comp in PASSIVE:  # a symmetric rating on the flow p0 (Lopf.scala:174-186)
            tab = network.table(comp)
            for l in tab.ids:
                if extendable(tab, l):
                    declare(comp, l, t, -math.inf, math.inf, 0.0)
                    continue
                lim = float(tab.value("s_nom", l)) * tab.at("s_max_pu", l, t)
                declare(comp, l, t, -lim, lim, 0.0)
        for k in links.ids:
            if extendable(links, k):
                declare("Link", k, t, -math.inf, math.inf, links.at("marginal_cost", k, t) * w)
                continue
            pn = float(links.value("p_nom", k))
            lo, hi = pn * links.at("p_min_pu", k, t), pn * links.at("p_max_pu", k, t)
            declare("Link", k, t, min(lo, hi), max(lo, hi), links.at("marginal_cost", k, t) * w)
        for u in units.ids:  # four non-negative variables per unit (Lopf.scala:200-240)
            pn = float(units.value("p_nom", u))
            ext = extendable(units, u)
            upper = (lambda v: math.inf) if ext else (lambda v: pn * v)
            declare("StorageUnit-p_dispatch", u, t, 0.0, upper(units.at("p_max_pu", u, t)),
                    units.at("marginal_cost", u, t) * w)
            declare("StorageUnit-p_store", u, t, 0.0, upper(-units.at("p_min_pu", u, t)), 0.0)
            declare("StorageUnit-state_of_charge", u, t, 0.0, upper(float(units.value("max_hours", u))),
                    units.at("marginal_cost_storage", u, t) * w)
            declare("StorageUnit-spill", u, t, 0.0, max(0.0, units.at("inflow", u, t)), units.at("spill_cost", u, t) * w)
        for s_ in stores.ids:  # energy and one signed, unrated power (Lopf.scala:242-265)
            if extendable(stores, s_):
                lo, hi = -math.inf, math.inf
            else:
                e_nom = float(stores.value("e_nom", s_))
                lo, hi = e_nom * stores.at("e_min_pu", s_, t), e_nom * stores.at("e_max_pu", s_, t)
            declare("Store-e", s_, t, min(lo, hi), max(lo, hi), stores.at("marginal_cost_storage", s_, t) * w)
            declare("Store-p", s_, t, -math.inf, math.inf, stores.at("marginal_cost", s_, t) * w)

    b = LpBuilder(len(bounds))
    for j, (lo, hi) in enumerate(bounds):
        b.bounds(j, lo, hi)
    for j, c in enumerate(costs):
        b.objective_coefficient(j, c)
    constant = sum(periodized_cost(tab, i) * float(tab.value(NOMINAL[c], i)) for c, tab, ids in expandable for i in ids)
    b.objective_offset(-constant)  # PyPSA reports the cost of the change (Lopf.scala:255-262)

    # what each bus sees, grouped once rather than scanned per bus and snapshot
    attached = {bus: {"gen": [], "unit": [], "store": [], "load": [], "branch": []} for bus in buses}
    for g in gens.ids:
        attached[str(gens.value("bus", g))]["gen"].append(g)
    for u in units.ids:
        attached[str(units.value("bus", u))]["unit"].append(u)
    for s_ in stores.ids:
        attached[str(stores.value("bus", s_))]["store"].append(s_)
    for d in loads.ids:
        attached[str(loads.value("bus", d))]["load"].append(d)
    for comp in PASSIVE + ("Link",):  # the branches the model builds (a process is refused)
        tab = network.table(comp)
        ports = link_ports(tab) if comp == "Link" else ["bus0", "bus1"]  # a line's flow has two ends
        for e in tab.ids:  # bus0 first, so a branch looping onto one bus lists -1 then its efficiency
            for port in ports:
                bus = tab.endpoint(port, e)  # '' for a port this link leaves unconnected
                if bus in attached:
                    attached[bus]["branch"].append((comp, e, port))

    balance_rows, row = {}, 0
    for t in range(T):
        for bus in buses:
            at = attached[bus]
            terms = [(columns[("Generator", g, t)], 1.0) for g in at["gen"]]
            for u in at["unit"]:
                terms.append((columns[("StorageUnit-p_dispatch", u, t)], 1.0))
                terms.append((columns[("StorageUnit-p_store", u, t)], -1.0))
            terms += [(columns[("Store-p", s_, t)], 1.0) for s_ in at["store"]]
            for comp, e, port in at["branch"]:
                col = columns[(comp, e, t)]
                if port == "bus0":  # flow enters the branch at bus0
                    terms.append((col, -1.0))
                else:  # and arrives at every other port scaled by that port's efficiency
                    terms.append((col, port_efficiency(links, e, port, t) if comp == "Link" else 1.0))
            demand = sum(loads.at("p_set", d, t) for d in at["load"])
            b.equality_constraint(terms, demand)
            balance_rows[(bus, t)] = row
            row += 1

    # state of charge, the one constraint coupling snapshots (Lopf.scala:336-395)
    for u in units.ids:
        cyclic = bool(units.value("cyclic_state_of_charge", u))
        initial = float(units.value("state_of_charge_initial", u))
        for t in range(T):
            eh = network.weighting("stores", t)
            eff_d, eff_s = units.at("efficiency_dispatch", u, t), units.at("efficiency_store", u, t)
            if not eff_d > 0.0:
                raise UnsupportedNetwork(f"StorageUnit '{u}' has efficiency_dispatch = {eff_d} at snapshot {t}")
            stand = math.pow(1.0 - units.at("standing_loss", u, t), eh)
            terms = [(columns[("StorageUnit-state_of_charge", u, t)], 1.0),
                     (columns[("StorageUnit-p_dispatch", u, t)], eh / eff_d),
                     (columns[("StorageUnit-p_store", u, t)], -eh * eff_s),
                     (columns[("StorageUnit-spill", u, t)], eh)]
            prev = t - 1 if t > 0 else (T - 1 if cyclic else None)
            if prev is not None:
                terms.append((columns[("StorageUnit-state_of_charge", u, prev)], -stand))
            b.equality_constraint(terms, eh * units.at("inflow", u, t) + (initial if prev is None else 0.0))
            target = units.at("state_of_charge_set", u, t)
            if math.isfinite(target):
                b.equality_constraint([(columns[("StorageUnit-state_of_charge", u, t)], 1.0)], target)

    cycles = cycle_basis(network)
    imp = {(c, e): impedance(network, c, e, cy.carrier) for cy in cycles for c, e, _ in cy.terms}
    for cy in cycles:
        if not any(imp[(c, e)] != 0.0 for c, e, _ in cy.terms):
            raise UnsupportedNetwork("every branch in a cycle has zero impedance, so Kirchhoff's voltage law "
                                     "would impose nothing on it")
    for t in range(T):
        for cy in cycles:
            b.equality_constraint([(columns[(c, e, t)], o * imp[(c, e)]) for c, e, o in cy.terms], 0.0)

    # a store's energy: e(t) = (1 - standing_loss)^eh e(t-1) - eh p(t) (Lopf.scala:440-467)
    for s_ in stores.ids:
        cyclic = bool(stores.value("e_cyclic", s_)) is True
        initial = float(stores.value("e_initial", s_))
        for t in range(T):
            eh = network.weighting("stores", t)
            stand = math.pow(1.0 - stores.at("standing_loss", s_, t), eh)
            terms = [(columns[("Store-e", s_, t)], 1.0), (columns[("Store-p", s_, t)], eh)]
            prev = t - 1 if t > 0 else (T - 1 if cyclic else None)
            if prev is not None:
                terms.append((columns[("Store-e", s_, prev)], -stand))
            b.equality_constraint(terms, initial if prev is None else 0.0)

    # capacity coupling, after every equality block (Lopf.scala:453-478)
    for c, tab, ids in expandable:
        nom = NOMINAL[c]
        for i in ids:
            cap = columns[(f"{c}-{nom}", i, -1)]
            for t in range(T):
                if c in PASSIVE:
                    mx = tab.at("s_max_pu", i, t)
                    pairs = [(c, -mx, mx)]
                elif c == "StorageUnit":
                    pairs = [("StorageUnit-p_dispatch", -math.inf, tab.at("p_max_pu", i, t)),
                             ("StorageUnit-p_store", -math.inf, -tab.at("p_min_pu", i, t)),
                             ("StorageUnit-state_of_charge", -math.inf, float(tab.value("max_hours", i)))]
                elif c == "Store":
                    pairs = [("Store-e", tab.at("e_min_pu", i, t), tab.at("e_max_pu", i, t))]
                else:
                    pairs = [(c, tab.at("p_min_pu", i, t), tab.at("p_max_pu", i, t))]
                for var, min_pu, max_pu in pairs:
                    col = columns[(var, i, t)]
                    if math.isfinite(max_pu):
                        b.less_than([(col, 1.0), (cap, -max_pu)], 0.0)
                    if math.isfinite(min_pu):
                        b.greater_than([(col, 1.0), (cap, -min_pu)], 0.0)

    constraints = network.table("GlobalConstraint")
    carriers = network.table("Carrier")
    for gc in constraints.ids:
        kind, sense = str(constraints.value("type", gc)), str(constraints.value("sense", gc))
        if kind != "primary_energy":
            raise UnsupportedNetwork(f"global constraint '{gc}' has type '{kind}'; only 'primary_energy' is implemented")
        if sense != "<=":
            raise UnsupportedNetwork(f"global constraint '{gc}' has sense '{sense}'; only '<=' is implemented")
        attribute = str(constraints.value("carrier_attribute", gc))
        terms = []
        for t in range(T):
            w = network.weighting("generators", t)
            for g in gens.ids:
                carrier = str(gens.value("carrier", g))
                intensity = float(carriers.value(attribute, carrier)) if carrier in carriers.ids else 0.0
                if not math.isfinite(intensity):
                    intensity = 0.0
                eff = gens.at("efficiency", g, t)
                if intensity != 0.0 and eff != 0.0:
                    terms.append((columns[("Generator", g, t)], intensity / eff * w))
        if terms:
            b.less_than(terms, float(constraints.value("constant", gc)))

    problem, translation = b.build()
    return Model(problem, translation, columns, balance_rows, cycles, constant, network)


def solve(network: Network, params: PdhgParams = PdhgParams(), precision: int = 64, device: int = 0,
          mixed: bool = False, ctx=None) -> LopfResult:
    """Build and solve on the GPU (``Lopf.solve``, :566-571); ``mixed`` runs
    the FP32 refinement scheme instead of plain FP64 PDHG."""
    return _solve_model(network, build(network), params, precision, device, mixed, ctx)


def _solve_model(network, model: Model, params, precision, device, mixed, ctx) -> LopfResult:
    from ..prima import cuda
    if mixed:
        sol = cuda.mixed_solve(model.problem, params, ctx=ctx, device=device).solution
    else:
        sol = cuda.solve(model.problem, params, precision=precision, device=device, ctx=ctx)
    return LopfResult(network, model, sol)


# ---- security-constrained LOPF (N-1) ------------------------------------------

class SubNetwork(tuple):
    """One island of ``sub_networks``; unpacks as (carrier, buses,
    branches) and carries ``mixed_carriers`` (``SubNetwork``,
    Topology.scala:64-75)."""

    def __new__(cls, carrier: str, buses: list, branches: list, mixed_carriers: bool = False):
        self = super().__new__(cls, (carrier, buses, branches))
        self.mixed_carriers = mixed_carriers
        return self

    carrier = property(lambda self: self[0])
    buses = property(lambda self: self[1])
    branches = property(lambda self: self[2])  # (component, id) of its passive branches, lines first


def sub_networks(network: Network) -> list:
    """``Topology.subNetworks`` (modules/network-model/.../Topology.scala:
    104-161): the buses connected over passive branches -- links join no
    islands -- with each island's buses sorted, its carrier label that of the
    first sorted bus, and the islands in order of their first bus.  An island
    whose buses disagree about carrier keeps that label and is flagged
    ``mixed_carriers``, as PyPSA warns rather than fails.  A passive branch
    table without a bus0 or bus1 column, or an endpoint that is blank or
    names no bus, raises ``MalformedNetwork``: a dropped edge would split an
    island and still look like a network."""
    bus_tab = network.table("Bus")
    if not bus_tab.ids:
        return []
    dangling = dangling_references(network, PASSIVE)
    if dangling:
        comp, i, port, bus = dangling[0]
        more = f" (and {len(dangling) - 1} other dangling reference(s))" if len(dangling) > 1 else ""
        raise MalformedNetwork(f"{comp} '{i}' references unknown bus '{bus}' via {port}{more}")
    parent = {b: b for b in bus_tab.ids}

    def find(x):
        root = x
        while parent[root] != root:
            root = parent[root]
        while parent[x] != root:  # path compression: a long radial feeder stays linear
            parent[x], x = root, parent[x]
        return root

    branches = passive_branches(network)
    for _, _, b0, b1 in branches:
        r0, r1 = find(b0), find(b1)
        if r0 != r1:
            parent[r0] = r1
    islands: dict = {}
    for b in bus_tab.ids:
        islands.setdefault(find(b), []).append(b)
    out = []
    for members in islands.values():
        buses = sorted(members)
        carriers = list(dict.fromkeys(str(bus_tab.value("carrier", b)) for b in buses))
        out.append(SubNetwork(carriers[0], buses, [], len(carriers) > 1))
    out.sort(key=lambda sub: sub.buses[0])
    island_of = {b: sub for sub in out for b in sub.buses}
    for c, i, b0, _ in branches:
        island_of[b0].branches.append((c, i))
    return out


class Lodf(tuple):
    """Outage factors of one sub-network (``Lodf``, Lodf.scala:14-66);
    unpacks as (branches, factors, populated).  ``factor(affected, outage)``
    is the share of the outaged branch's flow that reappears on the affected
    one."""

    def __new__(cls, branches: list, factors: np.ndarray, populated: np.ndarray):
        self = super().__new__(cls, (branches, factors, populated))
        self.index = {b: k for k, b in enumerate(branches)}
        return self

    branches = property(lambda self: self[0])

    def __contains__(self, branch) -> bool:
        return branch in self.index

    def _column(self, outage) -> int:
        j = self.index[outage]
        if not self[2][j]:
            raise KeyError(f"the outage column for {outage} was not computed: it was not among the requested "
                           "contingencies, so its factors were never validated")
        return j

    def factor(self, affected, outage) -> float:
        """Refuses a branch this sub-network does not hold, and a column that
        was never computed: neither is a zero."""
        for b in (affected, outage):
            if b not in self.index:
                raise KeyError(f"no branch {b} here")
        return float(self[1][self.index[affected], self._column(outage)])

    def factor_or_zero(self, affected, outage) -> float:
        """As ``factor``, but zero when either branch is in another
        sub-network, which is physically zero (``factorOrZero``)."""
        if affected not in self.index or outage not in self.index:
            return 0.0
        return float(self[1][self.index[affected], self._column(outage)])


def lodf(network: Network, carrier: str, buses: list, branches: list, outages: Optional[set] = None) -> Lodf:
    """Branch outage distribution factors of one sub-network (``Lodf.of``,
    modules/network-pf/.../Lodf.scala): PTDF = diag(b) A B^-1 with the first
    bus as reference (the factors do not depend on that choice), and
    LODF[l, o] = PTDF_l(o) / (1 - PTDF_o(o)), -1 on the diagonal, with b the
    per-unit ``susceptance``.  A bridge (a denominator within 1e-7 of zero)
    has no post-outage flow: it is refused if requested as a contingency and
    left unpopulated otherwise; a requested column with a non-finite factor
    is refused too (Lodf.scala:187-230).  ``branches`` are
    (component, id) keys.  Returns a ``Lodf``: (branches, factors m x m,
    populated per outage column), read by branch with ``factor``."""
    m = len(branches)
    if m == 0:
        return Lodf([], np.zeros((0, 0)), np.zeros(0, dtype=bool))
    index = {b: i for i, b in enumerate(buses[1:])}
    n = len(index)
    y = np.array([susceptance(network, c, i, carrier) for c, i in branches])
    A = np.zeros((m, n))
    for k, (c, i) in enumerate(branches):
        tab = network.table(c)
        b0, b1 = str(tab.value("bus0", i)), str(tab.value("bus1", i))
        if b0 in index:
            A[k, index[b0]] += 1.0
        if b1 in index:
            A[k, index[b1]] -= 1.0
    B = A.T @ (y[:, None] * A)
    try:
        np.linalg.cholesky(B)
    except np.linalg.LinAlgError as e:
        raise UnsupportedNetwork(f"sub-network {buses} has no unique power flow: {e}") from None
    ptdf = (y[:, None] * A) @ np.linalg.inv(B)       # [m branches, n buses]
    branch_ptdf = ptdf @ A.T                           # [m, m]: flow on l per unit shifted across o
    factors = np.zeros((m, m))
    populated = np.zeros(m, dtype=bool)
    for j, key in enumerate(branches):
        denominator = 1.0 - branch_ptdf[j, j]
        requested = outages is None or key in outages
        if abs(denominator) < 1e-7:
            if requested:
                raise UnsupportedNetwork(f"{key[0]} '{key[1]}' is a bridge: removing it disconnects the "
                                         "sub-network, so it is not a credible contingency")
            continue
        populated[j] = True
        factors[:, j] = branch_ptdf[:, j] / denominator
        factors[j, j] = -1.0
        if requested and not np.isfinite(factors[:, j]).all():
            raise UnsupportedNetwork(f"outage of {key[0]} '{key[1]}' gives a non-finite factor, so its "
                                     "sub-network's susceptance matrix did not solve cleanly")
    return Lodf(list(branches), factors, populated)


def _outage_key(network: Network, o) -> tuple:
    """An outage named by (component, id), or by id alone for a line (or a
    transformer when no line has that name)."""
    if isinstance(o, (tuple, list)):
        key = (str(o[0]), str(o[1]))
    else:
        key = next(((c, str(o)) for c in PASSIVE if str(o) in network.table(c).ids), ("Line", str(o)))
    if key[0] not in PASSIVE or key[1] not in network.table(key[0]).ids:
        raise UnsupportedNetwork(f"'{key[1]}' is not a passive branch of this network, so it cannot be a contingency")
    return key


def build_sclopf(network: Network, outages: Optional[list] = None) -> Model:
    """``Sclopf.build`` (modules/network-lopf/.../Sclopf.scala:80-239): the
    dispatch LP plus, per snapshot, monitored passive branch l and
    contingency o != l of its sub-network with a non-zero factor, the rating
    row -s_nom_l s_max_pu <= f_l + LODF[l, o] f_o <= s_nom_l s_max_pu.
    ``outages`` defaults to every passive branch."""
    network = standard_types.expand(network)  # factors come from the typed impedances (Sclopf.scala:84)
    base = build(network)
    if outages is not None and not outages:
        return base
    for c in PASSIVE:  # before any factor is computed (Sclopf.scala:94-127)
        tab = network.table(c)
        ext = [i for i in tab.ids if extendable(tab, i)]
        if ext:
            raise UnsupportedNetwork(f"{c} '{ext[0]}' is extendable; the security rows cap post-contingency flow "
                                     "at the rating in the file, so a secure dispatch would be priced against a "
                                     "different network")
    requested = [(c, i) for c, i, _, _ in passive_branches(network)] if outages is None else \
        [_outage_key(network, o) for o in outages]
    wanted = set(requested)
    subs = [(carrier, buses, keys, lodf(network, carrier, buses, keys, wanted))
            for carrier, buses, keys in sub_networks(network)]
    where = {}
    for s_idx, (_, _, _, (names, factors, populated)) in enumerate(subs):
        for k, key in enumerate(names):
            where[key] = (s_idx, k)
    p = base.problem
    b = LpBuilder(p.num_variables)
    for j in range(p.num_variables):
        b.bounds(j, float(p.variable_lower[j]), float(p.variable_upper[j]))
        b.objective_coefficient(j, float(p.objective[j]))
    b.objective_offset(p.objective_offset)
    K = p.constraint_matrix
    # standard-form rows that came from a <= row (copied back as <= rows)
    negated = {base.translation.expansion_of(r).row for r in range(base.translation.num_original_rows)
               if isinstance(base.translation.expansion_of(r), Negated)}
    for r in range(p.num_constraints):
        a, e = K.row_ptr[r], K.row_ptr[r + 1]
        terms = [(int(c), float(v)) for c, v in zip(K.col_indices[a:e], K.values[a:e])]
        q = float(p.rhs[r])
        if r < p.num_equalities:
            b.equality_constraint(terms, q)
        elif r in negated:
            b.less_than([(c, -v) for c, v in terms], -q)
        else:
            b.greater_than(terms, q)
    for t in range(len(network.snapshots)):
        for s_idx, (_, _, _, (names, factors, populated)) in enumerate(subs):
            for k, (c, l) in enumerate(names):
                tab = network.table(c)
                limit = float(tab.value("s_nom", l)) * tab.at("s_max_pu", l, t)
                col = base.columns[(c, l, t)]
                for o in requested:
                    if o == (c, l) or where.get(o, (None,))[0] != s_idx:
                        continue
                    j = where[o][1]
                    factor = float(factors[k, j]) if populated[j] else 0.0
                    if factor != 0.0:
                        b.constraint([(col, 1.0), (base.columns[(o[0], o[1], t)], factor)], -limit, limit)
    problem, translation = b.build()
    return Model(problem, translation, base.columns, base.balance_rows, base.cycles, base.objective_constant,
                 network)


def solve_sclopf(network: Network, outages: Optional[list] = None, params: PdhgParams = PdhgParams(),
                 precision: int = 64, device: int = 0, mixed: bool = False, ctx=None) -> LopfResult:
    """Build the security-constrained LP and solve it on the GPU
    (``Sclopf.solve``, Sclopf.scala:66-74); ``outages`` defaults to every
    passive branch, and an empty list is the dispatch model."""
    return _solve_model(network, build_sclopf(network, outages), params, precision, device, mixed, ctx)
