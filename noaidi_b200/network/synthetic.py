"""Capacity-expansion LOPF with storage over a year of hours: a seeded
synthetic network and its LP.

The network: a random spanning tree plus chords (``random_network``: line
reactance U[0.01, 0.1], s_nom U[100, 1000] MW); every generator extendable
from zero at capital cost U[2e4, 1.5e5] per MW-year, a third each
dispatchable (always available, marginal cost U[0, 100]), wind (an AR(1)
availability around 0.35) and solar (the daily sine, clipped at zero, times
a slow AR(1) cloud factor), renewables at a tenth of the drawn marginal
cost; storage units of U[50, 300] MW at random buses with 0.9 efficiency
each way, 6 hours and a cyclic state of charge; one load per bus,
lognormal(3, 0.5) MW scaled by a daily sine (+-25 %) and an AR(1) noise.

``expansion_storage_network`` returns that network for the LOPF builder
(``noaidi_b200.network.lopf.build``).  ``expansion_storage`` returns the same
LP built with array operations -- the builder's layout exactly (capacity
columns first, then per snapshot generators, lines and four columns per
storage unit; bus balance, state of charge unit by unit, Kirchhoff rows,
then two capacity rows per generator and snapshot), so the result is equal
to ``lopf.build(expansion_storage_network(...)).problem`` entry for entry,
which the tests check at small sizes -- because the builder's per-entity
Python loops would take minutes and gigabytes of tuples at 8,760
snapshots.
"""
from __future__ import annotations

import math

import numpy as np

from ..prima.generators import random_network
from ..prima.model import LpProblem, SparseMatrix
from .pypsa_csv import Network, Table

EFFICIENCY = 0.9
MAX_HOURS = 6.0


def _ar1(rng, shape, phi: float, sigma: float) -> np.ndarray:
    out = np.empty(shape)
    out[0] = rng.normal(0.0, sigma / math.sqrt(1.0 - phi * phi), shape[1:])
    noise = rng.normal(0.0, sigma, shape)
    for t in range(1, shape[0]):
        out[t] = phi * out[t - 1] + noise[t]
    return out


def _draw(seed: int, buses: int, lines: int, generators: int, storage: int, snapshots: int) -> dict:
    rng = np.random.default_rng(seed)
    net = random_network(rng, buses, lines, generators)
    T, B, G = snapshots, buses, generators
    hours = np.arange(T)
    daily = np.sin(2.0 * math.pi * ((hours % 24) - 6) / 24.0)
    kind = rng.integers(0, 3, G)                      # 0 dispatchable, 1 wind, 2 solar
    wind = np.clip(0.35 + _ar1(rng, (T, G), 0.95, 0.08), 0.0, 1.0)
    cloud = np.clip(0.8 + _ar1(rng, (T, G), 0.98, 0.03), 0.2, 1.0)
    solar = np.clip(np.maximum(daily, 0.0)[:, None] * cloud, 0.0, 1.0)
    p_max_pu = np.where(kind == 0, 1.0, np.where(kind == 1, wind, solar))
    marginal = np.where(kind == 0, net.cost, 0.1 * net.cost)
    capital = rng.uniform(2e4, 1.5e5, G)
    base = rng.lognormal(3.0, 0.5, B)
    noise = np.clip(1.0 + _ar1(rng, (T, B), 0.9, 0.05), 0.2, None)
    load = base[None, :] * (1.0 + 0.25 * daily)[:, None] * noise
    unit_bus = rng.integers(0, B, storage)
    unit_p_nom = rng.uniform(50.0, 300.0, storage)
    return dict(net=net, p_max_pu=p_max_pu, marginal=marginal, capital=capital, load=load, unit_bus=unit_bus,
                unit_p_nom=unit_p_nom, T=T)


def _network(d: dict) -> Network:
    net, T = d["net"], d["T"]
    B, L, G, U = net.buses, net.lines, net.generators, len(d["unit_bus"])
    bus = [f"b{k}" for k in range(B)]
    gid, lid, uid, did = ([f"{p}{k}" for k in range(n)] for p, n in (("g", G), ("l", L), ("s", U), ("d", B)))
    tables = {
        "Bus": Table("Bus", bus, {"v_nom": dict.fromkeys(bus, 1.0)}),
        "Line": Table("Line", lid, {"bus0": {i: bus[f] for i, f in zip(lid, net.line_from)},
                                    "bus1": {i: bus[t] for i, t in zip(lid, net.line_to)},
                                    "x": dict(zip(lid, map(float, net.reactance))),
                                    "s_nom": dict(zip(lid, map(float, net.s_nom)))}),
        "Generator": Table("Generator", gid, {"bus": {i: bus[b] for i, b in zip(gid, net.gen_bus)},
                                              "p_nom": dict.fromkeys(gid, 0.0),
                                              "p_nom_extendable": dict.fromkeys(gid, True),
                                              "capital_cost": dict(zip(gid, map(float, d["capital"]))),
                                              "marginal_cost": dict(zip(gid, map(float, d["marginal"])))},
                           {"p_max_pu": d["p_max_pu"]}),
        "Load": Table("Load", did, {"bus": dict(zip(did, bus))}, {"p_set": d["load"]}),
    }
    if U:
        tables["StorageUnit"] = Table("StorageUnit", uid, {
            "bus": {i: bus[b] for i, b in zip(uid, d["unit_bus"])},
            "p_nom": dict(zip(uid, map(float, d["unit_p_nom"]))),
            "max_hours": dict.fromkeys(uid, MAX_HOURS),
            "efficiency_store": dict.fromkeys(uid, EFFICIENCY),
            "efficiency_dispatch": dict.fromkeys(uid, EFFICIENCY),
            "cyclic_state_of_charge": dict.fromkeys(uid, True)})
    return Network("expansion-storage", list(range(T)), {}, tables)


def expansion_storage_network(seed: int = 0, buses: int = 200, lines: int = 300, generators: int = 400,
                              storage: int = 50, snapshots: int = 8760) -> Network:
    return _network(_draw(seed, buses, lines, generators, storage, snapshots))


def expansion_storage(seed: int = 0, buses: int = 200, lines: int = 300, generators: int = 400, storage: int = 50,
                      snapshots: int = 8760) -> LpProblem:
    """The capacity-expansion LP with storage, equal to the LOPF builder's."""
    from .lopf import cycle_basis
    d = _draw(seed, buses, lines, generators, storage, snapshots)
    net, T = d["net"], d["T"]
    B, L, G, U = net.buses, net.lines, net.generators, len(d["unit_bus"])
    E, W = G, G + L + 4 * U                 # capacity columns; columns per snapshot
    n = E + T * W
    t_idx = np.arange(T)

    def col(local):                          # [T, k] columns of a per-snapshot local index set
        return E + t_idx[:, None] * W + np.asarray(local)[None, :]

    g_loc, l_loc = np.arange(G), G + np.arange(L)
    u_loc = G + L + 4 * np.arange(U)         # + 0 dispatch, 1 store, 2 state of charge, 3 spill

    # bounds and costs
    lower, upper, cost = np.full(n, -np.inf), np.full(n, np.inf), np.zeros(n)
    lower[:E], upper[:E], cost[:E] = 0.0, np.inf, d["capital"]
    block_lo, block_hi, block_c = np.full(W, -np.inf), np.full(W, np.inf), np.zeros(W)
    block_c[g_loc] = d["marginal"]
    block_lo[l_loc], block_hi[l_loc] = -net.s_nom, net.s_nom
    p_nom = d["unit_p_nom"]
    for k, hi in ((0, p_nom), (1, p_nom), (2, p_nom * MAX_HOURS), (3, np.zeros(U))):
        block_lo[u_loc + k], block_hi[u_loc + k] = 0.0, hi
    lower[E:], upper[E:], cost[E:] = np.tile(block_lo, T), np.tile(block_hi, T), np.tile(block_c, T)

    rr, cc, vv, rhs = [], [], [], []
    # bus balance, snapshot-major: generators +1, units +dispatch -store, lines -1 at bus0 and +1 at bus1
    ones = np.ones
    entries = [(net.gen_bus, g_loc, ones(G)), (d["unit_bus"], u_loc, ones(U)), (d["unit_bus"], u_loc + 1, -ones(U)),
               (net.line_from, l_loc, -ones(L)), (net.line_to, l_loc, ones(L))]
    for b_of, loc, val in entries:
        rr.append((t_idx[:, None] * B + b_of[None, :]).ravel())
        cc.append(col(loc).ravel())
        vv.append(np.tile(val, T))
    rhs.append(d["load"].ravel())            # one load per bus
    row0 = T * B
    # state of charge, unit-major: soc(t) + dispatch/eff - eff store + spill - soc(t-1, cyclic) = 0
    prev = np.roll(t_idx, 1)
    for k, v in ((2, 1.0), (0, 1.0 / EFFICIENCY), (1, -EFFICIENCY), (3, 1.0)):
        rr.append((row0 + np.arange(U)[:, None] * T + t_idx[None, :]).ravel())
        cc.append(col(u_loc + k).T.ravel())
        vv.append(np.full(U * T, v))
    rr.append((row0 + np.arange(U)[:, None] * T + t_idx[None, :]).ravel())
    cc.append((E + prev[None, :] * W + (u_loc + 2)[:, None]).ravel())
    vv.append(np.full(U * T, -1.0))
    rhs.append(np.zeros(U * T))
    row0 += U * T
    # Kirchhoff: per snapshot and cycle, sum of orientation x reactance x flow = 0 (v_nom = 1)
    network = _network(d)
    cycles = cycle_basis(network)
    C = len(cycles)
    cyc = [(k, int(l[1:]), o) for k, cy in enumerate(cycles) for _, l, o in cy.terms]
    ck = np.array([k for k, _, _ in cyc], dtype=np.int64)
    cl = np.array([l for _, l, _ in cyc], dtype=np.int64)
    cv = np.array([o * float(net.reactance[l]) for _, l, o in cyc])
    rr.append((row0 + t_idx[:, None] * C + ck[None, :]).ravel())
    cc.append(col(G + cl).ravel())
    vv.append(np.tile(cv, T))
    rhs.append(np.zeros(T * C))
    num_eq = row0 + T * C
    # capacity rows, generator by generator and snapshot: -p + max_pu cap >= -0, p - 0 cap >= 0
    base = num_eq + 2 * (np.arange(G)[:, None] * T + t_idx[None, :])   # [G, T]
    p_cols = col(g_loc).T                                                # [G, T]
    cap = np.broadcast_to(np.arange(G)[:, None], (G, T))
    for r_off, c_arr, v_arr in ((0, p_cols, -ones((G, T))), (0, cap, d["p_max_pu"].T), (1, p_cols, ones((G, T)))):
        rr.append((base + r_off).ravel())
        cc.append(np.ascontiguousarray(c_arr).ravel())
        vv.append(np.ascontiguousarray(v_arr).ravel())
    q = np.concatenate(rhs + [np.tile([-0.0, 0.0], G * T)])
    K = SparseMatrix.from_triplets(num_eq + 2 * G * T, n, np.concatenate(rr), np.concatenate(cc),
                                   np.concatenate(vv))
    return LpProblem(cost, K, q, num_eq, lower, upper, -0.0)
