"""Seeded synthetic LPs with the shapes and value distributions of the
benchmark workloads.  Every generator takes a seed; the same seed gives the
same bytes, so the oracle, HiGHS and the GPU see identical instances.

* :func:`random_sparse_lp` -- ``min c'x  s.t.  Ax <= b, 0 <= x <= 10``, m x n,
  ``per_column`` nonzeros per column at distinct uniform rows, N(0,1) values,
  ``b = A x0 + U[0,1]`` with ``x0 ~ U[0,10]`` (feasible), ``c ~ U[-1,1]``.
  The ``<=`` rows enter standard form negated (``LpProblem.scala:236``).
* :func:`dc_lopf` -- DC linear optimal power flow over ``T`` hourly
  snapshots in the angle formulation: dispatch ``p``, line flows ``f``,
  voltage angles ``theta`` per snapshot; nodal balance and
  ``f_l - (theta_i - theta_j)/x_l = 0`` equalities; slack bus angle fixed by
  its bounds.  Network: a random spanning tree plus chords.
* :func:`lopf_batch` -- uneven-size sweep of :func:`dc_lopf` instances.
"""
from __future__ import annotations

import dataclasses
import hashlib

import numpy as np

from .model import LpProblem, SparseMatrix


def problem_hash(p: LpProblem) -> str:
    h = hashlib.sha256()
    K = p.constraint_matrix
    for a in (K.row_ptr, K.col_indices, K.values, p.objective, p.rhs, p.variable_lower, p.variable_upper):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(np.array([p.num_equalities, p.objective_offset]).tobytes())
    return h.hexdigest()[:16]


def random_sparse_lp(seed: int = 0, m: int = 400, n: int = 600, per_column: int = 5) -> LpProblem:
    rng = np.random.default_rng(seed)
    rows = np.stack([rng.choice(m, size=per_column, replace=False) for _ in range(n)])  # n x k
    cols = np.repeat(np.arange(n), per_column)
    vals = rng.standard_normal(n * per_column)
    A = SparseMatrix.from_triplets(m, n, rows.ravel(), cols, vals)
    x0 = rng.uniform(0.0, 10.0, n)
    b = A.multiply(x0) + rng.uniform(0.0, 1.0, m)
    c = rng.uniform(-1.0, 1.0, n)
    K = SparseMatrix(m, n, A.row_ptr, A.col_indices, -A.values)
    return LpProblem(c, K, -b, 0, np.zeros(n), np.full(n, 10.0))


@dataclasses.dataclass
class Network:
    buses: int
    line_from: np.ndarray
    line_to: np.ndarray
    reactance: np.ndarray
    s_nom: np.ndarray
    gen_bus: np.ndarray
    p_nom: np.ndarray
    cost: np.ndarray

    @property
    def lines(self) -> int:
        return int(self.line_from.shape[0])

    @property
    def generators(self) -> int:
        return int(self.gen_bus.shape[0])


def random_network(rng: np.random.Generator, buses: int, lines: int, generators: int) -> Network:
    """A random spanning tree (each bus attaches to a uniformly chosen earlier
    bus) plus distinct chords up to ``lines`` branches."""
    assert lines >= buses - 1
    frm = [int(rng.integers(0, i)) for i in range(1, buses)]
    to = list(range(1, buses))
    seen = {(min(a, b), max(a, b)) for a, b in zip(frm, to)}
    while len(frm) < lines:
        a, b = (int(v) for v in rng.integers(0, buses, 2))
        if a == b or (min(a, b), max(a, b)) in seen:
            continue
        seen.add((min(a, b), max(a, b)))
        frm.append(a)
        to.append(b)
    L = len(frm)
    return Network(buses, np.array(frm, np.int64), np.array(to, np.int64), rng.uniform(0.01, 0.1, L),
                   rng.uniform(100.0, 1000.0, L), rng.integers(0, buses, generators),
                   rng.uniform(50.0, 800.0, generators), rng.uniform(0.0, 100.0, generators))


def dc_lopf(seed: int = 0, buses: int = 2000, lines: int = 3000, generators: int = 1000, snapshots: int = 168,
            load_scale: float = 0.7, network: Network | None = None, voll: float = 1000.0) -> LpProblem:
    """DC-LOPF dispatch LP.  Per snapshot the columns are ``p`` (G generators),
    ``shed`` (B buses), ``f`` (L lines), ``theta`` (B buses) and the rows are
    B nodal balances then L flow definitions, so ``n = T(G + 2B + L)``,
    ``m = T(B + L)``, ``nnz = T(G + B + 2L + 3L)``.  Loads are
    lognormal(3, 0.5) per bus-hour, rescaled each hour to ``load_scale`` times
    the available capacity; ``shed`` (load shedding at ``voll`` per MWh,
    bounded by the bus load) keeps every hour feasible under line limits."""
    rng = np.random.default_rng(seed)
    net = network or random_network(rng, buses, lines, generators)
    B, L, G, T = net.buses, net.lines, net.generators, snapshots
    avail = rng.uniform(0.3, 1.0, (T, G))
    load = rng.lognormal(3.0, 0.5, (T, B))
    load *= (load_scale * (avail * net.p_nom).sum(axis=1) / load.sum(axis=1))[:, None]

    P0, S0, F0, A0 = 0, G, G + B, G + B + L  # column offsets within a snapshot
    nv = G + 2 * B + L
    nr = B + L  # rows per snapshot: balance | flow
    inv_x = 1.0 / net.reactance
    r_flow = B + np.arange(L)
    rr = np.concatenate([net.gen_bus, np.arange(B), net.line_from, net.line_to, r_flow, r_flow, r_flow])
    cc = np.concatenate([P0 + np.arange(G), S0 + np.arange(B), F0 + np.arange(L), F0 + np.arange(L),
                         F0 + np.arange(L), A0 + net.line_from, A0 + net.line_to])
    vv = np.concatenate([np.ones(G), np.ones(B), -np.ones(L), np.ones(L), np.ones(L), -inv_x, inv_x])
    one = SparseMatrix.from_triplets(nr, nv, rr, cc, vv)
    # block-diagonal over snapshots
    nnz1 = one.nnz
    row_ptr = (np.arange(T)[:, None] * nnz1 + one.row_ptr[None, :-1]).ravel()
    row_ptr = np.append(row_ptr, T * nnz1)
    col_idx = (np.arange(T)[:, None] * nv + one.col_indices[None, :]).ravel()
    values = np.tile(one.values, T)
    K = SparseMatrix(T * nr, T * nv, row_ptr, col_idx, values)

    c = np.tile(np.concatenate([net.cost, np.full(B, voll), np.zeros(L + B)]), T)
    lo = np.concatenate([np.zeros((T, G + B)), np.tile(-net.s_nom, (T, 1)), np.full((T, B), -np.inf)], axis=1)
    hi = np.concatenate([avail * net.p_nom, load, np.tile(net.s_nom, (T, 1)), np.full((T, B), np.inf)], axis=1)
    lo[:, A0] = 0.0  # slack bus angle
    hi[:, A0] = 0.0
    q = np.concatenate([load, np.zeros((T, L))], axis=1).ravel()
    return LpProblem(c, K, q, T * nr, lo.ravel(), hi.ravel())


def lopf_batch(seed: int = 0, count: int = 256, min_buses: int = 100, max_buses: int = 2000,
               min_snapshots: int = 24, max_snapshots: int = 168) -> list[LpProblem]:
    """Scenario sweep of uneven sizes: per instance ``B ~ U{min..max}``,
    ``T ~ U{..}``, 1.5 B lines, 0.5 B generators, load scale ``U[0.6, 0.95]``,
    instance seed ``seed + i``."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        B = int(rng.integers(min_buses, max_buses + 1))
        T = int(rng.integers(min_snapshots, max_snapshots + 1))
        scale = float(rng.uniform(0.6, 0.95))
        out.append(dc_lopf(seed + i, B, (3 * B) // 2, B // 2, T, scale))
    return out
