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


def lodf_matrix(net: Network) -> tuple[np.ndarray, np.ndarray]:
    """Line outage distribution factors of a connected network (susceptance
    1/x, bus 0 as reference): LODF[l, o] = PTDF_l(o) / (1 - PTDF_o(o)) with
    -1 on the diagonal, and a mask of the lines that are not bridges."""
    B, L = net.buses, net.lines
    A = np.zeros((L, B - 1))
    idx = np.arange(L)
    f, t = net.line_from, net.line_to
    A[idx[f > 0], f[f > 0] - 1] += 1.0
    A[idx[t > 0], t[t > 0] - 1] -= 1.0
    y = 1.0 / net.reactance
    ptdf = (y[:, None] * A) @ np.linalg.inv(A.T @ (y[:, None] * A))
    branch = ptdf @ A.T
    denominator = 1.0 - np.diag(branch)
    ok = np.abs(denominator) >= 1e-7
    lodf = np.zeros((L, L))
    lodf[:, ok] = branch[:, ok] / denominator[ok]
    np.fill_diagonal(lodf, -1.0)
    return lodf, ok


def sclopf_n1(seed: int = 0, buses: int = 500, lines: int = 750, generators: int = 300, snapshots: int = 24,
              outages: int = 200, load_scale: float = 0.7, voll: float = 1000.0) -> LpProblem:
    """N-1 security-constrained DC-LOPF: ``dc_lopf`` on a
    spanning tree plus chords, and for every snapshot, monitored line l and
    contingency o != l with a non-zero factor, the rating range
    ``-s_nom_l <= f_l + LODF[l, o] f_o <= s_nom_l`` -- the reference's
    formulation (Sclopf.scala:215-236), two standard-form rows of two
    nonzeros each.  The contingencies are the ``outages`` non-bridge lines
    carrying the most flow in a DC power flow of the average hour with
    generators dispatched in proportion to availability (a seeded stand-in
    for ranking by a base solve)."""
    rng = np.random.default_rng(seed)
    net = random_network(rng, buses, lines, generators)
    base = dc_lopf(seed, buses, lines, generators, snapshots, load_scale, network=net, voll=voll)
    # the same draws dc_lopf made after the network, for the ranking flow
    rng2 = np.random.default_rng(seed)
    random_network(rng2, buses, lines, generators)
    avail = rng2.uniform(0.3, 1.0, (snapshots, generators))
    load = rng2.lognormal(3.0, 0.5, (snapshots, buses))
    load *= (load_scale * (avail * net.p_nom).sum(axis=1) / load.sum(axis=1))[:, None]
    lodf, ok = lodf_matrix(net)
    inj = np.zeros(buses)
    gen = (avail * net.p_nom).mean(axis=0)
    np.add.at(inj, net.gen_bus, gen * load.mean(axis=0).sum() / gen.sum())
    inj -= load.mean(axis=0)
    A = np.zeros((net.lines, buses - 1))
    idx = np.arange(net.lines)
    f, t = net.line_from, net.line_to
    A[idx[f > 0], f[f > 0] - 1] += 1.0
    A[idx[t > 0], t[t > 0] - 1] -= 1.0
    y = 1.0 / net.reactance
    flow = (y[:, None] * A) @ np.linalg.solve(A.T @ (y[:, None] * A), inj[1:])
    candidates = np.flatnonzero(ok)
    chosen = candidates[np.argsort(-np.abs(flow[candidates]), kind="stable")[:outages]]
    chosen.sort()
    # security pairs (l, o) with a non-zero factor, the same every snapshot
    ll, oo = np.nonzero(lodf[:, chosen] != 0.0)
    oo = chosen[oo]
    keep = ll != oo
    ll, oo = ll[keep], oo[keep]
    F = lodf[ll, oo]
    G, L, Bn, T = generators, net.lines, buses, snapshots
    nv = G + 2 * Bn + L
    F0 = G + Bn
    P = ll.size
    t_idx = np.repeat(np.arange(T), P)
    cl = (t_idx * nv + F0 + np.tile(ll, T))
    co = (t_idx * nv + F0 + np.tile(oo, T))
    fv = np.tile(F, T)
    lim = np.tile(net.s_nom[ll], T)
    # two rows per pair: (f_l + F f_o >= -s) and (-f_l - F f_o >= -s); columns ascending within a row
    first = np.minimum(cl, co)
    second = np.maximum(cl, co)
    a_first = np.where(cl < co, 1.0, fv)
    a_second = np.where(cl < co, fv, 1.0)
    nrows = 2 * P * T
    sec_cols = np.stack([first, second, first, second], axis=1).reshape(-1, 2)
    sec_vals = np.stack([a_first, a_second, -a_first, -a_second], axis=1).reshape(-1, 2)
    K0 = base.constraint_matrix
    rp = np.concatenate([K0.row_ptr, K0.nnz + 2 * np.arange(1, nrows + 1)])
    ci = np.concatenate([K0.col_indices, sec_cols.ravel()])
    vv = np.concatenate([K0.values, sec_vals.ravel()])
    K = SparseMatrix(K0.rows + nrows, K0.cols, rp, ci, vv)
    q = np.concatenate([base.rhs, -np.repeat(lim, 2)])
    return LpProblem(base.objective, K, q, base.num_equalities, base.variable_lower, base.variable_upper)
