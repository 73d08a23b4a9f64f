"""LP instances with known answers, restating the reference's test fixtures.

* ``LpFixtures`` instances (``prima-core/src/test/.../LpFixtures.scala:25-159``),
  with their hand-derived optima.
* ``random_feasible`` (``LpFixtures.scala:174-213``), which draws from
  ``scala.util.Random(seed)``, i.e. ``java.util.Random``.  :class:`JavaRandom`
  restates that generator from the Java API specification (a 48-bit linear
  congruential generator; ``nextDouble`` from 26+27 bits; ``nextGaussian`` by
  the polar method; ``nextInt(bound)`` by rejection), so the same seeds give
  the same instances as the reference's validation ladder.
* the validation ladder itself (``prima-validation/.../ValidationLadder.scala:32-38``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence

from noaidi_b200.prima.model import LpBuilder, LpProblem
from noaidi_b200.prima.types import SolveStatus

INF = math.inf
NINF = -math.inf


class JavaRandom:
    """``java.util.Random`` per its published specification."""

    MULT = 0x5DEECE66D
    ADD = 0xB
    MASK = (1 << 48) - 1

    def __init__(self, seed: int):
        self.seed = (seed ^ self.MULT) & self.MASK
        self._next_gaussian: Optional[float] = None

    def next(self, bits: int) -> int:
        self.seed = (self.seed * self.MULT + self.ADD) & self.MASK
        r = self.seed >> (48 - bits)
        if r >= 1 << 31:  # the (int) cast, which only bites when bits == 32
            r -= 1 << 32
        return r

    def next_int(self, bound: int) -> int:
        if bound <= 0:
            raise ValueError("bound must be positive")
        if bound & (-bound) == bound:  # power of two
            return (bound * self.next(31)) >> 31
        while True:
            bits = self.next(31)
            val = bits % bound
            if bits - val + (bound - 1) < (1 << 31):
                return val

    def next_double(self) -> float:
        return ((self.next(26) << 27) + self.next(27)) * (1.0 / (1 << 53))

    def next_gaussian(self) -> float:
        if self._next_gaussian is not None:
            g, self._next_gaussian = self._next_gaussian, None
            return g
        while True:
            v1 = 2 * self.next_double() - 1
            v2 = 2 * self.next_double() - 1
            s = v1 * v1 + v2 * v2
            if s < 1 and s != 0:
                break
        multiplier = math.sqrt(-2 * math.log(s) / s)
        self._next_gaussian = v2 * multiplier
        return v1 * multiplier


@dataclass
class Instance:
    name: str
    problem: LpProblem
    expected_objective: Optional[float]
    expected_primal: Optional[Sequence[float]] = None
    expected_status: SolveStatus = SolveStatus.OPTIMAL


def tiny_lower_bound() -> Instance:
    b = LpProblem.builder(1)
    b.objective_coefficient(0, 1.0)
    b.bounds(0, 0.0, 10.0)
    b.greater_than([(0, 1.0)], 3.0)
    return Instance("tiny-lower-bound", b.build()[0], 3.0, [3.0])


def product_mix() -> Instance:
    b = LpProblem.builder(2)
    b.objective_coefficient(0, -3.0)
    b.objective_coefficient(1, -5.0)
    b.bounds(0, 0.0, INF)
    b.bounds(1, 0.0, INF)
    b.less_than([(0, 1.0)], 4.0)
    b.less_than([(1, 2.0)], 12.0)
    b.less_than([(0, 3.0), (1, 2.0)], 18.0)
    return Instance("product-mix", b.build()[0], -36.0, [2.0, 6.0])


def equality_split() -> Instance:
    b = LpProblem.builder(2)
    b.objective_coefficient(0, 2.0)
    b.objective_coefficient(1, 3.0)
    b.bounds(0, 0.0, 6.0)
    b.bounds(1, 0.0, 10.0)
    b.equality_constraint([(0, 1.0), (1, 1.0)], 10.0)
    return Instance("equality-split", b.build()[0], 24.0, [6.0, 4.0])


def degenerate() -> Instance:
    b = LpProblem.builder(2)
    b.objective_coefficient(0, 1.0)
    b.objective_coefficient(1, 1.0)
    b.bounds(0, 0.0, 5.0)
    b.bounds(1, 0.0, 5.0)
    b.greater_than([(0, 1.0), (1, 1.0)], 2.0)
    b.equality_constraint([(0, 1.0), (1, -1.0)], 0.0)
    return Instance("degenerate", b.build()[0], 2.0, [1.0, 1.0])


def free_sign() -> Instance:
    b = LpProblem.builder(2)
    b.objective_coefficient(0, 1.0)
    b.objective_coefficient(1, -1.0)
    b.bounds(0, -1.0, 1.0)
    b.bounds(1, -1.0, 1.0)
    b.equality_constraint([(0, 1.0), (1, 1.0)], 0.0)
    return Instance("free-sign", b.build()[0], -2.0, [-1.0, 1.0])


def range_row() -> Instance:
    b = LpProblem.builder(2)
    b.objective_coefficient(0, 1.0)
    b.bounds(0, -10.0, 10.0)
    b.bounds(1, 0.0, 0.0)
    b.constraint([(0, 1.0), (1, 1.0)], 2.0, 5.0)
    return Instance("range-row", b.build()[0], 2.0, [2.0, 0.0])


def infeasible() -> Instance:
    b = LpProblem.builder(1)
    b.objective_coefficient(0, 1.0)
    b.bounds(0, NINF, INF)
    b.greater_than([(0, 1.0)], 1.0)
    b.less_than([(0, 1.0)], 0.0)
    return Instance("infeasible", b.build()[0], None, None, SolveStatus.PRIMAL_INFEASIBLE)


def unbounded() -> Instance:
    b = LpProblem.builder(1)
    b.objective_coefficient(0, -1.0)
    b.bounds(0, 0.0, INF)
    b.greater_than([(0, 1.0)], 0.0)
    return Instance("unbounded", b.build()[0], None, None, SolveStatus.DUAL_INFEASIBLE)


def economic_dispatch() -> Instance:
    """Two buses, one 30 MW line, three generators, two snapshots; optimum 3700
    (``LpFixtures.scala:134-159``).  Variables ``[g1, g2, g3, flow]`` per snapshot."""
    loads_a, loads_b = [100.0, 80.0], [50.0, 70.0]
    costs, caps, line = [10.0, 30.0, 20.0], [120.0, 100.0, 90.0], 30.0
    b = LpProblem.builder(8)
    for t in range(2):
        base = 4 * t
        for g in range(3):
            b.objective_coefficient(base + g, costs[g])
            b.bounds(base + g, 0.0, caps[g])
        b.bounds(base + 3, -line, line)
        b.equality_constraint([(base, 1.0), (base + 1, 1.0), (base + 3, -1.0)], loads_a[t])
        b.equality_constraint([(base + 2, 1.0), (base + 3, 1.0)], loads_b[t])
    return Instance("economic-dispatch", b.build()[0], 3700.0,
                    [120.0, 0.0, 30.0, 20.0, 110.0, 0.0, 40.0, 30.0])


def optimal() -> list[Instance]:
    return [tiny_lower_bound(), product_mix(), equality_split(), degenerate(), free_sign(), range_row(),
            economic_dispatch()]


def conclusive() -> list[Instance]:
    return optimal() + [infeasible(), unbounded()]


def random_feasible(seed: int, num_variables: int, num_equalities: int, num_inequalities: int,
                    density: float = 0.3) -> LpProblem:
    """``LpFixtures.randomFeasible`` (``LpFixtures.scala:174-213``), draw for draw."""
    rng = JavaRandom(seed)
    b = LpProblem.builder(num_variables)
    witness = [0.0] * num_variables
    for i in range(num_variables):
        lo = -10.0 + rng.next_double() * 5.0
        hi = lo + 1.0 + rng.next_double() * 20.0
        b.bounds(i, lo, hi)
        witness[i] = lo + rng.next_double() * (hi - lo)
        b.objective_coefficient(i, rng.next_gaussian() * 5.0)

    def random_row():
        row = []
        for j in range(num_variables):
            if rng.next_double() < density:
                row.append((j, rng.next_gaussian() * 2.0))
        if not row:
            row.append((rng.next_int(num_variables), 1.0))
        return row

    def value_at(row):
        # Seq[Double].sum: a left fold over the mapped values, in order
        terms = [a * witness[j] for j, a in row]
        s = terms[0]
        for t in terms[1:]:
            s = s + t
        return s

    for _ in range(num_equalities):
        row = random_row()
        b.equality_constraint(row, value_at(row))
    for _ in range(num_inequalities):
        row = random_row()
        b.greater_than(row, value_at(row) - rng.next_double() * 5.0)
    return b.build()[0]


@dataclass
class LadderEntry:
    name: str
    problem: LpProblem
    expected: SolveStatus


def ladder() -> list[LadderEntry]:
    """``ValidationLadder.entries`` (``ValidationLadder.scala:32-38``)."""
    out = [LadderEntry(i.name, i.problem, i.expected_status) for i in conclusive()]
    out.append(LadderEntry("random-60x30", random_feasible(1, 60, 10, 20, 0.25), SolveStatus.OPTIMAL))
    out.append(LadderEntry("random-200x120", random_feasible(2, 200, 40, 80, 0.10), SolveStatus.OPTIMAL))
    out.append(LadderEntry("random-600x400", random_feasible(3, 600, 120, 280, 0.04), SolveStatus.OPTIMAL))
    return out


def relative_gap(mine: float, oracle: float) -> float:
    """``ValidationLadder.relativeGap`` (``ValidationLadder.scala:45-46``)."""
    return abs(mine - oracle) / max(1.0, abs(oracle))


# Published by the reference (prima-core NOTES.md:45-58, eps = 1e-9): the
# size string, iterations, restarts and (6-decimal) objective of each ladder
# instance.  These pin the oracle's trajectory, not just its answer.
LADDER_PINS = {
    "tiny-lower-bound": ("1v/1c/1nz", 64, 0, 3.000000),
    "product-mix": ("2v/3c/4nz", 128, 1, -36.000000),
    "equality-split": ("2v/1c/2nz", 64, 0, 24.000000),
    "degenerate": ("2v/2c/4nz", 64, 0, 2.000000),
    "free-sign": ("2v/1c/2nz", 2, 0, -2.000000),
    "range-row": ("2v/2c/4nz", 64, 0, 2.000000),
    "economic-dispatch": ("8v/4c/10nz", 256, 3, 3700.000000),
    "infeasible": ("1v/2c/2nz", 1088, 5, None),
    "unbounded": ("1v/1c/1nz", 64, 0, None),
    "random-60x30": ("60v/30c/439nz", 1280, 9, -773.369199),
    "random-200x120": ("200v/120c/2464nz", 6464, 18, -1796.551031),
    "random-600x400": ("600v/400c/9529nz", 35392, 17, -5285.522448),
}
