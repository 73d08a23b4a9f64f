"""The mixed-integer ladder of the reference's cross-solver check
(modules/prima-validation/src/test/scala/org/noaidi/prima/validation/
MilpLadder.scala:14-130): hand-sized instances whose relaxations are all
fractional, so agreement exercises the search, and the seeded random mixed
generator (``scala.util.Random`` is ``java.util.Random``), with the shared
branch-and-bound settings."""
from dataclasses import dataclass

import numpy as np

from noaidi_b200.prima import LpProblem, PdhgParams
from noaidi_b200.prima.bnb import BnbParams
from tests.lp_fixtures import JavaRandom

PARAMS = BnbParams(lp=PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=200_000), max_nodes=50_000)


@dataclass
class Instance:
    name: str
    problem: LpProblem
    integers: set


def fractional_pair() -> Instance:
    """maximise 5a + 4b s.t. 6a + 4b <= 24, a + 2b <= 6: relaxation
    (3, 1.5) at -21, integer optimum (4, 0) at -20 (:18-33)."""
    b = LpProblem.builder(2)
    b.objective_coefficient(0, -5.0).objective_coefficient(1, -4.0)
    b.bounds(0, 0.0, 10.0).bounds(1, 0.0, 10.0)
    b.less_than([(0, 6.0), (1, 4.0)], 24.0)
    b.less_than([(0, 1.0), (1, 2.0)], 6.0)
    return Instance("fractional-pair", b.build()[0], {0, 1})


def knapsack(name, values, weights, capacity) -> Instance:
    """0/1 knapsack as a minimisation of minus the value (:35-42)."""
    n = len(values)
    b = LpProblem.builder(n)
    for i, v in enumerate(values):
        b.objective_coefficient(i, -float(v)).bounds(i, 0.0, 1.0)
    b.less_than([(i, float(w)) for i, w in enumerate(weights)], float(capacity))
    return Instance(name, b.build()[0], set(range(n)))


def set_cover(name, sets, elements) -> Instance:
    """Fewest sets covering every element, >= rows (:49-66)."""
    b = LpProblem.builder(len(sets))
    for j in range(len(sets)):
        b.objective_coefficient(j, 1.0).bounds(j, 0.0, 1.0)
    for e in range(elements):
        covering = [(j, 1.0) for j, s in enumerate(sets) if e in s]
        if not covering:
            raise ValueError(f"{name}: element {e} is covered by no set")
        b.greater_than(covering, 1.0)
    return Instance(name, b.build()[0], set(range(len(sets))))


def random_mixed(seed: int, n: int, m: int) -> Instance:
    """Half the columns integer (the even ones), <= rows drawn at density 0.6
    (:71-83), in the reference's draw order."""
    rng = JavaRandom(seed)
    b = LpProblem.builder(n)
    for j in range(n):
        b.objective_coefficient(j, -(1.0 + rng.next_int(9)))
        b.bounds(j, 0.0, 1.0 + rng.next_int(3))
    for _ in range(m):
        terms = [(j, 1.0 + float(rng.next_int(5))) for j in range(n) if rng.next_double() < 0.6]
        if terms:
            b.less_than(terms, 3.0 + rng.next_int(10))
    return Instance(f"random-mixed-{seed}", b.build()[0], {j for j in range(n) if j % 2 == 0})


def instances() -> list:
    """The ladder (:107-130)."""
    k5 = [{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 0}, {0, 2}, {1, 3}, {2, 4}, {3, 0}, {4, 1}]
    return [
        fractional_pair(),
        knapsack("knapsack-8", [10, 13, 18, 31, 7, 15, 22, 9], [3, 4, 5, 9, 2, 5, 7, 3], 17.0),
        knapsack("knapsack-16", [41, 50, 49, 59, 45, 47, 12, 33, 21, 44, 51, 19, 28, 37, 40, 25],
                 [31, 27, 12, 34, 22, 19, 8, 16, 11, 24, 29, 9, 14, 20, 23, 13], 120.0),
        set_cover("set-cover-triangle", [{0, 1}, {1, 2}, {0, 2}], 3),
        set_cover("set-cover-k5-edges", k5, 5),
        random_mixed(1, 8, 4),
        random_mixed(9, 10, 5),
        random_mixed(3, 12, 6),
        random_mixed(4, 14, 7),
    ]


def highs_milp(problem: LpProblem, integers: set):
    """The independent exact MILP solver standing in for ojAlgo's: scipy's
    HiGHS branch-and-cut on the same standard form.  Returns (status,
    objective) with status "optimal", "infeasible" or something else."""
    from scipy.optimize import Bounds, LinearConstraint, milp
    K = problem.constraint_matrix.to_dense()
    q = np.asarray(problem.rhs)
    ne = problem.num_equalities
    lower = q.copy()
    upper = np.where(np.arange(len(q)) < ne, q, np.inf)
    integrality = np.array([1 if j in integers else 0 for j in range(problem.num_variables)])
    constraints = [LinearConstraint(K, lower, upper)] if K.shape[0] else []
    res = milp(np.asarray(problem.objective), constraints=constraints, integrality=integrality,
               bounds=Bounds(np.asarray(problem.variable_lower), np.asarray(problem.variable_upper)),
               options={"mip_rel_gap": 0.0})
    status = {0: "optimal", 2: "infeasible"}.get(res.status, f"status {res.status}")
    return status, (float(res.fun) + problem.objective_offset if res.status == 0 else None)
