"""Generates ladder_envelope.json: for each ladder instance whose trajectory
is not reproduced bit for bit, the iteration counts the oracle itself gives
when one objective coefficient is moved by one ulp (12 coefficients, both
directions alternately).

These instances are chaotic in the last bit: a 1-ulp change of a single
input (or of the summation order of a dot product, or of one pow result)
moves the iteration count by up to several times.  The spread is the yardstick
for the device's count, which differs from the oracle's in exactly such
last-bit details.

    python tests/golden/make_ladder_envelope.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from noaidi_b200.prima import LpProblem, PdhgParams  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests import lp_fixtures as F  # noqa: E402

P9 = PdhgParams(eps_abs=1e-9, eps_rel=1e-9, max_iterations=500_000)
CHAOTIC = ("infeasible", "random-60x30", "random-200x120", "random-600x400")
PERTURBATIONS = 12


def perturbed(p, k):
    c = p.objective.copy()
    j = (k * 7919) % len(c)
    c[j] = np.nextafter(c[j], np.inf if k % 2 else -np.inf)
    return LpProblem(c, p.constraint_matrix, p.rhs, p.num_equalities, p.variable_lower, p.variable_upper,
                     p.objective_offset)


def main():
    out = {}
    for e in F.ladder():
        if e.name not in CHAOTIC:
            continue
        base = O.solve(e.problem, P9)
        its = [O.solve(perturbed(e.problem, k), P9).iterations for k in range(PERTURBATIONS)]
        out[e.name] = {"iterations": base.iterations, "perturbed": sorted(its)}
        print(e.name, out[e.name], flush=True)
    with open(os.path.join(HERE, "ladder_envelope.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
