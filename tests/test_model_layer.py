"""The C++ model layer (MPS reader and presolve in libprima_cuda.so) against
the Python restatements in oracle/ on seeded random inputs: the same LP,
row translation, names and integer columns from every MPS text, the same
reductions, maps and reduced problem from every presolve, bit for bit, and
the same restored solutions."""
import math

import numpy as np
import pytest

from noaidi_b200.prima import mps as product_mps
from noaidi_b200.prima import presolve as product_presolve
from noaidi_b200.prima.model import LpBuilder

NUMBERS = ["1", "2.5", "-3", ".5", "4.", "1e1", "2.5E-1", "-1.5e+2", "3d", "0.75f", "0x1p-2", "-0x1.8p1", "7D"]


def _same_problem(a, b):
    assert (a.num_variables, a.num_constraints, a.num_equalities) == (b.num_variables, b.num_constraints,
                                                                       b.num_equalities)
    Ka, Kb = a.constraint_matrix, b.constraint_matrix
    for x, y in ((Ka.row_ptr, Kb.row_ptr), (Ka.col_indices, Kb.col_indices), (Ka.values, Kb.values),
                 (a.rhs, b.rhs), (a.objective, b.objective), (a.variable_lower, b.variable_lower),
                 (a.variable_upper, b.variable_upper)):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    assert a.objective_offset == b.objective_offset or (math.isnan(a.objective_offset) and
                                                        math.isnan(b.objective_offset))


def random_mps(seed: int) -> str:
    rng = np.random.default_rng(seed)
    num = lambda: NUMBERS[rng.integers(len(NUMBERS))]
    rows = [(f"r{i}", "LGE"[rng.integers(3)]) for i in range(int(rng.integers(2, 7)))]
    cols = [f"x{j}" for j in range(int(rng.integers(2, 8)))]
    eol = ["\n", "\r\n", "\r"][rng.integers(3)]
    out = [f"NAME rand{seed}", "* a comment", "ROWS", " N cost"]
    out += [f" {s}{chr(9) if rng.random() < 0.3 else ' '}{r}" for r, s in rows]
    spare = rng.random() < 0.5
    if spare:
        out.append(" N spare")  # a free row: dropped
    out.append("COLUMNS")
    marker = False
    for j, c in enumerate(cols):
        if rng.random() < 0.3 and not marker:
            out.append("    MARKER                 'MARKER'                 'INTORG'")
            marker = True
        entries = [("cost", num())] + [(r, num()) for r, _ in rows if rng.random() < 0.5]
        if spare and rng.random() < 0.3:
            entries.append(("spare", num()))
        if rng.random() < 0.2 and len(entries) > 1:
            entries.append(entries[1])  # a duplicate entry: summed
        for k in range(0, len(entries), 2):
            pair = entries[k:k + 2]
            out.append(f"    {c}  " + "  ".join(f"{a} {b}" for a, b in pair))
        if marker and rng.random() < 0.5:
            out.append("    MARKER                 'MARKER'                 'INTEND'")
            marker = False
    out.append("")
    out.append("RHS")
    for r, _ in rows:
        if rng.random() < 0.7:
            out.append(f"    {'RHS ' if rng.random() < 0.5 else ''}{r} {num()}")
    if rng.random() < 0.5:
        out.append(f"    RHS cost {num()}")
    out.append("RANGES")
    for r, _ in rows:
        if rng.random() < 0.3:
            out.append(f"    RNG {r} {num()}")
    out.append("BOUNDS")
    for c in cols:
        kind = ["UP", "LO", "FX", "FR", "MI", "PL", "BV", "LI", "UI", None][rng.integers(10)]
        if kind is None:
            continue
        value = num()
        if kind in ("LO", "LI"):
            value = "-" + value.lstrip("-")
        if kind in ("FR", "MI", "PL", "BV"):
            out.append(f" {kind} BND {c}" + (f" {value}" if rng.random() < 0.3 else ""))
        else:
            out.append(f" {kind} {'BND ' if rng.random() < 0.5 else ''}{c} {value}")
    out.append("ENDATA")
    return eol.join(out) + eol


def _read_both(text):
    from oracle import mps as oracle_mps
    results = []
    for reader, error in ((product_mps.read_string, product_mps.MpsParseError),
                          (oracle_mps.read_string, oracle_mps.MpsParseError)):
        try:
            results.append(("ok", reader(text, "fallback")))
        except error as e:
            results.append(("parse", str(e)))
        except ValueError as e:
            results.append(("value", str(e)))
    return results


@pytest.mark.parametrize("seed", range(60))
def test_random_mps_texts_read_alike(seed):
    (ka, a), (kb, b) = _read_both(random_mps(seed))
    assert ka == kb, (a, b)
    if ka != "ok":
        return
    assert (a.name, a.row_names, a.column_names, a.integer_columns) == (b.name, b.row_names, b.column_names,
                                                                        b.integer_columns)
    assert a.translation._expansions == b.translation._expansions
    _same_problem(a.problem, b.problem)


MALFORMED = [
    "ROWS\n N c\nCOLUMNS\n x c inf\n",                      # not a Java number
    "ROWS\n N c\nCOLUMNS\n x c 1 r 2\n",                    # unknown row
    "ROWS\n N c\n Q r\n",                                    # unknown row type
    "ROWS\n L r\nCOLUMNS\n x r 1\n",                         # no objective row
    "ROWS\n N c\nCOLUMNS\n x c\n",                           # malformed COLUMNS entry
    "ROWS\n N c\nCOLUMNS\n x c 1 c\n",                       # unpaired field
    "ROWS\n N c\nCOLUMNS\n x c 1\nBOUNDS\n UP BND y 1\n",     # bound on an undeclared column
    "ROWS\n N c\nCOLUMNS\n x c 1\nBOUNDS\n UP A B x 1\n",    # too many fields
    "ROWS\n N c\nCOLUMNS\n x c 1\nBOUNDS\n XX BND x 1\n",    # unknown bound type
    "NAME t\nOBJSENSE MAX\nROWS\n N c\n",                    # maximisation refused
    "NAME t\nOBJSENSE\n    MAXIMIZE\nROWS\n N c\n",          # ... also on its own line
    "ROWS\n N c\nCOLUMNS\n x c 1\nSOS\n S1 x 1\n",           # unexpected section data
    "ROWS\n N c\nCOLUMNS\n x c 1\nBOUNDS\n LO BND x 5\n UP BND x 1\n",  # empty bounds
    "ROWS\n N c\nCOLUMNS\n x c 1\nBOUNDS\n UP BND x 1e\n",   # exponent without digits
]


@pytest.mark.parametrize("text", MALFORMED)
def test_malformed_texts_are_refused_alike(text):
    (ka, a), (kb, b) = _read_both(text)
    assert ka == kb != "ok", (a, b)
    if "number" in b or "row" in b or "BOUNDS" in b or "section" in b:
        assert a == b


@pytest.mark.parametrize("token", ["1", "-2.5", ".5", "5.", "1e3", "1E-3", "+4d", "2f", "0x1p3", "0X.8P-1",
                                   "-0x1.8p1D", "NaN", "-Infinity", "+Infinity", "inf", "nan", "1e", "e1", ".",
                                   "0x1", "0x1p", "1d5", "++1", "1_0", "0b1", "Infinityd"])
def test_numbers_follow_javas_grammar_alike(token):
    from oracle import mps as oracle_mps
    text = f"ROWS\n N c\nCOLUMNS\n x c {token}\n"
    (ka, a), (kb, b) = _read_both(text)
    assert ka == kb
    want = oracle_mps.java_double(token)
    assert (want is None) == (ka == "parse")
    if ka == "ok":
        got = a.problem.objective[0]
        assert (math.isnan(got) and math.isnan(want)) or got == want


def test_line_endings_and_tabs_read_alike():
    base = "NAME t\nROWS\n N c\n L r\nCOLUMNS\n\tx c 1 r 2\nRHS\n RHS r 4\nENDATA\n"
    got = [product_mps.read_string(base.replace("\n", eol)) for eol in ("\n", "\r\n", "\r")]
    for g in got[1:]:
        _same_problem(got[0].problem, g.problem)
    assert got[0].row_names == ["r"] and got[0].column_names == ["x"]


def test_read_file_takes_the_base_name(tmp_path):
    path = tmp_path / "tiny.mps"
    path.write_text("ROWS\n N c\n G r\nCOLUMNS\n x c 1 r 1\nRHS\n RHS r 2\nENDATA\n")
    inst = product_mps.read_file(str(path))
    assert inst.name == "tiny.mps" and inst.problem.num_constraints == 1


# ---- presolve -----------------------------------------------------------------

def random_reducible_lp(seed: int):
    """Fixed columns, singleton rows of both senses and signs, empty rows
    and columns, and rows that only empty out once other reductions ran."""
    rng = np.random.default_rng(seed)
    n, m = int(rng.integers(8, 40)), int(rng.integers(5, 30))
    b = LpBuilder(n)
    x0 = rng.uniform(-2, 5, n)
    for j in range(n):
        b.objective_coefficient(j, float(rng.choice([0.0, rng.normal()])))
        kind = rng.integers(5)
        if kind == 0:
            b.bounds(j, float(x0[j]), float(x0[j]))                       # fixed
        elif kind == 1:
            b.bounds(j, -math.inf, math.inf)
        elif kind == 2:
            b.bounds(j, float(x0[j] - 3), float(x0[j] + 3))
        elif kind == 3:
            b.bounds(j, float(min(0.0, x0[j])), math.inf)
        else:
            b.bounds(j, -math.inf, float(max(0.0, x0[j]) + 1))
    for _ in range(m):
        k = int(rng.choice([0, 1, 1, 2, 3, 4]))
        cols = rng.choice(n, size=min(k, n), replace=False)
        terms = [(int(j), float(rng.choice([-2.0, -1.0, 0.5, 1.0, 3.0]))) for j in cols]
        act = sum(a * x0[j] for j, a in terms)
        sense = rng.integers(3)
        if sense == 0:
            b.equality_constraint(terms, float(act))
        elif sense == 1:
            b.greater_than(terms, float(act - rng.uniform(0, 1)))
        else:
            b.less_than(terms, float(act + rng.uniform(0, 1)))
    if rng.random() < 0.15:  # a contradiction: presolve proves infeasibility
        j = int(rng.integers(n))
        b.greater_than([(j, 1.0)], 1e6)
        b.less_than([(j, 1.0)], -1e6)
    return b.build()[0]


@pytest.mark.parametrize("seed", range(80))
def test_random_presolves_reduce_alike(seed):
    from oracle import presolve as oracle_presolve
    p = random_reducible_lp(seed)
    a, b = product_presolve.presolve(p), oracle_presolve.presolve(p)
    assert a.stats == b.stats
    assert (a.proven_infeasible, a.unbounded_if_feasible) == (b.proven_infeasible, b.unbounded_if_feasible)
    if a.proven_infeasible:
        with pytest.raises(RuntimeError):
            a.reduced
        return
    assert np.array_equal(a.column_map, b.column_map) and np.array_equal(a.row_map, b.row_map)
    _same_problem(a.reduced, b.reduced)
    # restore the same made-up reduced solution both ways
    from noaidi_b200.prima.types import KktError, LpSolution, SolveStatus
    rng = np.random.default_rng(1000 + seed)
    r = a.reduced
    sol = LpSolution(SolveStatus.OPTIMAL, rng.normal(size=r.num_variables), rng.normal(size=r.num_constraints),
                     rng.normal(size=r.num_variables), 0.0, 0.0, 1, 0, 0, KktError(0.0, 0.0, 0.0, 0.0))
    ra, rb = a.restore(sol), b.restore(sol)
    assert ra.status == rb.status
    for x, y in ((ra.primal, rb.primal), (ra.dual, rb.dual), (ra.reduced_costs, rb.reduced_costs)):
        np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-12)
    assert ra.objective_value == pytest.approx(rb.objective_value, rel=1e-12, abs=1e-12)


def test_presolve_of_a_million_column_lp_is_quick():
    """The config-2 DC-LOPF (1.34M columns, 3.0M nonzeros) presolves in the
    C++ layer without a per-row interpreter loop: the slack angle columns
    are fixed and their entries fold into the flow rows."""
    import time
    from noaidi_b200.prima import generators as G
    p = G.dc_lopf(seed=0)
    t0 = time.perf_counter()
    r = product_presolve.presolve(p)
    took = time.perf_counter() - t0
    assert r.stats.fixed_columns >= 168 and not r.proven_infeasible
    assert r.reduced.num_variables == p.num_variables - r.stats.fixed_columns - r.stats.empty_columns
    assert took < 30.0, took
