"""MpsReaderSuite's conventions (modules/prima-mps/src/test/scala/org/noaidi/
prima/mps/MpsReaderSuite.scala) as small MPS texts with hand-derived optima,
checked through a solver passed in (the oracle on CPU, the device on GPU)."""
import math

import pytest

from noaidi_b200.prima import PdhgParams, SolveStatus
from noaidi_b200.prima.mps import MpsParseError, read_string

PARAMS = PdhgParams(eps_abs=1e-9, eps_rel=1e-9)
INF = math.inf

# min x + y s.t. x + y >= 2, x <= 3, x, y >= 0: optimum 2
BASIC = """NAME          BASIC
ROWS
 N  COST
 G  LIM1
 L  LIM2
COLUMNS
    X         COST      1.0        LIM1      1.0
    X         LIM2      1.0
    Y         COST      1.0        LIM1      1.0
RHS
    RHS       LIM1      2.0        LIM2      3.0
ENDATA
"""


def ranged(sense: str, rng: str, cost: float) -> str:
    """min cost*x over one row of the given sense with rhs 10 and a range."""
    return f"""NAME          RNG
ROWS
 N  COST
 {sense}  R1
COLUMNS
    X         COST      {cost}        R1        1.0
RHS
    RHS       R1        10.0
RANGES
    RNG       R1        {rng}
BOUNDS
 FR BND       X
ENDATA
"""


def bounds_of(lines: str):
    text = f"""NAME          BND
ROWS
 N  COST
 G  R1
COLUMNS
    X         COST      1.0        R1        1.0
RHS
    RHS       R1        -1000.0
BOUNDS
{lines}
ENDATA
"""
    p = read_string(text).problem
    return float(p.variable_lower[0]), float(p.variable_upper[0])


def run_all(solve):
    inst = read_string(BASIC)
    assert inst.name == "BASIC" and inst.column_names == ["X", "Y"] and inst.row_names == ["LIM1", "LIM2"]
    assert not inst.is_mixed_integer
    s = solve(inst.problem)
    assert s.status == SolveStatus.OPTIMAL and s.objective_value == pytest.approx(2.0, abs=1e-6)

    decorated = "\n".join(x for l in BASIC.splitlines() for x in ("* a comment", "", l.replace("    ", "\t")))
    assert solve(read_string(decorated).problem).objective_value == pytest.approx(2.0, abs=1e-6)

    # later N rows are free rows and dropped; the first is the objective
    free = BASIC.replace(" N  COST\n", " N  COST\n N  OTHER\n").replace(
        "    Y         COST      1.0        LIM1      1.0", "    Y         COST      1.0        OTHER     7.0\n"
                                                          "    Y         LIM1      1.0")
    inst = read_string(free)
    assert inst.row_names == ["LIM1", "LIM2"]
    assert solve(inst.problem).objective_value == pytest.approx(2.0, abs=1e-6)

    # an RHS on the objective row is a negated constant
    const = BASIC.replace("    RHS       LIM1      2.0        LIM2      3.0",
                          "    RHS       LIM1      2.0        LIM2      3.0\n    RHS       COST      5.0")
    assert solve(read_string(const).problem).objective_value == pytest.approx(2.0 - 5.0, abs=1e-6)

    # RANGES: G upwards, L downwards, E by the sign of the range
    opt = lambda sense, rng, cost: solve(read_string(ranged(sense, rng, cost)).problem).objective_value
    assert opt("G", "4.0", 1.0) == pytest.approx(10.0, abs=1e-6)
    assert opt("G", "4.0", -1.0) == pytest.approx(-14.0, abs=1e-6)
    assert opt("L", "4.0", 1.0) == pytest.approx(6.0, abs=1e-6)
    assert opt("L", "4.0", -1.0) == pytest.approx(-10.0, abs=1e-6)
    assert opt("E", "2.0", 1.0) == pytest.approx(10.0, abs=1e-6)
    assert opt("E", "2.0", -1.0) == pytest.approx(-12.0, abs=1e-6)
    assert opt("E", "-2.0", 1.0) == pytest.approx(8.0, abs=1e-6)
    assert opt("E", "-2.0", -1.0) == pytest.approx(-10.0, abs=1e-6)

    # bound kinds
    assert bounds_of(" UP BND       X         4.0") == (0.0, 4.0)
    assert bounds_of(" LO BND       X         -2.0") == (-2.0, INF)
    assert bounds_of(" FX BND       X         7.0") == (7.0, 7.0)
    assert bounds_of(" FR BND       X") == (-INF, INF)
    assert bounds_of(" MI BND       X") == (-INF, INF)
    assert bounds_of(" PL BND       X") == (0.0, INF)
    assert bounds_of(" BV BND       X") == (0.0, 1.0)
    assert bounds_of(" MI BND       X         0.0") == (-INF, INF)
    assert bounds_of(" FR BND       X         0.0") == (-INF, INF)
    assert bounds_of(" MI X         0.0") == (-INF, INF)
    assert bounds_of(" FR X") == (-INF, INF)
    assert bounds_of(" MI BND       X\n UP BND2      X         5.0") == (-INF, 5.0)
    assert bounds_of(" UP BND       X         -3.0") == (-INF, -3.0)
    assert bounds_of(" LO BND       X         -9.0\n UP BND       X         -3.0") == (-9.0, -3.0)

    # integer markers are recorded
    ints = """NAME          INT
ROWS
 N  COST
 G  R1
COLUMNS
    MARKER                 'MARKER'                 'INTORG'
    X         COST      1.0        R1        1.0
    MARKER                 'MARKER'                 'INTEND'
    Y         COST      1.0        R1        1.0
RHS
    RHS       R1        1.0
ENDATA
"""
    inst = read_string(ints)
    assert inst.is_mixed_integer and inst.integer_columns == {0}

    # duplicate objective coefficients accumulate: 3 per unit, x = 5
    dup = """NAME          DUP
ROWS
 N  COST
 G  R1
COLUMNS
    X         COST      1.0
    X         COST      2.0        R1        1.0
RHS
    RHS       R1        5.0
ENDATA
"""
    assert solve(read_string(dup).problem).objective_value == pytest.approx(15.0, abs=1e-6)

    # an infeasible file parses and solves to PrimalInfeasible
    infeas = """NAME          INFEAS
ROWS
 N  COST
 G  R1
 L  R2
COLUMNS
    X         COST      1.0        R1        1.0
    X         R2        1.0
RHS
    RHS       R1        5.0        R2        1.0
BOUNDS
 FR BND       X
ENDATA
"""
    assert solve(read_string(infeas).problem).status == SolveStatus.PRIMAL_INFEASIBLE


def check_rejections():
    bad = [
        "ROWS\n X  BAD\nENDATA\n",
        "ROWS\n G  R1\nENDATA\n",
        "ROWS\n N  C\n G  R1\nCOLUMNS\n    X    NOSUCHROW   1.0\nENDATA\n",
        "ROWS\n N  C\n G  R1\nCOLUMNS\n    X    R1   notanumber\nENDATA\n",
        "ROWS\n N  C\n G  R1\nCOLUMNS\n    X    R1   1.0\nBOUNDS\n UP BND  NOSUCHCOL  4.0\nENDATA\n",
        "ROWS\n N  C\n G  R1\nCOLUMNS\n    X    R1   1.0\n    Y    R1   1.0\nBOUNDS\n UP BND  X  4.0  Y  5.0\nENDATA\n",
        "OBJSENSE\n    MAX\nROWS\n N  C\n G  R1\nCOLUMNS\n    X    R1   1.0\nENDATA\n",
    ]
    for text in bad:
        with pytest.raises(MpsParseError):
            read_string(text)
