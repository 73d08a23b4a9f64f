"""bench.py's reference arm runs without a GPU and prints the contract's JSON
line: the oracle (the reference's FP64 PDHG restated) timed on the host."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                          "--cpu-sample-iterations", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600,
                         check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("dc-lopf")
    # the same config as the device arm, with the shape of the instance
    assert (d["config"]["n"], d["config"]["m"], d["config"]["nnz"]) == (1_344_000, 840_000, 3_024_000)
    assert d["cpu_baseline"]["extrapolated"] is True and "EXTRAPOLATED" in d["cpu_baseline"]["sample"]
    assert d["cpu_baseline"]["host_cores"] >= 1
    c1 = d["sparse_lp_measured"]
    assert c1["status"] == "OPTIMAL" and c1["time_to_tolerance_s"] > 0 and c1["iterations"] > 0


def test_highs_fixture_still_describes_the_bench_instances():
    """tests/golden/bench_highs.json holds HiGHS's optimum of the bench
    workload per seed; the generator must still build those exact bytes."""
    sys.path.insert(0, ROOT)
    from noaidi_b200.prima import generators as G
    from noaidi_b200.prima.generators import problem_hash
    fix = json.load(open(os.path.join(ROOT, "tests", "golden", "bench_highs.json")))
    assert {"0", "1", "2"} <= set(fix)
    p = G.dc_lopf(seed=0, buses=2000, lines=3000, generators=1000, snapshots=168)
    assert problem_hash(p) == fix["0"]["hash"]
    assert fix["0"]["highs_objective"] > 0
