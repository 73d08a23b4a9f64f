"""Time-to-tolerance benchmark of the B200 PDHG path.

Workload (N=1): the 1.34M-variable synthetic DC-LOPF dispatch LP (2,000 buses,
3,000 lines, 1,000 generators, 168 hourly snapshots, seeded), solved to a
relative KKT tolerance of 1e-8 by FP32 PDHG with FP64 refinement on the
device.  A "step" is one full solve.  With N GPUs every rank solves its own
instance (seed = rank): independent LPs, no collective on the data path
(weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value   whole-job LPs/s; each step is one prima_problem_mixed_solve on a
        problem already resident (and equilibrated) on the device, timed with
        CUDA events on the library's stream; max over ranks.
e2e     the same metric through the one-shot C-ABI call with host buffers
        (upload, device equilibration, both passes, download of x, y and the
        reduced costs inside the timed region), on the first --e2e-steps steps.
fp64    plain FP64 device PDHG (the reference algorithm, ScalaKernels
        semantics) on the same instance, solved to the same tolerance in full
        once per run: its time, iteration count, status and objective.
error   the refinement's objective against that FP64 answer and against
        HiGHS's optimum of the instance (tests/golden/bench_highs.json, made
        by tests/golden/make_bench_fixtures.py).
batch   (--batch K, 256 by default) the uneven sweep of K DC-LOPF instances,
        FP32 refinement to 1e-6, one launch per pass: LPs/s, its own
        roofline, a CPU estimate and errors against HiGHS on a sample.
sparse_lp the 600-column random sparse LP solved to 1e-6 by the device and by
        the oracle on a host core, both measured in full.

``--impl reference`` times the CPU restatement of the reference FP64 PDHG
(single-threaded, like the reference's ScalaKernels backend) on a bounded
sample of the same instance on the host cores, rank 0 only, and solves the
600-column LP to tolerance in full.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LPs/s to 1e-8 relative KKT: FP32+FP64-refinement PDHG on the 1.3M-variable DC-LOPF"
UNIT = "LPs/s"
EPS = 1e-8
WORKLOAD = dict(buses=2000, lines=3000, generators=1000, snapshots=168)
WORKLOAD_NAME = "dc-lopf-2000bus-3000line-1000gen-168h (n=1,344,000 m=840,000 nnz=3,024,000)"
# Iterations the plain FP64 device PDHG needed to reach 1e-8 on the seed-0
# instance in a full solve (the default run measures it again and reports the
# count it saw); only the reference arm, which runs without a GPU, uses this.
FP64_ITERATIONS_TO_TOLERANCE = 1_104_256
ROUND_REDUCTION = 10.0
BATCH_EPS = 1e-6
SPARSE_LP = dict(m=400, n=600, per_column=5)
SPARSE_LP_EPS = 1e-6
# DRAM bytes (read + write) per step-size trial of pdhg_kernel<float> on this
# workload: dram__bytes_read.sum + dram__bytes_write.sum of an ncu capture of
# one plain FP32 solve of 200 trials on it, 29.69 GB / 200.  The refinement's
# anchored trials also read the dual bound (m words, 3.4 MB more at most).
TRAFFIC_BYTES_PER_TRIAL = 148.5e6


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "MEASURED_PEAKS.json hbm_gbs"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback 6.65 TB/s"


def host_info():
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"host_cores": os.cpu_count(), "cpu_model": model}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [num(r[0]) for r in self.rows if num(r[0]) is not None]
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = sorted({self.NAMES[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": num(self.rows[0][1]), "reasons": reasons,
                "samples": len(self.rows), "power_w_max": max(num(r[2]) or 0.0 for r in self.rows)}


def algorithmic_bytes(problem, trials: int, iterations: int, word: int, anchored: bool = False) -> float:
    """Compulsory HBM bytes of the fused iteration, per trial: an accepted trial streams both matrices once (index + value
    per nonzero, one row pointer per row), gathers the other side's vector
    once, and moves 13n + 11m vector words (x, c, l, u, K'y, x', xbar, the
    two column running sums read+write; y, kx, q, y', kx', the two row sums
    read+write); a rejected trial has no K'y product and no running sums
    (7n + 6m words, one matrix).  The residual problem's dual bound adds m
    words per trial in anchored mode."""
    K = problem.constraint_matrix
    n, m, nnz = problem.num_variables, problem.num_constraints, K.nnz
    extra = m * word if anchored else 0
    acc = (13 * n + 11 * m) * word + 2 * nnz * (4 + word) + 4 * (n + m) + extra
    rej = (7 * n + 6 * m) * word + nnz * (4 + word) + 4 * m + extra
    return acc * iterations + rej * max(0, trials - iterations)


def bench_config(problem, eps, world, round_reduction):
    K = problem.constraint_matrix
    return {"workload": WORKLOAD_NAME, "n": problem.num_variables, "m": problem.num_constraints, "nnz": int(K.nnz),
            "eps": eps, "seed": "rank", "parallelism": f"independent instances x{world}",
            "scheme": f"fp32 pass + fp32 refinement around an fp64 anchor, round reduction {round_reduction:g}",
            "l2": "working set larger than L2 (no flush needed)"}


def highs_reference(seed, problem):
    """HiGHS's optimum of the bench instance with this seed, if recorded for
    exactly these bytes."""
    from noaidi_b200.prima.generators import problem_hash
    try:
        rec = json.load(open(os.path.join(ROOT, "tests", "golden", "bench_highs.json"))).get(str(seed))
    except (OSError, ValueError):
        return None
    if not rec or rec.get("hash") != problem_hash(problem):
        return None
    return float(rec["highs_objective"])


def rel_err(a, b):
    return None if a is None or b is None else abs(a - b) / max(1.0, abs(b))


# ---- CPU legs (the oracle: test infrastructure, timed as the CPU baseline) ----

def cpu_sample(problem, iters: int, repeats: int = 1):
    """The oracle (reference FP64 PDHG restated in C, one thread) for a fixed
    number of iterations: seconds per iteration, setup (equilibration) taken
    out by differencing against a one-iteration run."""
    from noaidi_b200.prima import PdhgParams
    from oracle import oracle as O
    times = []
    for _ in range(repeats):
        t = time.perf_counter()
        O.solve(problem, PdhgParams(eps_abs=EPS, eps_rel=EPS, max_iterations=1))
        t1 = time.perf_counter() - t
        t = time.perf_counter()
        s = O.solve(problem, PdhgParams(eps_abs=EPS, eps_rel=EPS, max_iterations=iters))
        tn = time.perf_counter() - t
        times.append(max(tn - t1, 1e-9) / max(1, s.iterations - 1))
    return float(np.median(times)), s.iterations


def sparse_lp_problem():
    from noaidi_b200.prima import generators as G
    return G.random_sparse_lp(seed=0, **SPARSE_LP)


def sparse_lp_oracle():
    """The 600-column LP solved to 1e-6 by the oracle on one host core, in full."""
    from noaidi_b200.prima import PdhgParams
    from oracle import oracle as O
    p = sparse_lp_problem()
    params = PdhgParams(eps_abs=SPARSE_LP_EPS, eps_rel=SPARSE_LP_EPS, max_iterations=1_000_000)
    O.solve(p, params.copy(max_iterations=64))  # warm the library
    t = time.perf_counter()
    s = O.solve(p, params)
    secs = time.perf_counter() - t
    return {"seconds": secs, "iterations": s.iterations, "status": s.status.name, "objective": s.objective_value}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from noaidi_b200.prima import generators as G
    problem = G.dc_lopf(seed=0, **WORKLOAD)
    for _ in range(min(args.warmup, 1)):
        cpu_sample(problem, 1)
    per_iter, done = cpu_sample(problem, args.cpu_sample_iterations, args.steps)
    iters = FP64_ITERATIONS_TO_TOLERANCE
    lps = 1.0 / (per_iter * iters)
    hi = host_info()
    c1 = sparse_lp_oracle()
    line = {"impl": "reference", "metric": METRIC, "value": lps, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / lps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(problem, EPS, world, args.round_reduction),
            "cpu_baseline": {"value": lps, "unit": UNIT, "cores": 1, **hi, "kind": "port", "extrapolated": True,
                             "sample": f"EXTRAPOLATED, not solved: {done} FP64 PDHG iterations per step of the seed-0 "
                                       f"instance on one host core (the oracle, Pdhg.Solve + ScalaKernels restated "
                                       f"in C, single-threaded like the reference), {per_iter * 1e3:.1f} "
                                       f"ms/iteration, times the {iters} iterations the same algorithm needed on the "
                                       f"device in FP64 to reach 1e-8 (a full run of that solve on the CPU would "
                                       f"take about {per_iter * iters / 3600:.1f} h)"},
            "e2e": {"value": lps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "sparse_lp_measured": {"workload": "random sparse LP m=400 n=600 (5 nonzeros per column), seed 0",
                                 "eps": SPARSE_LP_EPS, "cores": 1, "time_to_tolerance_s": c1["seconds"],
                                 "iterations": c1["iterations"], "status": c1["status"],
                                 "objective": c1["objective"], "lps_per_s": 1.0 / c1["seconds"]}}
    print(json.dumps(line), flush=True)


def _oracle_seconds_per_iteration(spec, iters: int = 16) -> float:
    """One instance on one host core: FP64 PDHG iterations of the oracle,
    setup taken out by differencing against a one-iteration run."""
    from noaidi_b200.prima import PdhgParams, generators as G
    from oracle import oracle as O
    problem = G.dc_lopf(*spec)
    t = time.perf_counter()
    O.solve(problem, PdhgParams(eps_abs=BATCH_EPS, eps_rel=BATCH_EPS, max_iterations=1))
    t1 = time.perf_counter() - t
    t = time.perf_counter()
    s = O.solve(problem, PdhgParams(eps_abs=BATCH_EPS, eps_rel=BATCH_EPS, max_iterations=iters))
    return max(time.perf_counter() - t - t1, 1e-9) / max(1, s.iterations - 1)


def _batch_specs(seed: int, count: int, min_buses=100, max_buses=2000, min_snapshots=24, max_snapshots=168):
    """The (seed, buses, lines, generators, snapshots, load scale) of each
    instance of ``generators.lopf_batch``, drawn the same way."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        B = int(rng.integers(min_buses, max_buses + 1))
        T = int(rng.integers(min_snapshots, max_snapshots + 1))
        scale = float(rng.uniform(0.6, 0.95))
        out.append((seed + i, B, (3 * B) // 2, B // 2, T, scale))
    return out


def _highs_lopf(spec):
    """HiGHS's optimum of one batch instance, snapshot by snapshot (nothing
    couples the snapshots of a dispatch LP)."""
    from noaidi_b200.prima import generators as G
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_bench_fixtures import highs_by_snapshot
    return highs_by_snapshot(G.dc_lopf(*spec), spec[4])


def batch_cpu_baseline(pool, specs, nnz, iterations, sample: int = 8):
    """``PrimaZio.solveAll``'s CPU shape -- one single-threaded FP64 solve per
    host core at a time -- estimated from a bounded sample: up to ``sample``
    instances spread over the sizes are timed per iteration in parallel
    processes (spawned, so none inherits a GPU context); seconds per
    iteration per nonzero from them, times each instance's nonzeros and the
    iterations its device solve took, summed over the instances and shared
    over the cores."""
    cores = os.cpu_count() or 1
    order = sorted(range(len(specs)), key=lambda i: nnz[i])
    picks = sorted({order[round(k * (len(order) - 1) / max(1, sample - 1))] for k in range(min(sample, len(order)))})
    per_iter = pool.map(_oracle_seconds_per_iteration, [specs[i] for i in picks])
    rate = float(np.median([t / nnz[i] for t, i in zip(per_iter, picks)]))
    cpu_seconds = sum(rate * nnz[i] * iterations[i] for i in range(len(specs))) / cores
    return {"value": len(specs) / cpu_seconds, "unit": "LPs/s", "cores": cores, "kind": "port", "extrapolated": True,
            "sample": f"ESTIMATED: {len(picks)} of the instances timed over 16 FP64 PDHG iterations each on the "
                      f"oracle, one process per instance; {rate * 1e9:.2f} ns per nonzero-iteration extrapolated to "
                      f"every instance's nonzeros and the iterations its device solve took, over {cores} cores"}


def run_batch(args, rank, world, dist, pool):
    """The batch sweep: an uneven sweep of ``--batch`` DC-LOPF instances (buses
    U{100..2000}, snapshots U{24..168}, load scale U[0.6, 0.95], seeded), FP32
    refinement to 1e-6, each pass one launch for all of this rank's
    instances (host buffers in and out: upload, equilibration and download
    are inside the wall time).  Ranks take longest-processing-time shards;
    LPs/s is all instances over the slowest rank's device span."""
    import torch
    from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, cuda, generators as G
    from noaidi_b200.prima.sharding import instance_size, shard
    problems = G.lopf_batch(seed=0, count=args.batch)
    specs = _batch_specs(0, args.batch)
    mine = shard([instance_size(p) for p in problems], world)[rank]
    params = PdhgParams(eps_abs=BATCH_EPS, eps_rel=BATCH_EPS, max_iterations=args.max_iterations)
    mixed = MixedPrecisionParams(reduced_max_iterations=args.max_iterations)
    ctx = cuda.Context(int(os.environ.get("LOCAL_RANK", "0")), 32)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t = time.perf_counter()
    res = cuda.mixed_solve_batch([problems[i] for i in mine], params, mixed, scheme=cuda.MIXED_REFINEMENT,
                                 round_reduction=args.round_reduction, ctx=ctx) if mine else []
    torch.cuda.synchronize()
    secs = time.perf_counter() - t
    span = max((r.solution.span_ms for r in res), default=0.0) / 1e3
    kern = max((r.solution.device_ms for r in res), default=0.0) / 1e3
    agg = torch.tensor([span, secs], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(agg, op=dist.ReduceOp.MAX)
    ctx.close()
    its = [r.reduced_iterations + r.refinement_iterations for r in res]
    statuses = sorted({r.solution.status.name for r in res})
    out = {"workload": f"batch sweep: {args.batch} uneven DC-LOPF instances (buses U{{100..2000}}, snapshots "
                       f"U{{24..168}}), FP32 refinement to {BATCH_EPS:g}",
           "instances": args.batch, "lps_per_s": args.batch / float(agg[0]), "seconds": float(agg[0]),
           "wall_seconds": float(agg[1]), "statuses_rank0": statuses,
           "iterations_rank0": {"min": int(min(its)), "median": float(np.median(its)), "max": int(max(its))}
           if its else None,
           "columns": int(sum(p.num_variables for p in problems)),
           "nnz": int(sum(p.constraint_matrix.nnz for p in problems))}
    if rank == 0 and res:
        pk, pk_src = peaks()
        byts = sum(algorithmic_bytes(problems[i], r.solution.trials, r.reduced_iterations + r.refinement_iterations,
                                     4, anchored=True) for i, r in zip(mine, res))
        achieved = byts / max(kern, 1e-9) / 1e9 if kern > 0 else None
        out["roofline"] = {"kernel": "pdhg_batch_kernel<float>", "bound": "hbm", "achieved": achieved,
                           "peak": pk["hbm_gbs"], "unit": "GB/s",
                           "frac": achieved / pk["hbm_gbs"] if achieved else None, "peak_source": pk_src,
                           "note": "algorithmic bytes of every instance's trials over the longest pass sum of device "
                                   "time (the launches of one pass run concurrently)"}
        # errors against HiGHS on the three smallest instances of this rank
        small = sorted(range(len(mine)), key=lambda k: instance_size(problems[mine[k]]))[:3]
        highs = pool.map(_highs_lopf, [specs[mine[k]] for k in small]) if pool else []
        errs = [rel_err(res[k].solution.objective_value, h) for k, h in zip(small, highs)]
        out["error_vs_highs"] = {"instances": [int(mine[k]) for k in small],
                                 "objective_rel_err_max": max(errs) if errs else None}
        if not args.skip_cpu:
            out["cpu_baseline"] = batch_cpu_baseline(pool, [specs[i] for i in mine],
                                                     [problems[i].constraint_matrix.nnz for i in mine], its)
    return out


def profile_problem(workload: str, snapshots: int):
    """The LP of a named workload: the DC-LOPF dispatch (optionally fewer
    snapshots), the N-1 security-constrained LOPF, or the capacity-expansion
    LOPF with storage over 8,760 hours."""
    from noaidi_b200.prima import generators as G
    if workload == "sclopf-n1":
        return G.sclopf_n1(seed=0)
    if workload == "expansion-storage":
        from noaidi_b200.network.synthetic import expansion_storage
        return expansion_storage(seed=0)
    return G.dc_lopf(seed=0, **dict(WORKLOAD, snapshots=snapshots))


def run_profile_case(args) -> None:
    """A bounded run for profilers and per-trial timing: the workload
    resident on the device, one plain PDHG solve capped at
    --profile-iterations iterations in the chosen precision, or with
    --profile-mixed the FP32 refinement scheme to --profile-tolerance."""
    from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, cuda
    t0 = time.perf_counter()
    problem = profile_problem(args.profile_workload, args.profile_snapshots)
    build_s = time.perf_counter() - t0
    eps = args.profile_tolerance
    params = PdhgParams(eps_abs=eps, eps_rel=eps, max_iterations=args.profile_iterations)
    out = {"profile_case": True, "workload": args.profile_workload, "n": problem.num_variables,
           "m": problem.num_constraints, "nnz": problem.constraint_matrix.nnz, "build_s": build_s, "eps": eps}
    ctx = cuda.Context(0, 32 if args.profile_mixed else args.profile_precision)
    if args.profile_layout:
        ctx.set_solver_layout(*[int(v) for v in args.profile_layout.split(",")])
    if args.profile_mixed:
        resident = cuda.DeviceProblem(problem, params, ctx=ctx)
        scheme = cuda.MIXED_TWO_PASS if args.profile_scheme == "two-pass" else cuda.MIXED_REFINEMENT
        r = resident.mixed_solve(params, MixedPrecisionParams(reduced_max_iterations=params.max_iterations),
                                 scheme=scheme, round_reduction=args.round_reduction, want_solution=False)
        s = r.solution
        out.update(precision="fp32+fp64", scheme=args.profile_scheme, round_reduction=args.round_reduction,
                   reduced_iterations=r.reduced_iterations, refinement_iterations=r.refinement_iterations)
    else:
        resident = cuda.DeviceProblem(problem, params, ctx=ctx)
        s = resident.solve(params, want_solution=False)
        out.update(precision=args.profile_precision)
    out.update(status=s.status.name, objective=s.objective_value, iterations=s.iterations, trials=s.trials,
               blocks=s.blocks, tile_rows=s.tile_rows, device_s=s.device_ms / 1e3, us_per_trial=1e3 * s.device_ms / max(1, s.trials))
    resident.free()
    print(json.dumps(out), flush=True)


def spmv_bytes(rows, cols, nnz, word):
    """Compulsory bytes of one SpMV: each nonzero's index and value, the row
    pointers, the input vector once and the output vector."""
    return nnz * (word + 4) + 4 * (rows + 1) + word * cols + word * rows


def run_spmv_case(args) -> None:
    """The seam's Kernels.spmv on the bench workload's equilibration-free K
    (m x n) and its transpose, in both precisions: --spmv-reps calls each,
    back to back on the context's stream, timed from the host around the
    whole run (launch-bound when a call is shorter than its submission).  For
    device-side times run it under ncu's launch list; the line gives each
    matrix's compulsory bytes to divide by them."""
    from noaidi_b200.prima import cuda, generators as G
    p = G.dc_lopf(seed=0, **WORKLOAD)
    K = p.constraint_matrix
    Kt = K.transpose
    out = {"spmv_case": True, "reps": args.spmv_reps, "matrices": {}}
    for prec in (32, 64):
        k = cuda.CudaKernels(0, prec)
        for name, A in (("K", K), ("Kt", Kt)):
            dA = k.upload_matrix(A)
            x = k.upload(np.random.default_rng(0).standard_normal(A.cols))
            y = k.allocate(A.rows)
            k.spmv(dA, x, y)
            k.dot(y, y)  # synchronises
            t = time.perf_counter()
            for _ in range(args.spmv_reps):
                k.spmv(dA, x, y)
            k.dot(y, y)
            secs = (time.perf_counter() - t) / args.spmv_reps
            byts = spmv_bytes(A.rows, A.cols, A.nnz, prec // 8)
            out["matrices"][f"{name}_fp{prec}"] = {"rows": A.rows, "cols": A.cols, "nnz": int(A.nnz),
                                                   "bytes": byts, "host_us_per_call": secs * 1e6,
                                                   "host_gbs": byts / secs / 1e9}
        k.close()
    print(json.dumps(out), flush=True)


def run_fp64_study(args) -> None:
    """The FP32 refinement against plain FP64 device PDHG, both solved to
    --eps in full, on every seed of --fp64-study: times, iterations, statuses,
    objectives and the speed-up per seed and its median (one JSON line)."""
    from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, cuda, generators as G
    seeds = [int(s) for s in args.fp64_study.split(",")]
    params = PdhgParams(eps_abs=args.eps, eps_rel=args.eps, max_iterations=args.max_iterations)
    mixed = MixedPrecisionParams(reduced_max_iterations=args.max_iterations)
    rows = []
    for seed in seeds:
        p = G.dc_lopf(seed=seed, **WORKLOAD)
        r32 = cuda.DeviceProblem(p, params, ctx=cuda.Context(0, 32))
        r = r32.mixed_solve(params, mixed, scheme=cuda.MIXED_REFINEMENT, round_reduction=args.round_reduction,
                            want_solution=False)
        r32.free()
        r64 = cuda.DeviceProblem(p, params, ctx=cuda.Context(0, 64))
        f = r64.solve(params, want_solution=False)
        r64.free()
        h = highs_reference(seed, p)
        rows.append({"seed": seed, "refinement_s": r.solution.span_ms / 1e3, "fp64_s": f.span_ms / 1e3,
                     "speedup": f.span_ms / r.solution.span_ms, "refinement_iterations":
                     [r.reduced_iterations, r.refinement_iterations], "fp64_iterations": f.iterations,
                     "status": [r.solution.status.name, f.status.name],
                     "objective": [r.solution.objective_value, f.objective_value],
                     "rel_err_vs_fp64": rel_err(r.solution.objective_value, f.objective_value),
                     "rel_err_vs_highs": [rel_err(r.solution.objective_value, h), rel_err(f.objective_value, h)]})
        print(json.dumps(rows[-1]), flush=True)
    print(json.dumps({"fp64_study": rows, "eps": args.eps,
                      "median_speedup": float(np.median([r["speedup"] for r in rows]))}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--max-iterations", type=int, default=5_000_000)
    ap.add_argument("--eps", type=float, default=EPS, help="relative KKT tolerance of the timed solves")
    ap.add_argument("--round-reduction", type=float, default=ROUND_REDUCTION)
    ap.add_argument("--e2e-steps", type=int, default=3,
                    help="one-shot solves with host buffers for the e2e figure (at most --steps)")
    ap.add_argument("--skip-fp64", action="store_true", help="leave out the full FP64 comparison solve")
    ap.add_argument("--cpu-sample-iterations", type=int, default=128)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--batch", type=int, default=256,
                    help="the batch sweep: solve this many uneven LOPF instances to 1e-6 as batches and report LPs/s under "
                         "'batch' (0: off)")
    ap.add_argument("--fp64-study", default="",
                    help="comma-separated seeds: only compare the refinement with plain FP64, both in full, per seed")
    ap.add_argument("--spmv-reps", type=int, default=0,
                    help="only time the seam SpMV on the workload's K and K' (this many calls each) and exit")
    ap.add_argument("--profile-iterations", type=int, default=0,
                    help="only run this many PDHG iterations of the workload (a bounded case for ncu) and exit")
    ap.add_argument("--profile-precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--profile-snapshots", type=int, default=WORKLOAD["snapshots"])
    ap.add_argument("--profile-workload", default="dc-lopf", choices=["dc-lopf", "sclopf-n1", "expansion-storage"])
    ap.add_argument("--profile-mixed", action="store_true")
    ap.add_argument("--profile-scheme", default="refinement", choices=["refinement", "two-pass"],
                    help="with --profile-mixed: FP32 refinement around an FP64 anchor, or the reference's FP32 "
                         "pass then FP64 finish")
    ap.add_argument("--profile-tolerance", type=float, default=EPS)
    ap.add_argument("--profile-layout", default="",
                    help="BLOCKS_PER_SM,TILE_ROWS: pin the solver's layout instead of choosing it by timing")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_iterations:
        return run_profile_case(args)
    if args.spmv_reps:
        return run_spmv_case(args)
    if args.fp64_study:
        return run_fp64_study(args)

    import multiprocessing as mp

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # the CPU legs run in spawned processes (none inherits a GPU context),
    # started before the first GPU call
    pool = mp.get_context("spawn").Pool(max(1, min(8, os.cpu_count() or 1))) if rank == 0 else None
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, cuda, generators as G

    problem = G.dc_lopf(seed=rank, **WORKLOAD)
    eps = args.eps
    params = PdhgParams(eps_abs=eps, eps_rel=eps, max_iterations=args.max_iterations)
    mixed = MixedPrecisionParams(reduced_max_iterations=args.max_iterations)
    ctx32 = cuda.Context(local, 32)
    resident = cuda.DeviceProblem(problem, params, ctx=ctx32)

    def step_resident():
        return resident.mixed_solve(params, mixed, scheme=cuda.MIXED_REFINEMENT,
                                    round_reduction=args.round_reduction, want_solution=False)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    for _ in range(args.warmup):
        step_resident()
    barrier()
    results = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            results.append(step_resident())
        barrier()
    span_s = sum(r.solution.span_ms for r in results) / 1e3
    kern_s = sum(r.solution.device_ms for r in results) / 1e3

    # CPU legs on the host cores while the device runs the comparison solves
    cpu_jobs = {}
    if pool is not None and not args.skip_cpu:
        cpu_jobs["sparse_lp"] = pool.apply_async(sparse_lp_oracle)

    # end to end through the one-shot C ABI call with host buffers
    barrier()
    e2e, e2e_steps = [], max(1, min(args.e2e_steps, args.steps))
    for _ in range(e2e_steps):
        t = time.perf_counter()
        r_e2e = cuda.mixed_solve(problem, params, mixed, scheme=cuda.MIXED_REFINEMENT,
                                 round_reduction=args.round_reduction, ctx=ctx32)
        e2e.append(time.perf_counter() - t)
    barrier()

    agg = torch.tensor([span_s, sum(e2e)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(agg, op=dist.ReduceOp.MAX)
    max_span, max_e2e = float(agg[0]), float(agg[1])

    # plain FP64 device PDHG on the same instance, solved in full
    fp64 = None
    if not args.skip_fp64:
        ctx64 = cuda.Context(local, 64)
        res64 = cuda.DeviceProblem(problem, params, ctx=ctx64)
        fp64 = res64.solve(params, want_solution=False)
        res64.free()
        ctx64.close()

    # the 600-column random sparse LP on the device to 1e-6, one-shot calls
    c1p = sparse_lp_problem()
    c1params = PdhgParams(eps_abs=SPARSE_LP_EPS, eps_rel=SPARSE_LP_EPS, max_iterations=1_000_000)
    cuda.mixed_solve(c1p, c1params, ctx=ctx32)  # warm
    t = time.perf_counter()
    c1_dev = cuda.mixed_solve(c1p, c1params, scheme=cuda.MIXED_REFINEMENT, ctx=ctx32)
    c1_dev_s = time.perf_counter() - t
    c1_64 = cuda.solve(c1p, c1params, precision=64)

    batch_line = run_batch(args, rank, world, dist, pool) if args.batch else None

    if rank == 0:
        pk, pk_src = peaks()
        n, m, nnz = problem.num_variables, problem.num_constraints, problem.constraint_matrix.nnz
        last = results[-1]
        sol = last.solution
        steps = args.steps
        line = {
            "metric": METRIC if eps == EPS else METRIC.replace("1e-8", f"{eps:g}"), "value": steps * world / max_span,
            "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * max_span / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 iterate, f64 anchor/KKT", "data": "synthetic",
            "config": bench_config(problem, eps, world, args.round_reduction),
            "clocks": clocks.summary(),
            "e2e": {"value": e2e_steps * world / max_e2e, "unit": UNIT, "steps": e2e_steps,
                    "h2d_bytes_per_step": int(nnz * 12 + (m + 1) * 4 + 8 * (3 * n + m)),
                    "d2h_bytes_per_step": int(8 * (2 * n + m))},
            "gpu_launches": 2 * steps,
            "solution": {"status": sol.status.name, "objective": sol.objective_value,
                         "primal_residual": sol.kkt.primal_residual_norm,
                         "dual_residual": sol.kkt.dual_residual_norm, "gap": sol.kkt.absolute_gap,
                         "fp32_pass_iterations": last.reduced_iterations,
                         "refinement_iterations": last.refinement_iterations,
                         "rounds": last.refinement_rounds, "layout": {"blocks": sol.blocks, "tile_rows": sol.tile_rows},
                         "e2e_status": r_e2e.solution.status.name},
        }
        h = highs_reference(0, problem) if rank == 0 else None
        line["error"] = {"objective_rel_err_vs_highs": rel_err(sol.objective_value, h), "highs_objective": h}
        iters64 = FP64_ITERATIONS_TO_TOLERANCE
        if fp64 is not None:
            iters64 = fp64.iterations
            fp64_s = fp64.span_ms / 1e3
            line["fp64_baseline"] = {
                "measured": "full solve to tolerance, once per run", "time_to_tolerance_ms": 1e3 * fp64_s,
                "device_ms": fp64.device_ms, "iterations_to_tolerance": fp64.iterations,
                "ms_per_iteration": fp64.device_ms / max(1, fp64.iterations), "status": fp64.status.name,
                "objective": fp64.objective_value, "status_identical": fp64.status == sol.status,
                "speedup_of_fp32_refinement": fp64_s / (max_span / steps)}
            line["error"]["objective_rel_err_vs_fp64"] = rel_err(sol.objective_value, fp64.objective_value)
            line["error"]["fp64_objective_rel_err_vs_highs"] = rel_err(fp64.objective_value, h)
        trials32 = sum(r.solution.trials for r in results)
        iters32 = sum(r.reduced_iterations + r.refinement_iterations for r in results)
        byts = algorithmic_bytes(problem, trials32, iters32, 4, anchored=True)
        achieved = byts / kern_s / 1e9
        line["roofline"] = {"kernel": "pdhg_kernel<float>", "bound": "hbm", "achieved": achieved,
                            "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                            "traffic": TRAFFIC_BYTES_PER_TRIAL * trials32 / len(results) if TRAFFIC_BYTES_PER_TRIAL else None,
                            "peak_source": pk_src,
                            "per_trial_bytes": byts / max(1, trials32), "kernel_ms": 1e3 * kern_s / steps}
        c1 = cpu_jobs["sparse_lp"].get() if "sparse_lp" in cpu_jobs else None
        line["sparse_lp"] = {"workload": "random sparse LP m=400 n=600 (5 nonzeros per column), seed 0",
                           "eps": SPARSE_LP_EPS, "device_refinement_s": c1_dev_s,
                           "device_status": c1_dev.solution.status.name,
                           "device_iterations": [c1_dev.reduced_iterations, c1_dev.refinement_iterations],
                           "device_fp64_s": c1_64.solve_time_millis / 1e3, "device_fp64_iterations": c1_64.iterations,
                           "oracle": c1, "measured": "every figure a full solve to tolerance"}
        if batch_line:
            line["batch"] = batch_line
        if not args.skip_cpu:
            per_iter, done = cpu_sample(problem, args.cpu_sample_iterations)
            lps = 1.0 / (per_iter * iters64)
            line["cpu_baseline"] = {"value": lps, "unit": UNIT, "cores": 1, **host_info(), "kind": "port",
                                    "extrapolated": True,
                                    "sample": f"EXTRAPOLATED, not solved: {done} FP64 PDHG iterations of the same "
                                              f"instance on one host core (the oracle, the reference's FP64 PDHG "
                                              f"restated), {per_iter * 1e3:.1f} ms/iteration, times the {iters64} "
                                              f"iterations the FP64 device solve of this run needed"}
        print(json.dumps(line), flush=True)
    ctx32.close()
    if pool is not None:
        pool.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
