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
        reduced costs inside the timed region).
fp64    plain FP64 device PDHG (the reference algorithm, ScalaKernels
        semantics): its per-iteration cost is measured on a bounded run and
        its time to 1e-8 is that cost times the iteration count the full FP64
        solve of this instance needs (FP64_ITERATIONS_TO_TOLERANCE, measured
        on a B200 with --full-fp64, which reruns it).

``--impl reference`` times the CPU restatement of the reference FP64 PDHG
(single-threaded, like the reference's ScalaKernels backend) on a bounded
sample of the same instance on the host cores, rank 0 only.
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
# Iterations the plain FP64 device PDHG needs to reach 1e-8 on the seed-0
# instance, from a full run (python bench.py --full-fp64); the CPU baseline
# uses the same count.
FP64_ITERATIONS_TO_TOLERANCE = 1_216_064
ROUND_REDUCTION = 10.0


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "MEASURED_PEAKS.json hbm_gbs"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback 6.65 TB/s"


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


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from noaidi_b200.prima import generators as G
    problem = G.dc_lopf(seed=0, **WORKLOAD)
    for _ in range(min(args.warmup, 1)):
        cpu_sample(problem, 1)
    per_iter, done = cpu_sample(problem, args.cpu_sample_iterations, args.steps)
    iters = FP64_ITERATIONS_TO_TOLERANCE or args.fp64_iterations
    lps = 1.0 / (per_iter * iters)
    line = {"impl": "reference", "metric": METRIC, "value": lps, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / lps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "eps": EPS, "seed": 0},
            "cpu_baseline": {"value": lps, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"{done} FP64 PDHG iterations per step of the same instance "
                                       f"(oracle restatement of Pdhg.Solve + ScalaKernels, 1 thread, like the "
                                       f"reference); {per_iter * 1e3:.1f} ms/iteration extrapolated to the "
                                       f"{iters} iterations the FP64 solve needs to 1e-8"},
            "e2e": {"value": lps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


BATCH_EPS = 1e-6


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


def batch_cpu_baseline(specs, nnz, iterations, sample: int = 8):
    """``PrimaZio.solveAll``'s CPU shape -- one single-threaded FP64 solve per
    host core at a time -- estimated from a bounded sample: up to ``sample``
    instances spread over the sizes are timed per iteration in parallel
    processes (spawned, so none inherits a GPU context); seconds per
    iteration per nonzero from them, times each instance's nonzeros and the
    iterations its device solve took, summed over the instances and shared
    over the cores."""
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    order = sorted(range(len(specs)), key=lambda i: nnz[i])
    picks = sorted({order[round(k * (len(order) - 1) / max(1, sample - 1))] for k in range(min(sample, len(order)))})
    with mp.get_context("spawn").Pool(min(cores, len(picks))) as pool:
        per_iter = pool.map(_oracle_seconds_per_iteration, [specs[i] for i in picks])
    rate = float(np.median([t / nnz[i] for t, i in zip(per_iter, picks)]))
    cpu_seconds = sum(rate * nnz[i] * iterations[i] for i in range(len(specs))) / cores
    return {"value": len(specs) / cpu_seconds, "unit": "LPs/s", "cores": cores, "kind": "port",
            "sample": f"{len(picks)} of the instances timed over 16 FP64 PDHG iterations each on the oracle, one "
                      f"process per instance; {rate * 1e9:.2f} ns per nonzero-iteration extrapolated to every "
                      f"instance's nonzeros and the iterations its device solve took, over {cores} cores"}


def run_batch(args, rank, world, dist, barrier):
    """Config 3: an uneven sweep of ``--batch`` DC-LOPF instances (buses
    U{100..2000}, snapshots U{24..168}, load scale U[0.6, 0.95], seeded), FP32
    refinement to 1e-6, each pass one launch for all of this rank's
    instances.  Ranks take longest-processing-time shards; LPs/s is all
    instances over the slowest rank's time."""
    import torch
    from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, cuda, generators as G
    from noaidi_b200.prima.sharding import instance_size, shard
    problems = G.lopf_batch(seed=0, count=args.batch)
    mine = shard([instance_size(p) for p in problems], world)[rank]
    params = PdhgParams(eps_abs=BATCH_EPS, eps_rel=BATCH_EPS, max_iterations=args.max_iterations)
    mixed = MixedPrecisionParams(reduced_max_iterations=args.max_iterations)
    ctx = cuda.Context(int(os.environ.get("LOCAL_RANK", "0")), 32)
    barrier()
    t = time.perf_counter()
    res = cuda.mixed_solve_batch([problems[i] for i in mine], params, mixed, scheme=cuda.MIXED_REFINEMENT,
                                 round_reduction=args.round_reduction, ctx=ctx) if mine else []
    torch.cuda.synchronize()
    secs = time.perf_counter() - t
    span = max((r.solution.span_ms for r in res), default=0.0) / 1e3
    agg = torch.tensor([span, secs], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(agg, op=dist.ReduceOp.MAX)
    ctx.close()
    its = [r.reduced_iterations + r.refinement_iterations for r in res]
    statuses = sorted({r.solution.status.name for r in res})
    cpu = None
    if rank == 0 and res and not args.skip_cpu:
        specs = _batch_specs(0, args.batch)
        cpu = batch_cpu_baseline([specs[i] for i in mine], [problems[i].constraint_matrix.nnz for i in mine], its)
    return {"workload": f"config 3: {args.batch} uneven DC-LOPF instances, FP32 refinement to {BATCH_EPS:g}",
            "cpu_baseline": cpu,
            "instances": args.batch, "lps_per_s": args.batch / float(agg[0]), "seconds": float(agg[0]),
            "wall_seconds": float(agg[1]), "statuses_rank0": statuses,
            "iterations_rank0": {"min": int(min(its)), "median": float(np.median(its)), "max": int(max(its))}
            if its else None,
            "columns": int(sum(p.num_variables for p in problems)),
            "nnz": int(sum(p.constraint_matrix.nnz for p in problems))}


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
    if args.profile_mixed:
        ctx = cuda.Context(0, 32)
        resident = cuda.DeviceProblem(problem, params, ctx=ctx)
        r = resident.mixed_solve(params, MixedPrecisionParams(reduced_max_iterations=params.max_iterations),
                                 scheme=cuda.MIXED_REFINEMENT, round_reduction=args.round_reduction,
                                 want_solution=False)
        s = r.solution
        out.update(precision="fp32+fp64", reduced_iterations=r.reduced_iterations,
                   refinement_iterations=r.refinement_iterations)
    else:
        resident = cuda.DeviceProblem(problem, params, precision=args.profile_precision)
        s = resident.solve(params, want_solution=False)
        out.update(precision=args.profile_precision)
    out.update(status=s.status.name, objective=s.objective_value, iterations=s.iterations, trials=s.trials,
               device_s=s.device_ms / 1e3, us_per_trial=1e3 * s.device_ms / max(1, s.trials))
    resident.free()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--max-iterations", type=int, default=5_000_000)
    ap.add_argument("--eps", type=float, default=EPS,
                    help="relative KKT tolerance of the timed solves; at any value but 1e-8 the FP64 comparison "
                         "arm is solved in full rather than sampled")
    ap.add_argument("--round-reduction", type=float, default=ROUND_REDUCTION)
    ap.add_argument("--fp64-sample-iterations", type=int, default=20_000)
    ap.add_argument("--fp64-iterations", type=int, default=2_000_000)
    ap.add_argument("--full-fp64", action="store_true", help="solve FP64 to tolerance instead of sampling")
    ap.add_argument("--cpu-sample-iterations", type=int, default=128)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--batch", type=int, default=0,
                    help="also solve this many config-3 instances (uneven LOPF sweep) to 1e-6 as batches "
                         "and report LPs/s under 'batch' (0: off)")
    ap.add_argument("--profile-iterations", type=int, default=0,
                    help="only run this many PDHG iterations of the workload (a bounded case for ncu) and exit")
    ap.add_argument("--profile-precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--profile-snapshots", type=int, default=WORKLOAD["snapshots"])
    ap.add_argument("--profile-workload", default="dc-lopf", choices=["dc-lopf", "sclopf-n1", "expansion-storage"])
    ap.add_argument("--profile-mixed", action="store_true")
    ap.add_argument("--profile-tolerance", type=float, default=EPS)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_iterations:
        return run_profile_case(args)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, cuda, generators as G

    problem = G.dc_lopf(seed=rank, **WORKLOAD)
    eps = args.eps
    if eps != EPS:  # the recorded FP64 iteration count is for 1e-8: measure the FP64 solve in full instead
        args.full_fp64 = True
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

    # end to end through the one-shot C ABI call with host buffers
    barrier()
    e2e = []
    for _ in range(args.steps):
        t = time.perf_counter()
        r_e2e = cuda.mixed_solve(problem, params, mixed, scheme=cuda.MIXED_REFINEMENT,
                                 round_reduction=args.round_reduction, ctx=ctx32)
        e2e.append(time.perf_counter() - t)
    barrier()

    agg = torch.tensor([span_s, sum(e2e)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(agg, op=dist.ReduceOp.MAX)
    max_span, max_e2e = float(agg[0]), float(agg[1])

    # plain FP64 device PDHG on the same resident problem
    ctx64 = cuda.Context(local, 64)
    res64 = cuda.DeviceProblem(problem, params, ctx=ctx64)
    p64 = params if args.full_fp64 else params.copy(max_iterations=args.fp64_sample_iterations)
    fp64 = res64.solve(p64, want_solution=False)
    fp64_ms_per_iter = fp64.device_ms / max(1, fp64.iterations)

    batch_line = run_batch(args, rank, world, dist, barrier) if args.batch else None

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
            "config": {"workload": WORKLOAD_NAME, "n": n, "m": m, "nnz": nnz, "eps": eps, "seed": "rank",
                       "parallelism": f"independent instances x{world}", "scheme": "fp32 pass + fp32 refinement "
                       f"around an fp64 anchor, round reduction {args.round_reduction:g}",
                       "l2": "working set larger than L2 (no flush needed)"},
            "clocks": clocks.summary(),
            "e2e": {"value": steps * world / max_e2e, "unit": UNIT,
                    "h2d_bytes_per_step": int(nnz * 12 + (m + 1) * 4 + 8 * (3 * n + m)),
                    "d2h_bytes_per_step": int(8 * (2 * n + m))},
            "gpu_launches": 2 * steps,
            "solution": {"status": sol.status.name, "objective": sol.objective_value,
                         "primal_residual": sol.kkt.primal_residual_norm,
                         "dual_residual": sol.kkt.dual_residual_norm, "gap": sol.kkt.absolute_gap,
                         "fp32_pass_iterations": last.reduced_iterations,
                         "refinement_iterations": last.refinement_iterations,
                         "rounds": last.refinement_rounds, "e2e_status": r_e2e.solution.status.name},
        }
        iters64 = fp64.iterations if args.full_fp64 and fp64.status.name == "OPTIMAL" else \
            (FP64_ITERATIONS_TO_TOLERANCE or args.fp64_iterations)
        fp64_ttt = fp64_ms_per_iter * iters64
        line["fp64_baseline"] = {
            "ms_per_iteration": fp64_ms_per_iter, "iterations_to_tolerance": iters64,
            "time_to_tolerance_ms": fp64_ttt, "measured": "full solve" if args.full_fp64 else
            f"{fp64.iterations}-iteration sample x iterations of a full FP64 solve", "status": fp64.status.name,
            "speedup_of_fp32_refinement": fp64_ttt / (1e3 * max_span / steps)}
        trials32 = sum(r.solution.trials for r in results)
        iters32 = sum(r.reduced_iterations + r.refinement_iterations for r in results)
        byts = algorithmic_bytes(problem, trials32, iters32, 4, anchored=True)
        achieved = byts / kern_s / 1e9
        line["roofline"] = {"kernel": "pdhg_kernel<float>", "bound": "hbm", "achieved": achieved,
                            "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                            "traffic": TRAFFIC_BYTES_PER_TRIAL * trials32 / len(results) if TRAFFIC_BYTES_PER_TRIAL else None,
                            "peak_source": pk_src,
                            "per_trial_bytes": byts / max(1, trials32), "kernel_ms": 1e3 * kern_s / steps}
        if batch_line:
            line["batch"] = batch_line
        if not args.skip_cpu:
            per_iter, done = cpu_sample(problem, args.cpu_sample_iterations)
            lps = 1.0 / (per_iter * iters64)
            line["cpu_baseline"] = {"value": lps, "unit": UNIT, "cores": 1, "kind": "port",
                                    "sample": f"{done} FP64 PDHG iterations of the same instance on one host core "
                                              f"(oracle restatement of the reference), {per_iter * 1e3:.1f} "
                                              f"ms/iteration extrapolated to {iters64} iterations"}
        print(json.dumps(line), flush=True)
    ctx32.close()
    ctx64.close()
    if dist:
        dist.destroy_process_group()


# DRAM bytes (read + write) per step-size trial of pdhg_kernel<float> on this
# workload, from an ncu capture of a bounded run of the same instance; None
# until measured.
TRAFFIC_BYTES_PER_TRIAL = 140.5e6

if __name__ == "__main__":
    main()
