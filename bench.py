"""Time-to-tolerance benchmark of the B200 PDHG path.

Workload (N=1): the 1M-variable synthetic DC-LOPF dispatch LP (2,000 buses,
3,000 lines, 1,000 generators, 168 hourly snapshots; seeded), solved to a
relative KKT tolerance of 1e-8 by the mixed-precision path (FP32 PDHG on the
device, FP64 finish on the device), next to the plain FP64 device PDHG.
A "step" is one full solve.  With N GPUs every rank solves its own instance
(seed = rank): independent LPs, no collective on the data path (weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``--impl reference`` times the CPU restatement of the reference's FP64 PDHG
(the oracle: single-threaded, like the reference's ScalaKernels) on a bounded
sample of the same workload on the host cores; rank 0 only.

Prints one JSON line (rank 0).  ``value`` is whole-job LPs/s from device
time with the problem already on the device; ``e2e`` is the same metric
through the C-ABI call with host buffers (scaling, upload and download inside
the timed region).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LPs/s to 1e-8 relative KKT, FP32+FP64-refinement PDHG (DC-LOPF 1M)"
UNIT = "LPs/s"
EPS = 1e-8
WORKLOAD = dict(buses=2000, lines=3000, generators=1000, snapshots=168)


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "_fallback": True}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(self.rows[0][1]) if self.rows[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(self.rows)}


def algorithmic_bytes(problem, trials: int, iterations: int, word: int) -> float:
    """Compulsory HBM bytes of the iteration ("Roofline"):
    per accepted trial 13n + 11m vector words plus both matrices
    (nnz index + value words each, row pointers) -- the y and xbar gathers
    count once; a rejected trial skips the K'y product and the running sums
    (7n + 6m words + one matrix)."""
    K = problem.constraint_matrix
    n, m, nnz = problem.num_variables, problem.num_constraints, K.nnz
    acc = (13 * n + 11 * m) * word + 2 * nnz * (4 + word) + 4 * (n + m)
    rej = (8 * n + 6 * m) * word + nnz * (4 + word) + 4 * m
    return acc * iterations + rej * max(0, trials - iterations)


def run_reference(args) -> None:
    """The oracle (reference restatement, FP64, one thread) on a bounded
    sample: a fixed number of PDHG iterations of the same instance, with the
    time to tolerance extrapolated from the FP64 iteration count."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from noaidi_b200.prima import PdhgParams, generators as G
    from oracle import oracle as O
    problem = G.dc_lopf(seed=0, **WORKLOAD)
    sample_iters = args.reference_sample_iterations
    p = PdhgParams(eps_abs=EPS, eps_rel=EPS, max_iterations=sample_iters)
    for _ in range(args.warmup if args.warmup < 1 else 1):
        O.solve(problem, PdhgParams(eps_abs=EPS, eps_rel=EPS, max_iterations=64))
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        s = O.solve(problem, p)
        times.append(time.perf_counter() - t)
    per_iter = float(np.median(times)) / max(1, s.iterations)
    iters_to_tol = args.fp64_iterations_to_tolerance
    lps = 1.0 / (per_iter * iters_to_tol)
    line = {"impl": "reference", "metric": METRIC, "value": lps, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / lps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "dc-lopf-2000bus-168h", "n": problem.num_variables,
                       "m": problem.num_constraints, "nnz": problem.constraint_matrix.nnz, "eps": EPS},
            "cpu_baseline": {"value": lps, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"{sample_iters} FP64 PDHG iterations per step (oracle, 1 thread); "
                                       f"{per_iter * 1e3:.1f} ms/iteration extrapolated to the "
                                       f"{iters_to_tol} iterations the FP64 solve needs to 1e-8"},
            "e2e": {"value": lps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--max-iterations", type=int, default=2_000_000)
    ap.add_argument("--reference-sample-iterations", type=int, default=128)
    ap.add_argument("--fp64-iterations-to-tolerance", type=int, default=0)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        if args.fp64_iterations_to_tolerance <= 0:
            args.fp64_iterations_to_tolerance = FP64_ITERATIONS_TO_TOLERANCE
        return run_reference(args)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from noaidi_b200.prima import MixedPrecisionParams, PdhgParams, cuda, generators as G

    problem = G.dc_lopf(seed=rank, **WORKLOAD)
    params = PdhgParams(eps_abs=EPS, eps_rel=EPS, max_iterations=args.max_iterations)
    mixed = MixedPrecisionParams(reduced_max_iterations=args.max_iterations)
    ctx32 = cuda.Context(local, 32)
    ctx64 = cuda.Context(local, 64)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def one_mixed():
        return cuda.mixed_solve(problem, params, mixed, scheme=cuda.MIXED_TWO_PASS, ctx=ctx32)

    for _ in range(args.warmup):
        r = one_mixed()
    barrier()
    dev_ms, wall = [], []
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        results = []
        for _ in range(args.steps):
            ts = time.perf_counter()
            r = one_mixed()
            wall.append(time.perf_counter() - ts)
            results.append(r)
        barrier()
        elapsed = time.perf_counter() - t0
    # device time of the solver kernels (CUDA events around each launch)
    dev_s = sum(getattr(r.solution, "device_ms", 0.0) for r in results) / 1e3
    red = [r.reduced_device_ms for r in results] if hasattr(results[0], "reduced_device_ms") else None
    total_dev = torch.tensor([dev_s, elapsed], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(total_dev, op=dist.ReduceOp.MAX)
    max_dev, max_wall = float(total_dev[0]), float(total_dev[1])
    sol = results[-1].solution

    # plain FP64 device PDHG, for the ratio and the roofline of the FP64 kernel
    fp64 = None
    if not args.skip_fp64:
        fp64 = cuda.solve(problem, params, precision=64, ctx=ctx64)

    if rank == 0:
        pk = peaks()
        n, m = problem.num_variables, problem.num_constraints
        line = {
            "metric": METRIC, "value": args.steps * world / max_dev if max_dev > 0 else None, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * max_dev / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": "dc-lopf-2000bus-168h", "n": n, "m": m, "nnz": problem.constraint_matrix.nnz,
                       "eps": EPS, "seed": "rank", "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (no flush needed)", "scheme": "two-pass"},
            "clocks": clocks.summary(),
            "e2e": {"value": args.steps * world / max_wall, "unit": UNIT,
                    "h2d_bytes_per_step": int(problem.constraint_matrix.nnz * 12 + (n + 1) * 4 + 4 * 8 * n + 8 * m),
                    "d2h_bytes_per_step": int(8 * (2 * n + m))},
            "gpu_launches": 2 * args.steps,
            "solution": {"status": sol.status.name, "objective": sol.objective_value,
                         "iterations_fp32": results[-1].reduced_iterations,
                         "iterations_fp64": results[-1].refinement_iterations,
                         "primal_residual": sol.kkt.primal_residual_norm, "dual_residual": sol.kkt.dual_residual_norm},
        }
        if fp64 is not None:
            line["fp64_baseline"] = {"ms": fp64.device_ms, "iterations": fp64.iterations, "status": fp64.status.name,
                                     "objective": fp64.objective_value,
                                     "speedup_of_mixed": fp64.device_ms / (1e3 * max_dev / args.steps)}
            byts = algorithmic_bytes(problem, fp64.trials, fp64.iterations, 8)
            achieved = byts / (fp64.device_ms * 1e-3) / 1e9
            line["roofline"] = {"kernel": "pdhg_kernel<double>", "bound": "hbm", "achieved": achieved,
                                "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                                "traffic": None, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
        print(json.dumps(line), flush=True)
    ctx32.close()
    ctx64.close()
    if dist:
        dist.destroy_process_group()


FP64_ITERATIONS_TO_TOLERANCE = 100_000  # replaced by the measured device FP64 count

if __name__ == "__main__":
    main()
