#!/usr/bin/env python
"""Benchmark of the space-time full gradient on B200.

One step = one evaluation of the full 16-stage space-time objective and its gradient
on a 2048 x 1024 Q4 grid: the virtual-heat time-field solve, stage membership
``t <= s/16``, 16 self-weight stage solves (one batched device PCG, rtol 1e-8, FP32
V-cycle inside FP64 PCG), the stage adjoints, the heat adjoint and the sensitivity
field.  Metric: converged stage solves per second (16 per step); the JSON line also
carries the time per full gradient.

``--impl reference`` times the CPU restatement of the reference algorithm (the oracle;
the reference itself is Python and is not installed on the GPU box) on the same
full-size workload with every host core (stages in a process pool, the heat adjoint
beside them), as many whole evaluations as fit its time budget.

Multi-GPU (``--gpus N`` under torchrun): one objective split over the ranks -- rank 0
solves the heat field and broadcasts tPhys, each rank solves its share of the 16 stages
and their adjoints, one all-reduce combines the gradient and the stage compliances
(strong scaling); the time is the max over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NELX, NELY, N_STAGE = 2048, 1024, 16
SEED = 3
METRIC = "stage solves/s (space-time objective + full gradient, 2048x1024 Q4, 16 stages, rtol 1e-8)"
UNIT = "stage solves/s"
# Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the roofline
# kernels from ncu captures: the FP32 level-0 apply over 16 stage rows, and the FP64 p.Ap
# pass per stage row (a 4-row capture of bench.py --pcg-only, divided by its 4 rows).
NCU_TRAFFIC = {"l0_apply_fp32_16rows": 687000576, "pcg_pap_fp64_per_row": 198669505}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--roofline-only", action="store_true",
                    help="run only the roofline kernel's timing (the small case for an ncu capture)")
    ap.add_argument("--vcycle-only", action="store_true",
                    help="run only V-cycles of the stage solve's 16-row mixed hierarchy (the small case for "
                         "ncu captures of the cycle's kernels; seeded uniform densities in [1e-3, 1])")
    ap.add_argument("--pcg-only", action="store_true",
                    help="run only a 4-row plane-stress PCG on the 2048x1024 grid (the small case for ncu "
                         "captures of the outer PCG's p.Ap pass, with the 32-row bands of the 16-row solve; "
                         "seeded densities and loads)")
    ap.add_argument("--no-uneven", action="store_true",
                    help="skip the batched uneven multi-problem measurement")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the library's launch-shape heuristics instead of the autotuner's measured choices")
    ap.add_argument("--no-mma", action="store_true", help="skip the MMA step measurement")
    ap.add_argument("--mma-only", action="store_true", help="only the MMA step measurement")
    ap.add_argument("--mma-vars", type=int, default=2 * NELX * NELY,
                    help="design variables of the MMA step (default 2 x 2048 x 1024; smaller for profiling)")
    ap.add_argument("--no-dropin", action="store_true",
                    help="skip the end-to-end timing through the reference-signature chain")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="seconds of full-size CPU evaluations the reference arm may spend (at least one)")
    ap.add_argument("--cpu-budget", type=float, default=0.0,
                    help="seconds of full-size CPU evaluations the cpu_baseline leg may spend (at least one)")
    ap.add_argument("--uneven-only", action="store_true",
                    help="run only the batched uneven multi-problem measurement")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---- CPU baseline: the oracle on the full workload -----------------------------------

def cpu_full_evaluations(max_evals: int, budget_s: float) -> dict:
    """Times the oracle's full space-time objective + gradient at 2048x1024 with 16 stages
    (the benchmark's seed), at most ``max_evals`` times and no more once ``budget_s`` is
    spent (at least once).  Every host core works: the 16 stages run in a spawn-started
    pool of single-threaded processes while the main process runs the heat adjoint, and
    the oracle's C/OpenMP loops use all threads in the main process.  A 64x32 evaluation
    first starts the pool's workers (untimed)."""
    import numpy as np

    from oracle import sttopt_oracle as O

    workers = os.cpu_count() or 1
    pool = O.stage_pool(workers)
    try:
        xs = O.smoothed_density(64, 32, SEED)
        O.spacetime_objective(xs, np.random.default_rng(SEED).uniform(-1, 1, xs.shape), n_stage=N_STAGE, pool=pool)
        x = O.smoothed_density(NELX, NELY, SEED)
        w = np.random.default_rng(SEED).uniform(-1, 1, (NELY, NELX))
        times, t_start = [], time.perf_counter()
        while len(times) < max(1, max_evals):
            t0 = time.perf_counter()
            out = O.spacetime_objective(x, w, n_stage=N_STAGE, pool=pool)
            times.append(time.perf_counter() - t0)
            if time.perf_counter() - t_start + times[-1] > budget_s:
                break
    finally:
        pool.close()
        pool.join()
    med = statistics.median(times)
    return dict(value=N_STAGE / med, full_gradient_ms=med * 1e3, evaluations=len(times), seconds=times,
                cores=workers, c_kernels=O.c_kernels() is not None, iterations=dict(
                    stage=out["forward_n_iter"], heat=out["heat_n_iter"], adjoint=out["adjoint_n_iter"],
                    heat_adjoint=out["heat_adjoint_n_iter"]),
                sample=(f"the full workload: {len(times)} evaluation(s) of the 2048x1024 x 16-stage objective + "
                        f"gradient ({', '.join(f'{t:.1f}' for t in times)} s), stages in a spawn pool of {workers} "
                        f"single-thread processes beside the heat adjoint, oracle C/OpenMP loops "
                        f"{'on' if O.c_kernels() is not None else 'absent (NumPy)'}; no scaling"))


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ.setdefault(k, str(threads))
    os.environ.setdefault("OMP_WAIT_POLICY", "passive")
    s = cpu_full_evaluations(args.steps, args.ref_budget)
    v = s["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": s["evaluations"], "warmup": 0, "ms_per_step": s["full_gradient_ms"],
        "requested": {"steps": args.steps, "warmup": args.warmup,
                      "note": "each step is a whole full-size CPU evaluation; as many as fit --ref-budget seconds "
                              "are timed (at least one), no warm-up evaluation at full size"},
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded N(0,1) noise, radius-4 cone filter, mapped to [1e-3, 1]; seeded U(-1,1) time weights)",
        "config": {"workload": "space-time objective + full gradient: heat time field, 16 hard-threshold gravity "
                               "stages, MG-PCG rtol 1e-8, stage + heat adjoints (CPU oracle, FP64)",
                   "nelx": NELX, "nely": NELY, "n_stage": N_STAGE},
        "iterations": s["iterations"],
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": s["cores"], "kind": "port", "sample": s["sample"],
                         "seconds_per_evaluation": s["seconds"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- batched uneven problems ---------------------------------------------------------

UNEVEN_SIZES = [(256, 128), (512, 256), (768, 384), (1024, 512), (1536, 768)]
UNEVEN_PROBLEMS = 64


def uneven_workload(dev, seed=SEED):
    """64 independent space-time problems: seeded grid sizes from UNEVEN_SIZES, 4-16
    stages each, seeded smoothed densities and time weights."""
    import numpy as np

    from sttopt_b200 import synthetic

    rng = np.random.default_rng(seed)
    picks = rng.integers(0, len(UNEVEN_SIZES), UNEVEN_PROBLEMS)
    stages = rng.integers(4, 17, UNEVEN_PROBLEMS)
    xs, ws = [], []
    for k, i in enumerate(picks):
        nx, ny = UNEVEN_SIZES[i]
        xs.append(synthetic.smoothed_density(nx, ny, 1000 * seed + k, device=dev))
        ws.append(synthetic.time_weights(nx, ny, 1000 * seed + k, device=dev))
    return xs, ws, [int(n) for n in stages]


def run_vcycles(dev, steps, warmup):
    """V-cycles z = M r on the 2048x1024 x 16-row mixed hierarchy of the stage solve (the
    bench's mesh and build-plate clamp; seeded densities): ms per cycle."""
    import numpy as np
    import torch

    from sttopt_b200 import fem, torch_mg

    rng = np.random.default_rng(SEED)
    rho = torch.as_tensor(rng.uniform(1e-3, 1.0, (N_STAGE, NELX * NELY)), device=dev)
    edof = torch.as_tensor(fem.element_dof_map(NELX, NELY, 2), device=dev)
    KE = torch.as_tensor(fem.plane_stress_KE(0.3), device=dev)
    ndof = 2 * (NELX + 1) * (NELY + 1)
    mask = torch.ones(ndof, dtype=torch.bool, device=dev)
    mask[-2 * (NELX + 1):] = False
    levels = torch_mg.build_hierarchy(rho, edof, KE, mask, NELX, NELY, precision="mixed")
    M = torch_mg.VCycle(levels)
    r = torch.as_tensor(rng.standard_normal((N_STAGE, ndof)), device=dev) * mask
    for _ in range(warmup):
        M(r)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        z = M(r)
    b.record()
    torch.cuda.synchronize()
    return {"ms_per_cycle": a.elapsed_time(b) / steps, "levels": len(levels), "rows": N_STAGE,
            "z_norm": float(z.norm())}


def run_pcg_small(dev, rows=4):
    """One mixed-precision PCG solve of `rows` plane-stress rows on the 2048x1024 grid (the
    bench's mesh and clamp; seeded densities and loads): iterations and time."""
    import numpy as np
    import torch

    from sttopt_b200 import fem, torch_fem, torch_mg

    rng = np.random.default_rng(SEED)
    rho = torch.as_tensor(rng.uniform(1e-3, 1.0, (rows, NELX * NELY)), device=dev)
    edof = torch.as_tensor(fem.element_dof_map(NELX, NELY, 2), device=dev)
    KE = torch.as_tensor(fem.plane_stress_KE(0.3), device=dev)
    ndof = 2 * (NELX + 1) * (NELY + 1)
    mask = torch.ones(ndof, dtype=torch.bool, device=dev)
    mask[-2 * (NELX + 1):] = False
    levels = torch_mg.build_hierarchy(rho, edof, KE, mask, NELX, NELY, precision="mixed")
    F = torch.as_tensor(rng.standard_normal((rows, ndof)), device=dev) * mask
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    _, n = torch_fem.pcg(levels[0], F, torch_mg.VCycle(levels), rtol=1e-8, max_iter=200)
    b.record()
    torch.cuda.synchronize()
    return {"rows": rows, "n_iter": n, "ms": a.elapsed_time(b)}


def run_uneven(dev, steps=2, warmup=1, memory_budget=None):
    """Stage solves per second over the 64 uneven problems (objective + full gradient of
    each), grouped per grid size into batched solves on concurrent streams; with
    ``memory_budget`` (bytes) the groups run in waves that fit it."""
    import torch

    from sttopt_b200 import spacetime

    xs, ws, ns = uneven_workload(dev)
    cache: dict = {}
    info: dict = {}
    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats(dev)
    kw = dict(problems=cache, info=info, memory_budget=memory_budget)
    from sttopt_b200 import autotune

    if autotune.mode() != "off":
        # the grid sizes' launch shapes tuned with the groups one after another (clean timings)
        prev = autotune.mode()
        autotune.enable()
        spacetime.objective_and_gradient_many(xs, ws, ns, problems=cache, concurrent=False)
        if prev == "frozen":
            autotune.freeze()
    for _ in range(warmup):
        spacetime.objective_and_gradient_many(xs, ws, ns, **kw)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        spacetime.objective_and_gradient_many(xs, ws, ns, **kw)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    # comparator (unbudgeted run only): the same problems one after another through the
    # single-problem entry point, each with its own hierarchies and solves
    single = None
    if memory_budget is None:
        for x, w, n in zip(xs[:4], ws[:4], ns[:4]):
            spacetime.objective_and_gradient(x, w, n_stage=n)
        torch.cuda.synchronize()
        a.record()
        for x, w, n in zip(xs, ws, ns):
            spacetime.objective_and_gradient(x, w, n_stage=n)
        b.record()
        torch.cuda.synchronize()
        ms1 = a.elapsed_time(b)
        single = {"value": sum(ns) / (ms1 / 1e3), "unit": UNIT, "ms_per_step": ms1,
                  "speedup_of_batching": ms1 / ms,
                  "path": "spacetime.objective_and_gradient per problem, one after another (1 pass)"}
    counts: dict = {}
    for x, n in zip(xs, ns):
        key = f"{x.shape[1]}x{x.shape[0]}"
        c = counts.setdefault(key, {"problems": 0, "stages": 0})
        c["problems"] += 1
        c["stages"] += n
    del cache
    torch.cuda.empty_cache()
    return {"metric": "stage solves/s (64 uneven space-time problems, objective + full gradient, rtol 1e-8)",
            "value": sum(ns) / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": warmup,
            "problems": len(xs), "stage_rows": sum(ns), "groups": counts,
            "peak_device_gib": round(torch.cuda.max_memory_allocated() / 2**30, 1),
            "iterations": {f"{k[0]}x{k[1]}": v for k, v in info.items()},
            "memory_budget_gib": None if memory_budget is None else round(memory_budget / 2**30, 1),
            "one_problem_at_a_time": single,
            "batching": "one batched device PCG per grid size (heat, stages, adjoints), the size groups "
                        "on concurrent CUDA streams" + ("" if memory_budget is None else
                                                        ", in waves whose estimated memory fits the budget")}


# ---- the MMA step the optimisation loop takes after each evaluation ----------------------

MMA_M = 17  # constraint rows of the space-time problem (volume, start points, stage bounds, ...)


def mma_workload(n, m, seed=SEED):
    """A seeded unit-box MMA step of the space-time problem's shape: n design variables
    (density and time field), m constraint rows, per-variable trust regions, the
    adaptive-asymptote branch (iteration 2)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    xval = rng.uniform(0.05, 0.95, n)
    xold1 = np.clip(xval + rng.normal(0, 0.02, n), 0, 1)
    xold2 = np.clip(xold1 + rng.normal(0, 0.02, n), 0, 1)
    return dict(xval=xval, xold1=xold1, xold2=xold2, df0dx=rng.normal(0, 1e-6, n), fval=rng.normal(0, 0.1, m),
                dfdx=rng.normal(0, 1e-6, (m, n)), move=rng.uniform(0.02, 0.1, n), low=xval - 0.2, upp=xval + 0.2)


def run_mma(dev, steps=3, warmup=1, cpu_sample=1 << 18, n=2 * NELX * NELY):
    """``mma.mmasub`` on 2 x 2048 x 1024 variables and 17 constraints (the step after each
    evaluation), timed with CUDA events; the HBM roofline of its passes (algorithmic bytes:
    one m x n read and the n-vectors of each pass); the oracle's mmasub on a sample of
    ``cpu_sample`` variables on the host."""
    import numpy as np
    import torch

    from sttopt_b200 import mma

    m = MMA_M
    p = mma_workload(n, m)
    t = {k: torch.as_tensor(v).to(dev) for k, v in p.items()}
    zeros = torch.zeros(m, dtype=torch.float64, device=dev)
    cc = torch.full((m,), 1000.0, dtype=torch.float64, device=dev)
    one, zero = torch.ones(n, dtype=torch.float64, device=dev), torch.zeros(n, dtype=torch.float64, device=dev)
    tr = mma.trust_region_params(t["move"], one)

    def call(stats=None):
        return mma.mmasub(m, n, 2, t["xval"], zero, one, t["xold1"], t["xold2"], 0.0, t["df0dx"], t["fval"],
                          t["dfdx"], t["low"], t["upp"], 1.0, zeros, cc, zeros, raa0=1e-5 / n, stats=stats, **tr)

    for _ in range(warmup):
        call()
    stats: dict = {}
    call(stats)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        call()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    newton, tries = stats["subsolv_newton_steps"], stats["subsolv_line_search_tries"]
    # bytes a variable: assemble 8m + 112 (with the pending step), step 8m + 88, search 8m + 88
    per_var = newton * (8 * m + 112 + 8 * m + 88) + tries * (8 * m + 88) + (8 * m + 112)
    achieved = per_var * n / (ms / 1e3) / 1e9
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    # CPU: the oracle's mmasub (NumPy, FP64) on a sample of the same workload
    from oracle import mma_oracle

    q = mma_workload(cpu_sample, m)
    trq = {"asyinit": q["move"], "asyclamp_min": 0.02 * q["move"], "asyclamp_max": 20.0 * q["move"],
           "move": q["move"]}
    from threadpoolctl import threadpool_limits

    t0 = time.perf_counter()
    with threadpool_limits(limits=1):
        mma_oracle.mmasub(m, cpu_sample, 2, q["xval"], np.zeros(cpu_sample), np.ones(cpu_sample), q["xold1"],
                          q["xold2"], 0.0, q["df0dx"], q["fval"], q["dfdx"], q["low"], q["upp"], 1.0, np.zeros(m),
                          np.full(m, 1000.0), np.zeros(m), raa0=1e-5 / cpu_sample, **trq)
    cpu_s = time.perf_counter() - t0
    return {"metric": f"mmasub calls/s (unit-box MMA step: {n} variables, 17 constraints, FP64)",
            "value": 1e3 / ms, "unit": "calls/s", "ms_per_call": ms, "steps": steps, "warmup": warmup,
            "newton_steps": newton, "line_search_tries": tries,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": "of measured" if "hbm_gbs" in peaks else "of fallback",
                         "bytes_per_variable": per_var,
                         "basis": "algorithmic bytes of all passes of the call (dfdx once a pass, the n-vectors a "
                                  "pass reads and writes) over the call's device time"},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "calls/s", "cores": 1, "kind": "port",
                             "sample": f"the oracle's mmasub (NumPy) on {cpu_sample} variables of the same workload "
                                       f"({cpu_s:.2f} s; the full call has {n // cpu_sample}x the variables)"}}


# ---- clocks -----------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- the GPU arm --------------------------------------------------------------------

def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from __graft_entry__ import load_package

    load_package()
    from sttopt_b200 import _lib, sharding, spacetime, synthetic

    # the one workload of every rank (with N ranks its 16 stages are split over them)
    x = synthetic.smoothed_density(NELX, NELY, SEED, device=dev)
    w = synthetic.time_weights(NELX, NELY, SEED, device=dev)
    problem = spacetime.SpaceTimeProblem(NELX, NELY, dev)
    if args.roofline_only:
        u = torch.randn(N_STAGE, 2 * problem.nnode, device=dev, dtype=torch.float64)
        roof, detail = roofline(_lib, problem, {"U": u}, dev)
        print(json.dumps({"roofline": roof, "roofline_detail": detail}), flush=True)
        return 0
    if args.pcg_only:
        print(json.dumps({"pcg": run_pcg_small(dev)}), flush=True)
        return 0
    if args.vcycle_only:
        print(json.dumps({"vcycle": run_vcycles(dev, max(args.steps, 1), max(args.warmup, 0))}), flush=True)
        return 0
    if args.uneven_only:
        print(json.dumps({"batched_uneven": run_uneven(dev, steps=max(args.steps, 1), warmup=max(args.warmup, 1))}),
              flush=True)
        return 0
    if args.mma_only:
        print(json.dumps({"mma_unit_box_step": run_mma(dev, steps=max(args.steps, 1), warmup=max(args.warmup, 1),
                                                       n=args.mma_vars)}), flush=True)
        return 0
    info: dict = {}
    from sttopt_b200 import autotune

    if not args.no_autotune:
        # launch shapes picked by measurement on one clean evaluation (the heat adjoint in
        # order, not beside the stage solves), then only reused
        autotune.enable()
        spacetime.objective_and_gradient(x, w, n_stage=N_STAGE, precision=args.precision, problem=problem,
                                         overlap=False)
        autotune.freeze()

    def step(xx, ww, precision=args.precision, batched=True):
        return spacetime.objective_and_gradient(xx, ww, n_stage=N_STAGE, precision=precision,
                                                problem=problem, info=info, batched=batched)

    def timed_step(xx, ww):
        """The measured step: the whole objective, or this rank's share of it split over
        the ranks (heat field broadcast from rank 0, one all-reduce)."""
        if world == 1:
            return step(xx, ww)
        return sharding.objective_and_gradient_split(xx, ww, n_stage=N_STAGE, precision=args.precision,
                                                     problem=problem, info=info)

    for _ in range(max(args.warmup, 0)):
        out = timed_step(x, w)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def device_allocs():
        st = torch.cuda.memory_stats(dev)
        return int(st.get("num_device_alloc", 0))

    # timed region: inputs resident in HBM
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    L = _lib.lib()
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        allocs0 = device_allocs()
        L.stt_pap_timing(1)  # events around the plane-stress p.Ap passes (the dominant kernel)
        start.record()
        for k in range(args.steps):
            marks[k].record()
            torch.cuda.nvtx.range_push("timed_step")  # lets a profiler select one step's launches
            out = timed_step(x, w)
            torch.cuda.nvtx.range_pop()
        marks[-1].record()
        end.record()
        torch.cuda.synchronize()
        barrier()
    elapsed_ms = start.elapsed_time(end)
    pap = (ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong())
    L.stt_pap_timing_read(ctypes.byref(pap[0]), ctypes.byref(pap[1]), ctypes.byref(pap[2]))
    L.stt_pap_timing(0)
    pap_live = {"ms": pap[0].value, "launches": pap[1].value, "rows": pap[2].value}
    timed_detail = {"step_ms": [round(marks[k].elapsed_time(marks[k + 1]), 3) for k in range(args.steps)],
                    "device_allocs": device_allocs() - allocs0}
    if world > 1:
        t = torch.tensor([elapsed_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    ms_per_step = elapsed_ms / args.steps
    value = N_STAGE * args.steps / (elapsed_ms / 1e3)  # one objective's 16 stages a step, on all ranks together
    iters = dict(info)

    # end to end through the public call with host buffers
    xh = x.detach().cpu().pin_memory()
    wh = w.detach().cpu().pin_memory()
    gh = torch.empty(NELY, NELX, dtype=torch.float64).pin_memory()
    oh = torch.empty(1, dtype=torch.float64).pin_memory()
    xd, wd = torch.empty_like(x), torch.empty_like(w)
    # untimed passes through the host-buffer path (allocator and copy engines warm; the
    # second one settles the allocator with a previous step's outputs alive, as in the loop)
    for _ in range(2):
        xd.copy_(xh, non_blocking=True)
        wd.copy_(wh, non_blocking=True)
        o = timed_step(xd, wd)
        gh.copy_(o["gradient"], non_blocking=True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    emarks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    allocs0 = device_allocs()
    e0.record()
    for k in range(args.steps):
        emarks[k].record()
        xd.copy_(xh, non_blocking=True)
        wd.copy_(wh, non_blocking=True)
        o = timed_step(xd, wd)
        gh.copy_(o["gradient"], non_blocking=True)
        oh.copy_(o["objective"].reshape(1), non_blocking=True)
    emarks[-1].record()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    e2e_detail = {"step_ms": [round(emarks[k].elapsed_time(emarks[k + 1]), 3) for k in range(args.steps)],
                  "device_allocs": device_allocs() - allocs0}
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = N_STAGE * args.steps / (e2e_ms / 1e3)
    h2d = xh.numel() * 8 + wh.numel() * 8
    d2h = gh.numel() * 8 + 8

    extra = {}
    if rank == 0:
        extra["roofline"], extra["roofline_detail"] = roofline(_lib, problem, out, dev, pap_live)
        # the plain FP64 GPU form: unbatched stages, FP64 V-cycle
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        step(x, w, precision="fp64", batched=False)
        p0.record()
        ref = step(x, w, precision="fp64", batched=False)
        p1.record()
        torch.cuda.synchronize()
        plain_ms = p0.elapsed_time(p1)
        c_err = float(((out["c_s"] - ref["c_s"]).abs() / ref["c_s"].abs()).max())
        g_err = float((out["gradient"] - ref["gradient"]).norm() / ref["gradient"].norm())
        extra["plain_fp64_form"] = {"full_gradient_ms": plain_ms, "speedup_batched_mixed": plain_ms / ms_per_step,
                                    "max_rel_err_stage_compliance": c_err, "rel_err_gradient_l2": g_err}
        if not args.no_profile:
            extra["gpu_launches_per_step"], extra["top_kernels"] = profile_step(step, x, w)
        if not args.no_dropin:
            extra["e2e_dropin"] = {p: run_dropin(dev, x, w, args.steps, max(args.warmup, 1), p, out)
                                   for p in ("fp64", "mixed")}
        if not args.no_uneven:
            del ref
            torch.cuda.empty_cache()
            extra["batched_uneven"] = run_uneven(dev)
            extra["batched_uneven_budget"] = run_uneven(dev, memory_budget=40 << 30)
        if not args.no_mma:
            extra["mma_unit_box_step"] = run_mma(dev)
        if world == 1 and not args.no_cpu_baseline:
            s = cpu_full_evaluations(1, args.cpu_budget)
            extra["cpu_baseline"] = {"value": s["value"], "unit": UNIT, "cores": s["cores"], "kind": "port",
                                     "sample": s["sample"], "full_gradient_ms": s["full_gradient_ms"],
                                     "iterations": s["iterations"]}
    if rank == 0:
        launches = extra.pop("gpu_launches_per_step", None)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f64 outer PCG + f32 V-cycle" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded N(0,1) noise, radius-4 cone filter, mapped to [1e-3, 1]; seeded U(-1,1) time weights)",
            "config": {"workload": "space-time objective + full gradient: heat time field, 16 hard-threshold "
                                   "gravity stages, batched MG-PCG rtol 1e-8, stage + heat adjoints",
                       "nelx": NELX, "nely": NELY, "n_stage": N_STAGE, "precision": args.precision,
                       "parallelism": (f"{world} ranks split the one objective: rank 0 solves the heat field and "
                                       "broadcasts tPhys, the 16 stages are spread over the ranks, one all-reduce "
                                       "of gradient and stage compliances") if world > 1 else "single GPU",
                       "l2": "working set (16 stage rows x 4.2M dofs, hierarchy) far above the 126 MB L2; no flush"},
            "full_gradient_ms": ms_per_step,
            "iterations": iters,
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "full_gradient_ms": e2e_ms / args.steps, "detail": e2e_detail},
            "timed_detail": timed_detail,
            "autotune": {"mode": autotune.mode(),
                         "choices": {k: {kk: v[kk] for kk in ("pcg_band", "level_waves")}
                                     for k, v in autotune.cache().items()}},
            "gpu_launches": None if launches is None else launches * args.steps,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_dropin(dev, x, w, steps, warmup, precision, fused):
    """End to end through the reference-signature chain (``spacetime.DropInChain``:
    heat_time_field -> batched_whole_and_gravity_compliance(mask_fn=hard_time_mask) ->
    jacobian_rows) with host buffers: each step copies x and w in from pinned host memory
    and the gradient and objective out.  Also the chain's agreement with the fused step."""
    import torch

    from sttopt_b200 import spacetime

    chain = spacetime.DropInChain(NELX, NELY, dev, n_stage=N_STAGE)
    xh, wh = x.detach().cpu().pin_memory(), w.detach().cpu().pin_memory()
    gh = torch.empty(NELY, NELX, dtype=torch.float64).pin_memory()
    oh = torch.empty(1, dtype=torch.float64).pin_memory()
    xd, wd = torch.empty_like(x), torch.empty_like(w)

    def one():
        xd.copy_(xh, non_blocking=True)
        wd.copy_(wh, non_blocking=True)
        o = chain(xd, wd, precision=precision)
        gh.copy_(o["gradient"], non_blocking=True)
        oh.copy_(o["objective"].reshape(1), non_blocking=True)
        return o

    for _ in range(warmup):
        o = one()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        o = one()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    c_err = float(((o["c_s"] - fused["c_s"]).abs() / fused["c_s"].abs()).max())
    g_err = float((o["gradient"] - fused["gradient"]).norm() / fused["gradient"].norm())
    del chain
    torch.cuda.empty_cache()
    return {"value": N_STAGE / (ms / 1e3), "unit": UNIT, "full_gradient_ms": ms, "steps": steps,
            "h2d_bytes_per_step": 2 * x.numel() * 8, "d2h_bytes_per_step": x.numel() * 8 + 8,
            "vs_fused_step": {"max_rel_err_stage_compliance": c_err, "rel_err_gradient_l2": g_err},
            "path": "heat_time_field -> batched_whole_and_gravity_compliance(mask_fn=hard_time_mask) -> "
                    "jacobian_rows" + (" (stage solve through the _solve_fe_batched patch point, FP32 V-cycle)"
                                       if precision == "mixed" else " (FP64, the reference's arithmetic)")}


def roofline(_lib, P, out, dev, pap_live=None):
    """The dominant kernel of the step, the outer PCG's FP64 p.Ap pass, timed live inside
    the timed region (CUDA events around its launches, stt_pap_timing); and, beside it,
    the level-0 operator apply over the 16 stage rows timed alone in FP32 and FP64."""
    import torch

    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "of measured" if "hbm_gbs" in peaks else "of fallback"
    L = _lib.lib()
    st = _lib.stream()
    ndof, nel = 2 * P.nnode, P.nel
    rows = N_STAGE
    detail = {}
    for name, dt, prec, es in [("l0_apply_fp32_16rows", torch.float32, _lib.STT_FP32, 4),
                               ("l0_apply_fp64_16rows", torch.float64, _lib.STT_FP64, 8)]:
        # the V-cycle's layout: rows padded to 16 bytes
        vs = (ndof + 3) // 4 * 4
        u = torch.zeros(rows, vs, device=dev, dtype=dt)
        u[:, :ndof] = (out["U"] if "U" in out else torch.randn(rows, ndof, device=dev, dtype=torch.float64)).to(dt)
        rho = torch.rand(rows, nel, device=dev, dtype=torch.float64).to(dt)
        o = torch.empty_like(u)
        for _ in range(3):
            _lib.check(L.stt_q4_apply(prec, 2, NELX, NELY, rows, _lib.ptr(u), vs, _lib.ptr(o), vs,
                                      _lib.ptr(rho), nel, None, 0, _lib.ptr(P.fixed2), 3, P.ke, st))
        n = 20
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            _lib.check(L.stt_q4_apply(prec, 2, NELX, NELY, rows, _lib.ptr(u), vs, _lib.ptr(o), vs,
                                      _lib.ptr(rho), nel, None, 0, _lib.ptr(P.fixed2), 3, P.ke, st))
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / n
        alg = rows * (2 * ndof * es + nel * es)  # read u, write Ku, read rho (flags: 1 B/node not counted)
        gbs = alg / (ms * 1e-3) / 1e9
        detail[name] = {"achieved": gbs, "ms_per_launch": ms, "algorithmic_bytes": alg, "frac": gbs / peak}
    for k in ("l0_apply_fp32_16rows",):
        detail[k]["traffic"] = NCU_TRAFFIC[k]
    if pap_live and pap_live["launches"]:
        # per row and launch: read p_old 8 ndof, z 4 ndof, x 8 ndof and rho 8 nel; write p, Ap and
        # x 8 ndof each (flags, 1 B a node, not counted)
        per_row = 44 * ndof + 8 * nel
        alg = per_row * pap_live["rows"] / pap_live["launches"]
        ms = pap_live["ms"] / pap_live["launches"]
        gbs = alg / (ms * 1e-3) / 1e9
        rows_per = pap_live["rows"] / pap_live["launches"]
        traffic = NCU_TRAFFIC.get("pcg_pap_fp64_per_row")
        roof = {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                "peak_source": peak_src,
                "kernel": "pcg_pap_kernel (FP64 outer PCG: p = beta p + z, A p, p.Ap, deferred x update), "
                          f"{rows_per:.0f} stage rows, timed live over {pap_live['launches']} launches",
                "algorithmic_bytes": alg, "ms_per_launch": ms,
                "traffic": None if traffic is None else traffic * rows_per}
    else:
        main_k = detail["l0_apply_fp32_16rows"]
        roof = {"bound": "hbm", "achieved": main_k["achieved"], "peak": peak, "unit": "GB/s",
                "frac": main_k["frac"], "peak_source": peak_src, "kernel": "l0 Q4 apply, FP32, 16 stage rows",
                "traffic": NCU_TRAFFIC["l0_apply_fp32_16rows"]}
    return roof, detail


def profile_step(step, x, w):
    """Kernel launches of one step (CUPTI through torch.profiler) and the top kernels."""
    import torch

    try:
        from torch.profiler import ProfilerActivity, profile

        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            step(x, w)
            torch.cuda.synchronize()
        totals: dict = {}
        count = 0
        for ev in prof.events():
            if ev.device_type.name != "CUDA":
                continue
            name = ev.name
            if "stt::" not in name:
                continue
            count += 1
            key = name.split("(")[0].replace("void ", "")
            t = totals.setdefault(key, [0, 0.0])
            t[0] += 1
            t[1] += ev.device_time_total if hasattr(ev, "device_time_total") else ev.cuda_time_total
        total = sum(v[1] for v in totals.values()) or 1.0
        top = sorted(totals.items(), key=lambda kv: -kv[1][1])[:30]
        return count, [{"kernel": k, "launches": v[0], "us": round(v[1], 1), "share": round(v[1] / total, 3)}
                       for k, v in top] + [{"kernel": "(sum of this library's kernels)", "us": round(total, 1)}]
    except Exception as exc:  # profiler unavailable: report, do not fail the bench
        return None, [{"error": str(exc)[:200]}]


if __name__ == "__main__":
    sys.exit(main())
