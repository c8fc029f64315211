#!/usr/bin/env python3
"""Benchmark of the B200 phase-retrieval backend on its headline workload.

Workload: 256 x 256 complex64, 32 starts, recipe
``repeat(10, RAAR(50, 0.9), Shrinkwrap(0.3, 1.0)), ER(200)`` (700 iterations),
on the seeded ``gaussians`` problem (5 Gaussians in a disk, ramp + filtered
noise phase, Poisson 1e6, beamstop r = 8, autocorrelation support). One step
is one run of the whole recipe over all 32 starts; the metric is
start-iterations per second (starts x iterations / time).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own 32 starts on its own GPU (independent
replicas, weak scaling); rank 0 prints one JSON line. ``--impl reference``
times the reference's CPU implementation of the same recipe on the host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "iterations/s per 256² start, batched vs plain, at <=1e-5 rel err; HBM GB/s"
UNIT = "start-iterations/s"
SHAPE = (256, 256)
STARTS = 32
SEED = 1000
WORKLOAD = "gaussians 256x256 complex64, 32 starts, repeat(10, RAAR(50,0.9), Shrinkwrap(0.3,1.0)), ER(200)"
# Algorithmic bytes per element of each fused line pass (what the pass must
# move at least): the modulus pass reads the wave and the FP32 amplitude and
# writes the wave; the update pass reads the wave, support and old iterate and
# writes the iterate and the next wave.
PASS_BYTES = {"modulus (y-axis fwd+P_M+inv)": 8 + 4 + 8, "update (x-axis inv+update+fwd)": 8 + 1 + 8 + 8 + 8}
# What the same work moves as separate kernels (one FFT pass = 16 B per
# element; modulus 20 B, update 25 B): the rate an unfused chain would need.
UNFUSED_BYTES = {"modulus (y-axis fwd+P_M+inv)": 16 + 20 + 16,
                 "update (x-axis inv+update+fwd)": 16 + 25 + 16}
L2_FLUSH_BYTES = 256 << 20


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        peaks = json.loads(path.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_value(key):
    """The value of a `key: value` line in the committed ncu summaries, or None."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for line in f.read_text().splitlines():
            if line.startswith(key + ":"):
                return line.split(":", 1)[1].split()[0]
    return None


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` ("modulus" or "update") from the
    committed ncu summary."""
    value = profile_value(f"dram_bytes_per_launch_{kernel}")
    try:
        return float(value) if value is not None else None
    except ValueError:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(f"/tmp/qpb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.path.open("w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, value in zip(names, parts[5:9]):
                if value.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        busy = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference arm
# A CPU step is the whole benchmark recipe (RAAR + Shrinkwrap + ER, 700
# iterations) on a sample of the 32 starts: starts 0..CPU_SAMPLE_STARTS-1,
# drawn exactly as the GPU arm draws its starts 0..3. The reference's CpuSolver
# runs the starts of a step one after another, each on every host thread, so
# the sample's rate per start-iteration is the whole job's.
CPU_SAMPLE_STARTS = 4
PORT_SAMPLE_STARTS = 2


def config_of(args, world):
    """The workload description both arms print (the arm-specific schedule and
    sampling are reported beside it)."""
    return {
        "workload": WORKLOAD,
        "shape": list(SHAPE),
        "starts_per_gpu": STARTS,
        "iterations": 700,
        "parallelism": f"replicas x{world}",
        "l2": f"GPU arm: {L2_FLUSH_BYTES >> 20} MiB write between steps, outside the step events; "
              "CPU arm: n/a",
    }


def reference_step(intensity, mask, starts, threads, port=False):
    """One CPU step: the whole recipe on `starts` starts with the reference's
    own CpuSolver (compiled from its sources) when available and `port` is
    false, else the oracle's numpy port of CpuSolver::iterate on scipy.fft
    (pocketfft C++). Solver construction is not timed. Returns (seconds, kind,
    label)."""
    from qoraphasecu_b200 import workloads

    recipe = workloads.gaussians_recipe().ops()
    from oracle import ref as oracle_ref

    if not port and oracle_ref.available():
        oracle_ref.load().qref_set_threads(threads)
        problem = oracle_ref.make_problem(intensity, None, mask)
        solver = oracle_ref.Solver(problem, starts=starts, seed=0)
        t0 = time.perf_counter()
        solver.run(recipe)
        return time.perf_counter() - t0, "reference", "QoraPhaseCU CpuSolver (OpenMP loops, project FFT shim)"
    import numpy as np

    from oracle import fp64

    problem = fp64.make_problem(intensity, None, mask)
    solver = fp64.Solver(problem, starts=starts, dtype=np.complex64, fft="scipy", workers=threads)
    t0 = time.perf_counter()
    solver.run(recipe)
    return time.perf_counter() - t0, "port", "numpy port of CpuSolver::iterate, scipy.fft (pocketfft)"


def cpu_baseline(intensity, mask, port=False):
    """The CPU figure beside the GPU line: one untimed step, then one timed step."""
    threads = len(os.sched_getaffinity(0))
    starts = PORT_SAMPLE_STARTS if port else CPU_SAMPLE_STARTS
    reference_step(intensity, mask, starts, threads, port)
    seconds, kind, label = reference_step(intensity, mask, starts, threads, port)
    return {
        "value": starts * 700 / seconds,
        "unit": UNIT,
        "cores": threads,
        "kind": kind,
        "sample": f"the whole 700-iteration recipe on {starts} of the 32 starts ({label}), "
                  f"{seconds:.2f} s",
    }


def run_reference(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    from qoraphasecu_b200 import workloads

    _, intensity, mask = workloads.gaussians(SHAPE[0], seed=SEED)
    threads = len(os.sched_getaffinity(0))
    for _ in range(args.warmup):
        reference_step(intensity, mask, CPU_SAMPLE_STARTS, threads)
    seconds = []
    for _ in range(args.steps):
        t, kind, label = reference_step(intensity, mask, CPU_SAMPLE_STARTS, threads)
        seconds.append(t)
    total = sum(seconds)
    value = CPU_SAMPLE_STARTS * 700 * args.steps / total
    sample = (f"each step: the whole 700-iteration recipe on starts 0-{CPU_SAMPLE_STARTS - 1} of "
              f"the 32 ({label}); {args.steps} steps in {total:.1f} s")
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded gaussians generator, seed 1000; random starts seed 0)",
        "config": config_of(args, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


REFERENCE_GPU_VARIANTS = {"graph": 2, "batched": 3, "half": 4, "mixed": 6}  # qpcu::Variant


def reference_gpu_baseline(intensity, mask, sync_every, *, starts=None, recipe=None):
    """The reference's own CUDA backend (src/cuda: cuFFT plans, its element-wise
    kernels, CUDA graphs) compiled from its sources (oracle/_ref/
    libqpcu_ref_cuda.so, cuFFT LTO callbacks off) on the same workload, timed
    as its bench/bench.cpp:33-45 does: per variant, one run of the whole recipe
    to warm up (plans, graphs), then one timed run, wall clock around run()
    (which ends with the errors copied to the host). Defaults: the benchmark's
    32 starts and recipe; the support is the reference's autocorrelation
    support (problem.cpp) unless the workload passes none either way."""
    import ctypes

    import numpy as np

    from oracle import ref as oracle_ref
    from qoraphasecu_b200 import workloads

    if not oracle_ref.CUDA_LIBRARY.exists():
        return {"unavailable": "oracle/_ref/libqpcu_ref_cuda.so was not built"}
    lib = oracle_ref.load_variant("cuda")
    if not lib.qref_cuda_available():
        return {"unavailable": "no CUDA device"}
    starts = starts or STARTS
    recipe = recipe or workloads.gaussians_recipe()
    iterations = recipe.iterations()
    amp, msk, sup = oracle_ref.make_problem(intensity, None, mask)
    ops = oracle_ref._ops(recipe.ops())
    count = len(recipe.ops())
    out = {"source": "QoraPhaseCU src/cuda compiled from its sources (nvcc sm_100a, cuFFT "
                     "11.4, LTO callbacks off)", "starts": starts, "sync_every": sync_every}
    for name, variant in REFERENCE_GPU_VARIANTS.items():
        handle = ctypes.c_void_p()
        status = lib.qref_create_backend(oracle_ref._p(amp), oracle_ref._p(msk),
                                         oracle_ref._p(sup), amp.ndim,
                                         oracle_ref._shape(amp.shape), starts,
                                         ctypes.c_uint64(0), None, sync_every, 1, variant, 0,
                                         ctypes.byref(handle))
        if status:
            out[name] = {"error": lib.qref_last_error().decode()}
            continue
        try:
            if lib.qref_run(handle, ops, count):
                out[name] = {"error": lib.qref_last_error().decode()}
                continue
            t0 = time.perf_counter()
            status = lib.qref_run(handle, ops, count)
            seconds = time.perf_counter() - t0
            if status:
                out[name] = {"error": lib.qref_last_error().decode()}
                continue
            n_err = lib.qref_error_count(handle)
            errors = np.empty((starts, n_err), np.float32)
            lib.qref_results(handle, None, None, oracle_ref._p(errors),
                             ctypes.byref(ctypes.c_size_t()))
            out[name] = {"value": starts * iterations / seconds, "unit": UNIT,
                         "us_per_iteration": seconds / iterations * 1e6,
                         "best_final_error": float(errors[:, -1].min())}
        finally:
            lib.qref_destroy(handle)
    return out


def parity_check(solver_kwargs, intensity, mask):
    """RAAR(0.9) x 2 from the timed solver's starts against the FP64 oracle
    (outside any timed region): the largest relative difference of the
    per-iteration Fourier errors and the largest relative L2 difference of the
    objects over all 32 starts."""
    import numpy as np

    import qoraphasecu_b200 as qpc
    from oracle import fp64
    from qoraphasecu_b200.recipe import RAAR, Recipe

    problem = qpc.make_problem(intensity, mask=mask)
    with qpc.Solver(problem, **solver_kwargs) as s:
        s.run(Recipe(RAAR(2, 0.9)))
        ours = s.results()
    ref = fp64.reconstruct(fp64.make_problem(intensity, None, mask), [fp64.op("raar", 2, 0.9)],
                           starts=solver_kwargs["starts"], seed=solver_kwargs["seed"])
    err = max(float(np.max(np.abs(r.errors - e) / e)) for r, (_, _, e) in zip(ours, ref))
    obj = max(fp64.relative_diff(r.object, o) for r, (o, _, _) in zip(ours, ref))
    return {"recipe": "RAAR(0.9) x 2, all 32 starts, the timed solver's options",
            "against": "FP64 oracle (numpy complex128 restatement of CpuSolver)",
            "error_rel_max": err, "object_rel_l2_max": obj, "bar": 1e-5,
            "ok": bool(err < 1e-5 and obj < 1e-5)}


def run_profile(iterations, schedule="streamed", workload=None):
    """The benchmark workload cut to a few iterations, all 32 starts in one
    launch per pass and no autotuning, so that an ncu capture sees each line
    pass after a short set-up: make_problem, solver construction, `iterations`
    RAAR iterations. With workload "crystal": the 128^3 crystal, its 4 starts
    in one launch per pass, `iterations` HIO iterations."""
    import qoraphasecu_b200 as qpc
    from qoraphasecu_b200 import workloads
    from qoraphasecu_b200.recipe import HIO, RAAR, Recipe

    if workload == "crystal":
        _, intensity = workloads.crystal(128, seed=3000)
        problem = qpc.make_problem(intensity)
        with qpc.Solver(problem, starts=4, seed=0, batch=4, schedule="streamed",
                        sync_every=1) as solver:
            solver.run(Recipe(HIO(iterations, 0.9)))
            print(json.dumps({"profile_iterations": iterations, "workload": "crystal",
                              "kernels": qpc.kernel_launches(),
                              "final_errors": [float(r.error) for r in solver.results()]}))
        return 0
    _, intensity, mask = workloads.gaussians(SHAPE[0], seed=SEED)
    problem = qpc.make_problem(intensity, mask=mask)
    if schedule == "resident":
        # one launch runs every iteration
        kw = dict(schedule="resident", sync_every=iterations)
    else:
        kw = dict(schedule="streamed", batch=STARTS, sync_every=1)
    with qpc.Solver(problem, starts=STARTS, seed=0, variant="batched", **kw) as solver:
        solver.run(Recipe(RAAR(iterations, 0.9)))
        print(json.dumps({"profile_iterations": iterations,
                          "kernels": qpc.kernel_launches(),
                          "final_errors": [float(r.error) for r in solver.results()[:4]]}))
    return 0


def run_profile_step(sync_every, batch=0, schedule="auto"):
    """One benchmark step (the whole recipe over 32 starts) after the solver is
    built, for an ncu launch list of the timed work. The autotuner times its
    candidates by wall clock, which a profiler distorts, so a launch list is
    taken with the schedule fixed (--batch/--schedule) to the one a plain run
    picks."""
    import qoraphasecu_b200 as qpc
    from qoraphasecu_b200 import workloads

    _, intensity, mask = workloads.gaussians(SHAPE[0], seed=SEED)
    problem = qpc.make_problem(intensity, mask=mask)
    with qpc.Solver(problem, starts=STARTS, seed=0, sync_every=sync_every, batch=batch or None,
                    schedule=schedule) as solver:
        before = qpc.kernel_launches()
        solver.run(workloads.gaussians_recipe())
        print(json.dumps({"step_kernels": qpc.kernel_launches() - before,
                          "tuning": qpc.api.tuning_report().strip()}))
    return 0


# ----------------------------------------------------- the other synthetic workloads
def tuned_batch(report):
    """Starts per launch the autotuner chose for the benchmark shape and start
    count (its report line "shape 1x256x256 starts 32 storage 0: batch 8 (...)"),
    "resident" for the resident schedule, None when it has not run."""
    key = f"shape 1x{SHAPE[0]}x{SHAPE[1]} starts {STARTS} storage 0: "
    for line in report.splitlines():
        if key in line:
            choice = line.split(key, 1)[1]
            if choice.startswith("batch "):
                return int(choice.split()[1])
            return choice.split()[0]  # "resident" or "persistent"
    return None


def _timed(fn, warmup=1, reps=3):
    """Median wall time of fn() after `warmup` calls (each call synchronises)."""
    for _ in range(warmup):
        fn()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t0)
    return statistics.median(times)


def workload_square(args):
    """64x64 square object (uniform amplitude and phase in a 24x24 box),
    noiseless, no mask, autocorrelation support, default recipe (720
    iterations), 8 starts, through the public reconstruct()."""
    import qoraphasecu_b200 as qpc
    from qoraphasecu_b200 import workloads

    obj = workloads.square(64, seed=0)
    intensity = workloads.simulate_intensity(obj)
    out = {}
    for storage in ("f32", "f16", "bf16"):
        ens = None

        def run():
            nonlocal ens
            ens = qpc.reconstruct(intensity, starts=8, seed=0, amp_storage=storage)

        s = _timed(run, warmup=args.warmup, reps=args.steps)
        out[storage] = {"start_iterations_per_s": 8 * 720 / s, "seconds": s,
                        "best_error": ens.best.error, "errors": [r.error for r in ens]}
    return {"workload": "square 64x64, 8 starts, default_recipe (720 iterations), e2e reconstruct()",
            "storage": out, "tuning": qpc.api.tuning_report().strip().splitlines()}


def workload_uneven(args):
    """64 problems with sides drawn from {64, 128, 256, 512}, square objects
    scaled to the side, Poisson 1e6, beamstop n/32, 4 starts each, recipe
    repeat(4, HIO(50), Shrinkwrap(rms 0.3)), ER(100), in one BatchSolver."""
    import numpy as np

    import qoraphasecu_b200 as qpc
    from qoraphasecu_b200 import workloads

    batch = workloads.uneven_batch(count=64, seed=2000)
    recipe = workloads.uneven_recipe()
    intensities = [b[1] for b in batch]
    masks = [b[2] for b in batch]
    sides = [int(b[1].shape[0]) for b in batch]
    elements = sum(s * s for s in sides)
    result = {}

    # Each call: make_problem for every intensity (autocorrelation supports),
    # the recipe, the results; the previous call's results are dropped first,
    # as a caller that consumed them would, so their host memory is reused.
    def run():
        result.clear()
        result["runs"] = qpc.reconstruct_batch(intensities, masks=masks, recipe=recipe, starts=4,
                                               seed=0, sync_every=50)

    s = _timed(run, warmup=args.warmup, reps=args.steps)
    qpc.api.clear_cache()
    problems = [qpc.make_problem(i, mask=m) for i, m in zip(intensities, masks)]

    def run_new_solver():
        result.clear()
        with qpc.BatchSolver(problems, starts=4, seed=0, sync_every=50) as solver:
            solver.run(recipe)
            result["runs"] = [tuple(r) for r in solver.results()]

    s_new = _timed(run_new_solver, warmup=1, reps=args.steps)
    iters = recipe.iterations()
    best = [min(r.error for r in runs) for runs in result["runs"]]
    per_side = {}
    for side, b in zip(sides, best):
        per_side.setdefault(side, []).append(b)
    return {
        "workload": "uneven batch: 64 problems, sides {64,128,256,512}, 4 starts, "
                    "repeat(4, HIO(50), Shrinkwrap(rms 0.3)), ER(100); each timed call is one "
                    "reconstruct_batch over the 64 host intensities (make_problem with "
                    "autocorrelation supports, the batch solver of the previous call reloaded, "
                    "random starts, the recipe, host results); the warm-up calls leave the "
                    "autotuner's choices and the solver cached",
        "problems_per_side": {str(k): len(v) for k, v in sorted(per_side.items())},
        "seconds": s,
        "seconds_new_batch_solver": s_new,
        "start_iterations_per_s": 64 * 4 * iters / s,
        "element_iterations_per_s": 4 * elements * iters / s,
        "best_error_median_per_side": {str(k): float(np.median(v))
                                       for k, v in sorted(per_side.items())},
        "tuning": qpc.api.tuning_report().strip().splitlines(),
    }


def workload_adam(args):
    """Differentiable reconstruction: one 512x512 square-object problem (box
    192, Poisson 1e7, beamstop r 12), a batch of 16 objects (random starts),
    500 Adam steps (lr 1e-2) on the amplitude loss with the support projection
    and the default magnitude bound, against RAAR(0.9) from the same starts for
    the same wall time; object sanity (largest pixel over the RMS amplitude the
    support carries) with and without the bound."""
    import numpy as np

    import qoraphasecu_b200 as qpc
    from qoraphasecu_b200 import autograd as qad
    from qoraphasecu_b200 import workloads
    from qoraphasecu_b200.recipe import RAAR, Recipe

    rng = np.random.default_rng(4000)
    obj = workloads.square(512, seed=4000)
    intensity = workloads.poisson(workloads.simulate_intensity(obj), 1e7, rng)
    problem = qpc.make_problem(intensity, mask=workloads.beamstop((512, 512), 12))
    qad.adam_reconstruct(problem, starts=16, steps=5, seed=0)  # warm-up
    # Each call draws its starts, captures its step graph and returns host
    # results, which moves its wall time by tens of milliseconds between calls:
    # three calls of 500 steps (median), and one of 1000 steps, whose excess
    # over the median is the time of 500 steps alone.
    runs_s = []
    for _ in range(3):
        t0 = time.perf_counter()
        adam = qad.adam_reconstruct(problem, starts=16, steps=500, lr=1e-2, seed=0)
        runs_s.append(time.perf_counter() - t0)
    t_adam = float(np.median(runs_s))
    t0 = time.perf_counter()
    qad.adam_reconstruct(problem, starts=16, steps=1000, lr=1e-2, seed=0)
    t_long = time.perf_counter() - t0
    free = qad.adam_reconstruct(problem, starts=16, steps=500, lr=1e-2, seed=0, bound=None)
    usable = np.asarray(problem.mask) == 0
    inside = max(int(np.count_nonzero(problem.support)), 1)
    rms = float(np.sqrt(np.sum(np.asarray(problem.amplitude, np.float64)[usable] ** 2) / inside))

    def largest(runs):
        return float(max(np.max(np.abs(r.object)) for r in runs) / rms)

    with qpc.Solver(problem, starts=16, seed=0, sync_every=50) as s:
        s.run(Recipe(RAAR(50, 0.9)))  # warm-up: tuning, graphs
    with qpc.Solver(problem, starts=16, seed=0, sync_every=50) as s:
        t0 = time.perf_counter()
        s.run(Recipe(RAAR(100, 0.9)))
        per_iter = (time.perf_counter() - t0) / 100
    n_raar = max(1, int(t_adam / per_iter))
    with qpc.Solver(problem, starts=16, seed=0, sync_every=50) as s:
        t0 = time.perf_counter()
        s.run(Recipe(RAAR(n_raar, 0.9)))
        t_raar = time.perf_counter() - t0
        raar = s.results()
    return {
        "workload": "square 512x512 (box 192), Poisson 1e7, beamstop r 12, 16 starts: "
                    "Adam(lr 1e-2) x 500 on sum_unmasked (|Fx| - sqrt(I))^2 with support "
                    "projection vs RAAR(0.9) for the same wall time",
        "adam": {"steps": 500, "seconds": t_adam, "steps_per_s": 500 / t_adam,
                 "seconds_per_call": runs_s, "seconds_1000_steps": t_long,
                 "steady_steps_per_s": 500 / (t_long - t_adam) if t_long > t_adam else None,
                 "final_error_median": float(np.median([r.error for r in adam])),
                 "final_error_best": float(min(r.error for r in adam)),
                 "bound": 16.0, "largest_pixel_over_rms": largest(adam)},
        "adam_unbounded": {"final_error_median": float(np.median([r.error for r in free])),
                           "largest_pixel_over_rms": largest(free)},
        "raar": {"iterations": n_raar, "seconds": t_raar, "largest_pixel_over_rms": largest(raar),
                 "final_error_median": float(np.median([r.error for r in raar])),
                 "final_error_best": float(min(r.error for r in raar))},
    }


def workload_crystal(args):
    """128^3 faceted crystal (12 half-spaces in a sphere of radius 40,
    displacement-field phase), Poisson 1e7, no mask, autocorrelation support,
    default recipe (720 iterations), 4 starts batched, FP32 and FP16 storage."""
    import qoraphasecu_b200 as qpc
    from qoraphasecu_b200 import workloads
    from qoraphasecu_b200.recipe import default_recipe

    _, intensity = workloads.crystal(128, seed=3000)
    problem = qpc.make_problem(intensity)
    out = {}
    for name, kw in (("f32", dict(amp_storage="f32")), ("f16 amplitude", dict(amp_storage="f16")),
                     ("half (fp16 iterate and wave)", dict(variant="half")),
                     ("mixed (fp16 wave for HIO/RAAR)", dict(variant="mixed"))):
        with qpc.Solver(problem, starts=4, seed=0, sync_every=50, **kw) as s:
            s.run(default_recipe())  # warm-up: tuning, graphs
            t0 = time.perf_counter()
            s.run(default_recipe())
            sec = time.perf_counter() - t0
            runs = s.results()
            pass_ms = s.profile_passes(5)
        out[name] = {"seconds": sec, "start_iterations_per_s": 4 * 720 / sec,
                     "errors": [r.error for r in runs], "pass_ms": pass_ms}
    reference = reference_gpu_baseline(intensity, None, 50, starts=4, recipe=default_recipe())
    return {"workload": "crystal 128^3, Poisson 1e7, 4 starts, default_recipe (720 iterations, "
                        "continued from a first run)", "storage": out,
            "reference_gpu_baseline": reference,
            "tuning": qpc.api.tuning_report().strip().splitlines()}


WORKLOADS = {"square": workload_square, "uneven": workload_uneven, "adam": workload_adam,
             "crystal": workload_crystal}


# ---------------------------------------------------------------------- our arm
def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--sync-every", type=int, default=50)
    parser.add_argument("--batch", type=int, default=0,
                        help="starts per launch; groups run as parallel graph branches (0 = all)")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    parser.add_argument("--no-extras", action="store_true", help="skip plain / f16 / e2e legs")
    parser.add_argument("--profile", type=int, default=0, metavar="ITERS",
                        help="only build the workload and run ITERS RAAR iterations (for ncu; "
                             "with --workload crystal, ITERS HIO iterations of the 128^3 crystal)")
    parser.add_argument("--schedule", choices=("auto", "streamed", "resident"), default="auto",
                        help="batched schedule of the timed solver (auto = autotuned)")
    parser.add_argument("--workload", choices=sorted(WORKLOADS), default=None,
                        help="report one of the other synthetic workloads instead of the "
                             "benchmark line (--steps timed runs after --warmup)")
    parser.add_argument("--profile-step", action="store_true",
                        help="only build the workload and run one benchmark step (for ncu)")
    args = parser.parse_args(argv)
    if args.profile:
        return run_profile(args.profile, "resident" if args.schedule == "resident" else "streamed",
                           args.workload)
    if args.profile_step:
        return run_profile_step(args.sync_every, args.batch, args.schedule)
    if args.workload:
        print(json.dumps({"workload_report": args.workload, **WORKLOADS[args.workload](args)}))
        return 0
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch

    import qoraphasecu_b200 as qpc
    from qoraphasecu_b200 import workloads

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    qpc.api.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    from qoraphasecu_b200.replicas import max_over_ranks, rank_seed

    seed = rank_seed(0, rank)  # replicas draw distinct random starts

    _, intensity, mask = workloads.gaussians(SHAPE[0], seed=SEED)
    recipe = workloads.gaussians_recipe()
    iters = recipe.iterations()
    stream = torch.cuda.current_stream()
    problem = qpc.make_problem(intensity, mask=mask)
    solver_kwargs = dict(starts=STARTS, seed=seed, sync_every=args.sync_every,
                         batch=args.batch or None, device=local, stream=stream.cuda_stream,
                         schedule=args.schedule)
    solver = qpc.Solver(problem, **solver_kwargs)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        solver.run(recipe)
    barrier()

    step_ms = []
    launches0 = qpc.api.kernel_launches()
    t_wall = time.perf_counter()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()  # L2 flushed between steps (outside the step events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solver.run(recipe)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
        barrier()
    wall_s = time.perf_counter() - t_wall
    launches = qpc.api.kernel_launches() - launches0
    total_ms = max_over_ranks(sum(step_ms))
    value = world * STARTS * iters * args.steps / (total_ms / 1e3)

    # Per-kernel device time: every pass of an iteration launched directly
    # between CUDA events on the same stream, all 32 starts in one launch.
    with qpc.Solver(problem, starts=STARTS, seed=seed, batch=STARTS, device=local,
                    stream=stream.cuda_stream) as single:
        single.run(workloads.hio_recipe(5))
        pass_ms = single.profile_passes(20)
    elems = STARTS * SHAPE[0] * SHAPE[1]
    # The same two kernels on more starts of the problem, whose iterate and
    # wave (128 starts: 134 MB; 512 starts: 537 MB) no longer fit in L2: one
    # launch per pass, outside the timed region.
    beyond_l2 = []
    for starts in (128, 512):
        with qpc.Solver(problem, starts=starts, seed=seed, batch=starts, device=local,
                        stream=stream.cuda_stream) as big:
            big.run(workloads.hio_recipe(5))
            big_ms = big.profile_passes(20)
        n_big = starts * SHAPE[0] * SHAPE[1]
        beyond_l2.append({"starts": starts, **{
            name.split(" ")[0]: {"ms": ms, "gbs": bpe * n_big / (ms * 1e6)}
            for (name, bpe), ms in zip(PASS_BYTES.items(), big_ms)}})
    passes = []
    for (name, bpe), ms in zip(PASS_BYTES.items(), pass_ms):
        unfused = UNFUSED_BYTES[name] * elems
        passes.append({"pass": name, "ms": ms, "bytes": bpe * elems, "gbs": bpe * elems / (ms * 1e6),
                       "unfused_equivalent_gbs": unfused / (ms * 1e6)})
    # The dominant kernel is the pass with the largest share of the step's
    # device time in the committed ncu launch list (its `dominant_kernel:`
    # line); the two passes' shares and single-launch times are close, so
    # picking the larger of two measured times would flip between runs. Both
    # passes are reported.
    dominant_name = profile_value("dominant_kernel") or "modulus"
    dominant = passes[0] if dominant_name == "modulus" else passes[1]
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic(dominant_name)
    # The whole iteration in the timed graph (parallel start groups, shrinkwrap
    # amortised): the minimum 21 B per element per iteration (iterate in and
    # out, amplitude, support) and the bytes the two fused passes move.
    iter_ms = total_ms / args.steps / iters
    fused_bytes = sum(PASS_BYTES.values()) * elems
    roofline = {
        "bound": "hbm",
        "kernel": dominant["pass"],
        "achieved": dominant["gbs"],
        "peak": peak,
        "peak_source": f"{peak_kind} hbm_gbs",
        "unit": "GB/s",
        "frac": dominant["gbs"] / peak,
        "traffic": traffic,
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, from the "
                          "committed summary under profiles/ (not measured in this run)",
        "passes": passes,
        "iteration": {
            "us": iter_ms * 1e3,
            "min_bytes": 21 * elems,
            "fused_pass_bytes": fused_bytes,
            "achieved_min_gbs": 21 * elems / (iter_ms * 1e6),
            "achieved_pass_gbs": fused_bytes / (iter_ms * 1e6),
        },
        "note": "32 starts x 256^2 (16 MiB iterate) stay L2-resident across an iteration; "
                "a launch of all 32 starts runs the modulus pass's 7-CTAs-per-SM variant "
                "(the timed graph's 4-start launches run the default 5 per SM)",
        "passes_beyond_l2": beyond_l2,
    }

    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded gaussians generator, seed 1000; random starts seed = rank)",
        "config": config_of(args, world),
        "schedule": {
            "variant": "batched, graph-captured",
            "starts_per_launch": args.batch or tuned_batch(qpc.api.tuning_report()),
            "sync_every": args.sync_every,
        },
        "gpu_launches": launches,
        "tuning": qpc.api.tuning_report().strip().splitlines(),
        "wall_s_timed_region": wall_s,
        "roofline": roofline,
    }

    if not args.no_extras:
        # Plain per-start path (the in-repo baseline), one step.
        plain = qpc.Solver(problem, starts=STARTS, seed=seed, sync_every=args.sync_every,
                           variant="plain", device=local, stream=stream.cuda_stream)
        plain.run(recipe)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plain.run(recipe)
        e1.record(stream)
        e1.synchronize()
        plain_ms = max_over_ranks(e0.elapsed_time(e1))
        plain.close()
        plain_value = world * STARTS * iters / (plain_ms / 1e3)
        # FP16 amplitude storage, same schedule.
        half = qpc.Solver(problem, starts=STARTS, seed=seed, sync_every=args.sync_every,
                          amp_storage="f16", device=local, stream=stream.cuda_stream)
        half.run(recipe)
        barrier()
        e0.record(stream)
        half.run(recipe)
        e1.record(stream)
        e1.synchronize()
        half_ms = max_over_ranks(e0.elapsed_time(e1))
        half.close()
        line["variants"] = {
            "plain_per_start": {"value": plain_value, "ms_per_step": plain_ms},
            "batched_over_plain": value / plain_value,
            "f16_amplitude": {"value": world * STARTS * iters / (half_ms / 1e3), "ms_per_step": half_ms},
        }
        # fp16 storage of the wave (and the iterate): the reference's half and
        # mixed variants, same schedule choice by the autotuner.
        for variant in ("half", "mixed"):
            with qpc.Solver(problem, starts=STARTS, seed=seed, sync_every=args.sync_every,
                            variant=variant, device=local, stream=stream.cuda_stream) as v:
                v.run(recipe)
                barrier()
                e0.record(stream)
                v.run(recipe)
                e1.record(stream)
                e1.synchronize()
                v_ms = max_over_ranks(e0.elapsed_time(e1))
                best = float(min(r.error for r in v.results()))
            line["variants"][f"f16_wave_{variant}"] = {
                "value": world * STARTS * iters / (v_ms / 1e3), "ms_per_step": v_ms,
                "best_final_error": best}

        # End to end through the public API with host buffers: intensity from
        # pinned memory in, objects/supports/errors out, every step.
        pinned = torch.empty(intensity.shape, dtype=torch.float32, pin_memory=True)
        pinned.numpy()[...] = intensity
        host_in = pinned.numpy()
        times = []
        for k in range(args.warmup + args.steps):
            barrier()
            t0 = time.perf_counter()
            ens = qpc.reconstruct(host_in, mask=mask, recipe=recipe, starts=STARTS, seed=seed,
                                  sync_every=args.sync_every)
            times.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(statistics.median(times[args.warmup:]))
        n = SHAPE[0] * SHAPE[1]
        line["e2e"] = {
            "value": world * STARTS * iters / e2e_s,
            "unit": UNIT,
            # up: the intensity for the autocorrelation support (4 B), then the
            # amplitude, mask and support the solver prepares on the device
            # (4 + 1 + 1 B); down: the support (1 B), every start's object and
            # support (8 + 1 B) and its FP64 error history
            "h2d_bytes_per_step": int(n * (4 + 4 + 1 + 1)),
            "d2h_bytes_per_step": int(n * 1 + STARTS * n * (8 + 1) + STARTS * iters * 8),
            "seconds_per_step": e2e_s,
            "path": "qoraphasecu_b200.reconstruct (make_problem + solver + results)",
        }
        del ens

    line["clocks"] = clocks.summary()
    if rank == 0 and world == 1 and not args.no_cpu:
        # The CPU leg, after every timed region: the reference's CPU path as the
        # baseline, and the FP64 oracle as the checker of the timed solver's
        # first two iterations.
        line["cpu_baseline"] = cpu_baseline(intensity, mask)
        if line["cpu_baseline"]["kind"] == "reference":
            # the second CPU figure: the same recipe on pocketfft (scipy.fft),
            # the FFT the reference's CPU backend links
            line["cpu_baseline_pocketfft"] = cpu_baseline(intensity, mask, port=True)
        line["parity"] = parity_check(solver_kwargs, intensity, mask)
        line["reference_gpu_baseline"] = reference_gpu_baseline(intensity, mask, args.sync_every)
    solver.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
