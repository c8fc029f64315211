#!/usr/bin/env python3
"""Error of the B200 backend against the FP64 oracle on every synthetic
workload, for FP32, FP16 and BF16 amplitude storage. Needs a GPU; prints one
JSON line per workload.

    python tests/precision_report.py [--full] [--only NAME ...]

For each workload and storage: prefixes of 2 and 10-20 iterations from the
same seeds (the random starts are bit-identical by construction) compared
start by start with the oracle -- the largest relative difference of the
per-iteration Fourier errors and the relative L2 difference of the objects --
and, where the oracle finishes in about a minute (or everywhere with --full),
the whole recipe: the best start's final Fourier error and its object error
against the ground truth (scaled to the data) after phase-ramp and twin
alignment. Every comparison is repeated for the oracle's own FP32 port
(complex64 numpy): iterative recipes are chaotic, and on some problems
rounding alone moves an HIO or RAAR run by order one within 20 iterations;
the port's numbers show how far it carries each recipe on each problem.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent))

from oracle import fp64  # noqa: E402

import qoraphasecu_b200 as qpc  # noqa: E402
from qoraphasecu_b200 import autograd as qad  # noqa: E402
from qoraphasecu_b200 import workloads  # noqa: E402
from qoraphasecu_b200.recipe import HIO, RAAR, Recipe, default_recipe  # noqa: E402

STORAGES = ("f32", "f16", "bf16")
WORKERS = len(os.sched_getaffinity(0))


def oracle_runs(intensity, support, mask, ops, starts, seed=0, dtype=np.complex128):
    problem = fp64.make_problem(intensity, support, mask)
    solver = fp64.Solver(problem, starts=starts, seed=seed, fft="scipy", workers=WORKERS,
                         dtype=dtype)
    solver.run(ops)
    return solver.results()


def gpu_runs(problem, recipe, starts, storage, seed=0):
    with qpc.Solver(problem, starts=starts, seed=seed, amp_storage=storage, sync_every=50) as s:
        s.run(recipe)
        return s.results()


def diffs(runs, ref):
    """Largest relative difference of the error histories and of the objects."""
    err = max(float(np.max(np.abs(np.asarray(r[2]) - e) / np.maximum(e, 1e-12)))
              for (_, _, e), r in zip(ref, runs))
    obj = max(fp64.relative_diff(r[0], o) for (o, _, _), r in zip(ref, runs))
    return {"max_rel_error_diff": err, "max_object_rel_l2": obj}


def prefix(intensity, support, mask, recipe, starts):
    """Start-by-start comparison over a short recipe, per storage, beside the
    same comparison for the oracle's own FP32 port: how far rounding alone
    carries this recipe on this problem."""
    ref = oracle_runs(intensity, support, mask, recipe.ops(), starts)
    port = oracle_runs(intensity, support, mask, recipe.ops(), starts, dtype=np.complex64)
    problem = qpc.make_problem(intensity, support=support, mask=mask)
    out = {"fp32_port": diffs(port, ref)}
    for storage in STORAGES:
        ours = [(r.object, r.support, r.errors) for r in gpu_runs(problem, recipe, starts, storage)]
        out[storage] = diffs(ours, ref)
    return {"recipe": repr(recipe.ops()), "starts": starts, "storage": out}


def prefixes(intensity, support, mask, kind, starts, lengths=(2, 20)):
    ops = {"raar": lambda n: Recipe(RAAR(n, 0.9)), "hio": lambda n: Recipe(HIO(n))}[kind]
    return {str(n): prefix(intensity, support, mask, ops(n), starts) for n in lengths}


def scaled_truth(truth, intensity):
    """The ground truth at the data's scale (Parseval with the unitary FFT)."""
    scale = np.sqrt(float(np.sum(intensity, dtype=np.float64)) /
                    float(np.sum(np.abs(truth.astype(np.complex128)) ** 2)))
    return truth * scale


def whole(intensity, support, mask, recipe, starts, truth):
    """Best start's final error and aligned object error for ours, the FP64
    oracle and its FP32 port."""
    truth = scaled_truth(truth, intensity)
    out = {}
    ref_err = ref_obj = None
    for name, dtype in (("oracle_fp64", np.complex128), ("fp32_port", np.complex64)):
        t0 = time.perf_counter()
        runs = oracle_runs(intensity, support, mask, recipe.ops(), starts, dtype=dtype)
        best = min(runs, key=lambda r: r[2][-1])
        err, obj = float(best[2][-1]), fp64.aligned_error(best[0], truth)
        if ref_err is None:
            ref_err, ref_obj = err, obj
        out[name] = {"best_final_error": err, "aligned_object_error": obj,
                     "seconds": time.perf_counter() - t0}
    problem = qpc.make_problem(intensity, support=support, mask=mask)
    for storage in STORAGES:
        b = min(gpu_runs(problem, recipe, starts, storage), key=lambda r: r.error)
        out[storage] = {"best_final_error": b.error,
                        "aligned_object_error": fp64.aligned_error(b.object, truth)}
    for v in out.values():
        v["final_error_diff"] = abs(v["best_final_error"] - ref_err)
        v["object_error_diff"] = abs(v["aligned_object_error"] - ref_obj)
    return out


def square_64(full):
    obj = workloads.square(64, seed=0)
    intensity = workloads.simulate_intensity(obj)
    support = qpc.autocorrelation_support(intensity)
    return {"workload": "square 64x64, 8 starts, default_recipe, noiseless, autocorrelation support",
            "prefix": prefixes(intensity, support, None, "raar", 8),
            "whole_recipe": whole(intensity, support, None, default_recipe(), 8, obj)}


def gaussians_256(full):
    obj, intensity, mask = workloads.gaussians(256, seed=1000)
    support = qpc.autocorrelation_support(intensity)
    out = {"workload": "gaussians 256x256, 32 starts, repeat(10, RAAR(50,0.9), Shrinkwrap(0.3,1)), "
                       "ER(200), Poisson 1e6, beamstop 8",
           "prefix": prefixes(intensity, support, mask, "raar", 32)}
    if full:
        out["whole_recipe"] = whole(intensity, support, mask, workloads.gaussians_recipe(), 32, obj)
    return out


def uneven(full):
    batch = workloads.uneven_batch(count=64, seed=2000)
    by_side = {}
    names = ("fp32_port",) + STORAGES
    for obj, intensity, mask in batch:
        support = qpc.autocorrelation_support(intensity)
        res = prefixes(intensity, support, mask, "hio", 4)
        side = by_side.setdefault(str(obj.shape[0]), {"problems": 0})
        side["problems"] += 1
        for n, r in res.items():
            cur = side.setdefault(n, {k: {"max_rel_error_diff": 0.0, "max_object_rel_l2": 0.0}
                                      for k in names})
            for k in names:
                for m in ("max_rel_error_diff", "max_object_rel_l2"):
                    cur[k][m] = max(cur[k][m], r["storage"][k][m])
    return {"workload": "uneven batch, 64 problems, sides {64,128,256,512}, 4 starts; per side "
                        "and prefix length (HIO iterations) the worst problem, from the same seeds",
            "prefix_by_side": by_side}


def adjoint_512(full):
    import torch

    rng = np.random.default_rng(4000)
    obj = workloads.square(512, seed=4000)
    intensity = workloads.poisson(workloads.simulate_intensity(obj), 1e7, rng)
    mask = workloads.beamstop((512, 512), 12)
    ref_p = fp64.make_problem(intensity, None, mask)
    p = qpc.make_problem(intensity, mask=mask)
    model = qad.AmplitudeModel(p)
    x = (obj + 0.1 * (rng.standard_normal(obj.shape) + 1j * rng.standard_normal(obj.shape))
         ).astype(np.complex64)
    xt = torch.from_numpy(np.ascontiguousarray(np.fft.ifftshift(x))).cuda()[None]
    loss, grad = qad._loss_and_grad(xt, model.signed, model.shape)
    g = np.fft.fftshift(grad[0].cpu().numpy())
    projected, _ = fp64.modulus_project(ref_p, x)
    identity = 2.0 * (x.astype(np.complex128) - projected)
    fft = fp64.Fft(2, backend="scipy", workers=WORKERS)
    y = fft.forward(fp64.to_fft_order(x.astype(np.complex128)))
    amp = fp64.to_fft_order(ref_p.amplitude).astype(np.float64)
    usable = fp64.to_fft_order(ref_p.mask) == 0
    ref_loss = float(np.sum(np.where(usable, (np.abs(y) - amp) ** 2, 0.0)))
    return {"workload": "square 512x512 (box 192), Poisson 1e7, beamstop 12: amplitude loss and "
                        "its gradient at a perturbed truth (FP32 amplitude)",
            "loss_rel_diff": abs(float(loss[0].item()) - ref_loss) / ref_loss,
            "gradient_rel_l2_vs_2(x-P_M x)": fp64.relative_diff(g, identity)}


def _adam_fp64(x0, scale, amp, usable, support, steps, lr, bound):
    """The Adam reconstruction of qoraphasecu_b200.autograd.adam_reconstruct
    in FP64 on the host (torch, complex128, torch.fft in place of the line
    passes): Adam on the real view of w = x / scale, the loss
    sum_usable (|F x| - A)^2 with F the unitary FFT, then the support
    projection and the magnitude bound. Returns the objects x (FFT order) and
    the Fourier error sqrt(loss / energy) of every step."""
    import torch

    w = torch.view_as_real(torch.from_numpy(x0 / scale)).clone().requires_grad_(True)
    opt = torch.optim.Adam([w], lr=lr)
    amp_t = torch.from_numpy(amp)
    usable_t = torch.from_numpy(usable.astype(np.float64))
    support_t = torch.from_numpy(support.astype(np.float64))
    energy = float(np.sum(np.where(usable, amp ** 2, 0.0)))
    errors = []
    for _ in range(steps):
        opt.zero_grad()
        y = torch.fft.fft2(torch.view_as_complex(w) * scale, norm="ortho")
        loss = (((torch.abs(y) - amp_t) ** 2) * usable_t).sum(dim=(-2, -1))
        loss.sum().backward()
        opt.step()
        with torch.no_grad():
            u = torch.view_as_complex(w)
            u.mul_(support_t)
            u.mul_(torch.clamp(bound / torch.abs(u).clamp_min(1e-300), max=1.0))
        errors.append(np.sqrt(loss.detach().numpy() / energy))
    x = (torch.view_as_complex(w.detach()) * scale).numpy()
    return x, np.stack(errors, axis=1)


def adam_512(full):
    """Config 4's optimisation itself: adam_reconstruct (FP32 line passes,
    torch's fused Adam on the real view, the fused support-and-bound
    projection, graph replay) against the same algorithm in FP64, from the
    same starts."""
    rng = np.random.default_rng(4000)
    obj = workloads.square(512, seed=4000)
    intensity = workloads.poisson(workloads.simulate_intensity(obj), 1e7, rng)
    mask = workloads.beamstop((512, 512), 12)
    p = qpc.make_problem(intensity, mask=mask)
    starts, lr, bound = 2, 1e-2, 16.0
    out = {"workload": "square 512x512 (box 192), Poisson 1e7, beamstop 12: Adam(lr 1e-2), "
                       "support projection, bound 16, 2 starts, FP32 against FP64"}
    with qpc.Solver(p, starts=starts, seed=0) as drawn:
        first = drawn.results()
    x0 = np.stack([np.fft.ifftshift(r.object) for r in first]).astype(np.complex128)
    amp = np.fft.ifftshift(np.asarray(p.amplitude, np.float64))
    usable = np.fft.ifftshift(np.asarray(p.mask)) == 0
    support = np.fft.ifftshift(np.asarray(p.support)) != 0
    energy = float(np.sum(np.where(usable, amp ** 2, 0.0)))
    scale = float(np.sqrt(energy / max(int(support.sum()), 1))) or 1.0
    for steps in (20, 200) if full else (20, 100):
        ours = qad.adam_reconstruct(p, starts=starts, steps=steps, lr=lr, seed=0, bound=bound)
        x, errors = _adam_fp64(x0, scale, amp, usable, support, steps, lr, bound)
        err = max(float(np.max(np.abs(r.errors - e) / e)) for r, e in zip(ours, errors))
        obj_diff = max(fp64.relative_diff(r.object, np.fft.fftshift(xs))
                       for r, xs in zip(ours, x))
        out[f"steps_{steps}"] = {"error_rel_max": err, "object_rel_l2_max": obj_diff,
                                 "final_error_fp32": [float(r.errors[-1]) for r in ours],
                                 "final_error_fp64": [float(e[-1]) for e in errors]}
    return out


def crystal_128(full):
    obj, intensity = workloads.crystal(128, seed=3000)
    support = qpc.autocorrelation_support(intensity)
    return {"workload": "crystal 128^3, Poisson 1e7, 4 starts",
            "prefix": prefixes(intensity, support, None, "hio", 4, lengths=(2, 10))}


REPORTS = {"square": square_64, "gaussians": gaussians_256, "uneven": uneven,
           "adjoint": adjoint_512, "adam": adam_512, "crystal": crystal_128}


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--full", action="store_true", help="whole recipes for every workload")
    parser.add_argument("--only", choices=sorted(REPORTS), action="append")
    args = parser.parse_args(argv)
    for name in args.only or REPORTS:
        t0 = time.perf_counter()
        line = {"report": name, **REPORTS[name](args.full)}
        line["seconds"] = time.perf_counter() - t0
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
