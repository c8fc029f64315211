"""Parity on the benchmark workload, in the schedules the benchmark runs.

The benchmark reconstructs the seeded ``gaussians`` problem (256 x 256, five
Gaussian blobs with a smooth phase, Poisson counts at 1e6, beamstop of radius
8 px, autocorrelation support) with 32 starts. Its timed solver runs streamed
passes with 4 starts per launch as 8 parallel graph branches, the amplitude
pre-tiled in the modulus pass's CTA order; the autotuner's other candidates
are the resident cluster kernel and larger launches (all 32 starts in one
launch runs the modulus pass's 7-CTAs-per-SM variant). These schedules are
checked here from the
bit-identical random starts of the FP64 oracle (oracle/fp64.py, which restates
the reference's CpuSolver, src/cpu/cpu_solver.cpp:82-93):

* RAAR(0.9) x 2: per-iteration Fourier errors and final objects within 1e-5
  relative of FP64 (the single-operator bar);
* RAAR(0.9) x 20: the drift from FP64 is compared with the drift of two FP32
  CPU implementations on the same starts (the oracle's complex64 numpy port
  and the reference's own CpuSolver compiled from its sources), which
  measures how far FP32 rounding alone carries these iterations;
* the 128^3 crystal with 4 starts, HIO x 2, against FP64 at 1e-5;
* whole recipes with the objects' true supports, where they converge to the
  noise floor: RAAR x 300 + ER x 200 on the gaussians object and HIO x 200 +
  ER x 100 on the crystal generator at 64^3, best final error and aligned
  object error within 1e-4 of FP64 (or twice the FP32 port's distance).
"""

import numpy as np
import pytest

from oracle import fp64, ref

import qoraphasecu_b200 as qpc
from qoraphasecu_b200 import workloads
from qoraphasecu_b200.recipe import ER, HIO, RAAR, Recipe

pytestmark = pytest.mark.gpu

STARTS = 32
SCHEDULES = {
    "streamed 4 per launch": dict(schedule="streamed", batch=4, sync_every=50),
    # all 32 starts in one launch: 1024 CTAs of the modulus pass, more than one
    # wave at its default occupancy, so its 7-CTAs-per-SM variant runs
    "streamed 32 per launch": dict(schedule="streamed", batch=32, sync_every=50),
    "resident": dict(schedule="resident", sync_every=50),
}


@pytest.fixture(scope="module")
def gaussians():
    _, intensity, mask = workloads.gaussians(256, seed=1000)
    return intensity, mask


@pytest.fixture(scope="module")
def fp64_raar(gaussians):
    """RAAR(0.9) from the benchmark's starts, after 2 and after 20 iterations:
    the FP64 oracle, the oracle's FP32 port (complex64 numpy) and the
    reference's own CPU path compiled from its sources (oracle/_ref, FP32 with
    the project FFT shim), all on one autocorrelation support."""
    intensity, mask = gaussians
    support = ref.autocorrelation_support(intensity)
    problem = fp64.make_problem(intensity, support, mask)
    out = {"support": support}
    for dtype in (np.complex128, np.complex64):
        solver = fp64.Solver(problem, starts=STARTS, seed=0, dtype=dtype)
        solver.run([fp64.op("raar", 2, 0.9)])
        two = solver.results()
        solver.run([fp64.op("raar", 18, 0.9)])
        out[np.dtype(dtype).name] = (two, solver.results())
    out["reference_cpu"] = ref.reconstruct(ref.make_problem(intensity, support, mask),
                                           [("raar", 20, 0.9, 0.0, 0.0, "max", 0)],
                                           starts=STARTS, seed=0)
    return out


def _distance(runs, reference, stat=max):
    """`stat` over the starts of the largest relative difference of the error
    histories, and of the relative L2 difference of the objects."""
    err = stat([float(np.max(np.abs(_errors(r) - e) / e)) for r, (_, _, e) in zip(runs, reference)])
    obj = stat([fp64.relative_diff(_object(r), o) for r, (o, _, _) in zip(runs, reference)])
    return err, obj


def _errors(run):
    return run.errors if hasattr(run, "errors") else run[2]


def _object(run):
    return run.object if hasattr(run, "object") else run[0]


def _ours(gaussians, support, schedule, iterations):
    intensity, mask = gaussians
    problem = qpc.make_problem(intensity, support=support, mask=mask)
    with qpc.Solver(problem, starts=STARTS, seed=0, **SCHEDULES[schedule]) as s:
        s.run(Recipe(RAAR(iterations, 0.9)))
        return s.results()


@pytest.mark.parametrize("schedule", sorted(SCHEDULES))
def test_two_raar_iterations_match_fp64(gpu, gaussians, fp64_raar, schedule):
    ours = _ours(gaussians, fp64_raar["support"], schedule, 2)
    err, obj = _distance(ours, fp64_raar["complex128"][0])
    assert err < 1e-5, err
    assert obj < 1e-5, obj


@pytest.mark.parametrize("schedule", sorted(SCHEDULES))
def test_twenty_raar_iterations_drift_like_fp32(gpu, gaussians, fp64_raar, schedule):
    """After 20 iterations every FP32 implementation has left FP64 by an amount
    set by its own rounding and by how sensitive each start is: the median
    start moves by about 2e-6 (errors) and 1e-4 (objects), the most sensitive
    of the 32 by up to 1e-4 and 1e-2, and the two CPU implementations (the
    numpy port and the reference's compiled CpuSolver) differ from each other
    by as much. Ours is held to the larger of the two CPU drifts: at most
    twice it over the median start, three times it over the worst start."""
    ours = _ours(gaussians, fp64_raar["support"], schedule, 20)
    truth = fp64_raar["complex128"][1]
    cpu = [fp64_raar["complex64"][1], fp64_raar["reference_cpu"]]
    for stat, factor in ((np.median, 2.0), (max, 3.0)):
        bound_err = max(_distance(c, truth, stat)[0] for c in cpu)
        bound_obj = max(_distance(c, truth, stat)[1] for c in cpu)
        err, obj = _distance(ours, truth, stat)
        assert err <= factor * bound_err, (stat.__name__, err, bound_err)
        assert obj <= factor * bound_obj, (stat.__name__, obj, bound_obj)


def test_crystal_two_hio_iterations_match_fp64(gpu):
    _, intensity = workloads.crystal(128, seed=3000)
    truth = fp64.reconstruct(fp64.make_problem(intensity), [fp64.op("hio", 2, 0.9)], starts=4,
                             seed=0)
    problem = qpc.make_problem(intensity)
    with qpc.Solver(problem, starts=4, seed=0, sync_every=50) as s:
        s.run(Recipe(HIO(2, 0.9)))
        ours = s.results()
    err, obj = _distance(ours, truth)
    assert err < 1e-5, err
    assert obj < 1e-5, obj


def test_known_support_whole_recipe_against_fp64(gpu, gaussians):
    """A whole recipe on the benchmark's object with its true support (the
    pixels above 2% of the peak amplitude) and no shrinkwrap: RAAR(0.9) x 300
    then ER x 200, 4 starts. The Poisson noise keeps the problem from a unique
    solution, so FP32 itself moves the result: the oracle's FP32 port lands
    about 1e-5 from FP64 in the best final error and 5e-4 in the aligned
    object error. Ours is held to 1e-4 or twice the port's distance,
    whichever is larger, on both."""
    intensity, mask = gaussians
    obj, _, _ = workloads.gaussians(256, seed=1000)
    support = np.abs(obj) > 0.02 * np.abs(obj).max()
    ops = [fp64.op("raar", 300, 0.9), fp64.op("er", 200)]
    problem = fp64.make_problem(intensity, support, mask)
    truth = fp64.reconstruct(problem, ops, starts=4, seed=0)
    port = fp64.Solver(problem, starts=4, seed=0, dtype=np.complex64)
    port.run(ops)
    port = port.results()
    p = qpc.make_problem(intensity, support=support, mask=mask)
    with qpc.Solver(p, starts=4, seed=0, sync_every=50) as s:
        s.run(Recipe(RAAR(300, 0.9), ER(200)))
        ours = s.results()
    # the object scaled to the data's photon count
    model = np.abs(np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(obj), norm="ortho"))) ** 2
    scaled = obj * np.sqrt(np.sum(np.where(mask, 0, intensity)) / np.sum(np.where(mask, 0, model)))

    def best(runs):
        final = [float(_errors(r)[-1]) for r in runs]
        k = int(np.argmin(final))
        return final[k], fp64.aligned_error(_object(runs[k]), scaled)

    t_err, t_obj = best(truth)
    p_err, p_obj = best(port)
    o_err, o_obj = best(ours)
    assert abs(o_err - t_err) <= max(1e-4, 2 * abs(p_err - t_err)), (o_err, t_err, p_err)
    assert abs(o_obj - t_obj) <= max(1e-4, 2 * abs(p_obj - t_obj)), (o_obj, t_obj, p_obj)


def _crystal_best(runs, scaled):
    final = [float(_errors(r)[-1]) for r in runs]
    k = int(np.argmin(final))
    return final[k], fp64.aligned_error(_object(runs[k]), scaled)


def test_crystal_known_support_whole_recipe_against_fp64(gpu):
    """The crystal generator at 64^3 with its true support: HIO(0.9) x 200
    then ER x 100, 2 starts, Poisson noise at the generator's 1e7 peak. The
    recipe converges to the noise floor (final Fourier error 0.019, aligned
    object error 0.011 in FP64, the FP32 port within 1e-6 of both), so the
    best final error and aligned object error are held to 1e-4 of FP64 (or
    twice the port's distance, if larger)."""
    obj, intensity = workloads.crystal(64, seed=3000)
    support = np.abs(obj) > 0
    model = workloads.simulate_intensity(obj)
    scaled = obj * np.sqrt(np.sum(intensity) / np.sum(model))
    ops = [fp64.op("hio", 200, 0.9), fp64.op("er", 100)]
    problem = fp64.make_problem(intensity, support)
    truth = fp64.reconstruct(problem, ops, starts=2, seed=0)
    port = fp64.Solver(problem, starts=2, seed=0, dtype=np.complex64, fft="scipy")
    port.run(ops)
    port = port.results()
    p = qpc.make_problem(intensity, support=support)
    with qpc.Solver(p, starts=2, seed=0, sync_every=50) as s:
        s.run(Recipe(HIO(200, 0.9), ER(100)))
        ours = s.results()
    t_err, t_obj = _crystal_best(truth, scaled)
    p_err, p_obj = _crystal_best(port, scaled)
    o_err, o_obj = _crystal_best(ours, scaled)
    assert abs(o_err - t_err) <= max(1e-4, 2 * abs(p_err - t_err)), (o_err, t_err, p_err)
    assert abs(o_obj - t_obj) <= max(1e-4, 2 * abs(p_obj - t_obj)), (o_obj, t_obj, p_obj)
