"""The resident schedule (each start held in a thread-block cluster's shared
memory for a chunk of iterations) against the FP64 oracle and against the
streamed line passes, on every side length it has (64, 128, 256)."""

import numpy as np
import pytest

from oracle import fp64
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200.recipe import ER, HIO, RAAR, Recipe, Shrinkwrap, detwin, repeat

pytestmark = pytest.mark.gpu


def run(problem, recipe, **kw):
    with qpc.Solver(problem, **kw) as s:
        s.run(recipe)
        return s.results()


@pytest.mark.parametrize("side,m,masked", [(64, 16, False), (128, 30, True), (256, 40, True)])
def test_short_recipe_matches_fp64(gpu, side, m, masked):
    """HIO, Shrinkwrap, RAAR, detwin(HIO), ER from the same seed, chunks of 4
    iterations (sync_every) so that every op boundary falls inside a chunk.
    (The 16-pixel triangle at 64 x 64 with a beamstop makes this HIO run
    chaotic enough that FP32 rounding alone, in either schedule, moves the
    error history by 1e-3 within 30 iterations; it runs unmasked.)"""
    _, support, intensity = triangle((side, side), m)
    mask = np.zeros((side, side), np.uint8)
    if masked:
        mask[side // 2 - 2: side // 2 + 3, side // 2 - 2: side // 2 + 3] = 1
    recipe = Recipe(HIO(15), Shrinkwrap(), RAAR(10), detwin(HIO(5)), ER(10))
    ref = fp64.reconstruct(fp64.make_problem(intensity, support, mask), recipe.ops(), starts=2,
                           seed=3)
    p = qpc.make_problem(intensity, support=support, mask=mask)
    ours = run(p, recipe, starts=2, seed=3, sync_every=4, schedule="resident")
    for (r_obj, r_sup, r_err), res in zip(ref, ours, strict=True):
        assert res.errors.shape == r_err.shape
        np.testing.assert_allclose(res.errors, r_err, rtol=1e-4, atol=1e-7)
        assert fp64.relative_diff(res.object, r_obj) < 1e-4
        np.testing.assert_array_equal(res.support, r_sup)


def test_single_iteration_is_fp32_exact(gpu):
    obj, support, intensity = triangle((256, 256), 40)
    ref = fp64.reconstruct(fp64.make_problem(intensity, support), Recipe(ER(1)).ops(), starts=3,
                           seed=11)
    p = qpc.make_problem(intensity, support=support)
    ours = run(p, Recipe(ER(1)), starts=3, seed=11, schedule="resident")
    for (r_obj, _, r_err), res in zip(ref, ours, strict=True):
        assert abs(res.errors[0] - r_err[0]) <= 1e-5 * r_err[0]
        assert fp64.relative_diff(res.object, r_obj) < 1e-5


@pytest.mark.parametrize("side", [64, 128, 256])
def test_resident_equals_streamed(gpu, side):
    """Same transforms, projection and update in the same order: the two
    schedules agree to FP32 rounding over a 60-iteration recipe."""
    _, _, intensity = triangle((side, side), side // 4)
    p = qpc.make_problem(intensity)
    recipe = Recipe(RAAR(20), repeat(2, HIO(10), Shrinkwrap(method="rms")), ER(20))
    a = run(p, recipe, starts=4, seed=9, sync_every=10, schedule="resident")
    b = run(p, recipe, starts=4, seed=9, sync_every=10, schedule="streamed")
    for ra, rb in zip(a, b, strict=True):
        assert fp64.relative_diff(ra.object, rb.object) < 1e-5
        np.testing.assert_allclose(ra.errors, rb.errors, rtol=1e-5)


def test_given_start_and_continued_runs(gpu):
    """A given start, odd chunk lengths (sync_every 7) and a second run() that
    continues from the first: the error history is that of one long run."""
    _, support, intensity = triangle((128, 128), 30)
    p = qpc.make_problem(intensity, support=support)
    init = np.stack([random_field(128 * 128, s).reshape(128, 128) for s in (1, 2)])
    with qpc.Solver(p, starts=2, init=init, sync_every=7, schedule="resident") as s:
        s.run(Recipe(HIO(11)))
        s.run(Recipe(ER(9)))
        split = s.results()
    ref = fp64.reconstruct(fp64.make_problem(intensity, support), Recipe(HIO(11), ER(9)).ops(),
                           starts=2, start=init)
    for (r_obj, _, r_err), res in zip(ref, split, strict=True):
        assert res.errors.shape == (20,)
        np.testing.assert_allclose(res.errors, r_err, rtol=1e-4, atol=1e-7)
        assert fp64.relative_diff(res.object, r_obj) < 1e-4


@pytest.mark.parametrize("storage,floor", [("f16", 3e-3), ("bf16", 2e-2)])
def test_reduced_amplitude_storage(gpu, storage, floor):
    obj, support, intensity = triangle((128, 128), 30)
    runs = qpc.reconstruct(intensity, support=support, recipe=Recipe(HIO(200), ER(100)),
                           starts=2, amp_storage=storage, schedule="resident")
    assert min(r.error for r in runs) < floor


def test_resident_needs_a_supported_shape(gpu):
    for shape in ((64, 32), (96, 96), (16, 16, 16)):
        _, _, intensity = triangle(shape, 6)
        p = qpc.make_problem(intensity)
        with pytest.raises(ValueError, match="resident"):
            qpc.Solver(p, starts=2, schedule="resident")
    _, _, intensity = triangle((64, 64), 8)
    with pytest.raises(ValueError, match="resident"):
        qpc.Solver(qpc.make_problem(intensity), starts=2, variant="plain", schedule="resident")


def test_tuning_report_lists_the_resident_candidate(gpu):
    _, _, intensity = triangle((128, 128), 30)
    p = qpc.make_problem(intensity)
    with qpc.Solver(p, starts=4, seed=1) as s:
        s.run(Recipe(ER(2)))
    report = qpc.api.tuning_report()
    lines = [l for l in report.splitlines() if "1x128x128 starts 4 " in l]
    assert any("resident (" in l and "clusters of 2 CTAs" in l for l in lines)
