"""Whole reconstructions on the device against the FP64 oracle.

Short recipes run from identical starts (the random phases are bit-identical
by construction), so the per-iteration Fourier errors and the objects can be
compared directly. Long recipes are chaotic (docs/ARCHITECTURE.md:77-87 in the
reference), so they are compared through the final Fourier error and the
object error against the ground truth after alignment, both within 1e-4.
"""

import numpy as np
import pytest

from oracle import fp64
from synthetic import corner, random_field, readme_triangle, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200.recipe import ER, HIO, RAAR, Recipe, Shrinkwrap, default_recipe, detwin, repeat

pytestmark = pytest.mark.gpu


def run_both(intensity, support, recipe, *, mask=None, starts=1, seed=0, init=None, **kw):
    ref_p = fp64.make_problem(intensity, support, mask)
    ref = fp64.reconstruct(ref_p, recipe.ops(), starts=starts, seed=seed, start=init)
    p = qpc.make_problem(intensity, support=support, mask=mask)
    with qpc.Solver(p, starts=starts, seed=seed, init=init, **kw) as s:
        s.run(recipe)
        ours = s.results()
    return ref, ours


@pytest.mark.parametrize("variant", ["batched", "plain"])
def test_short_recipe_matches_fp64(gpu, variant):
    """tests/test_cuda.cpp:64-87: HIO, Shrinkwrap, RAAR, detwin(HIO), ER from the same seed."""
    obj, support, intensity = triangle((64, 48), 16)
    recipe = Recipe(HIO(15), Shrinkwrap(), RAAR(10), detwin(HIO(5)), ER(10))
    ref, ours = run_both(intensity, support, recipe, starts=2, seed=3, sync_every=4,
                         variant=variant)
    for (r_obj, r_sup, r_err), run in zip(ref, ours, strict=True):
        assert run.errors.shape == r_err.shape
        np.testing.assert_allclose(run.errors, r_err, rtol=1e-4, atol=1e-7)
        assert fp64.relative_diff(run.object, r_obj) < 1e-4
        np.testing.assert_array_equal(run.support, r_sup)


def test_single_iteration_is_fp32_exact(gpu):
    """One ER iteration from a random start: errors 1e-5 relative, object 1e-5."""
    obj, support, intensity = triangle((256, 256), 40)
    ref, ours = run_both(intensity, support, Recipe(ER(1)), starts=3, seed=11)
    for (r_obj, _, r_err), run in zip(ref, ours, strict=True):
        assert abs(run.errors[0] - r_err[0]) <= 1e-5 * r_err[0]
        assert fp64.relative_diff(run.object, r_obj) < 1e-5


@pytest.mark.parametrize("shape,m", [((21, 15), 6), ((17, 24), 8), ((16, 20, 12), 6),
                                     ((32, 32, 32), 10)])
def test_odd_and_3d_shapes_match_fp64(gpu, shape, m):
    """tests/test_cuda.cpp:89-102 plus 3D: the generic mixed-radix passes."""
    _, support, intensity = triangle(shape, m)
    recipe = Recipe(HIO(10), Shrinkwrap(), ER(10))
    ref, ours = run_both(intensity, support, recipe, starts=2, seed=0)
    for (r_obj, r_sup, r_err), run in zip(ref, ours, strict=True):
        np.testing.assert_allclose(run.errors, r_err, rtol=1e-4, atol=1e-7)
        assert fp64.relative_diff(run.object, r_obj) < 1e-4
        np.testing.assert_array_equal(run.support, r_sup)


@pytest.mark.parametrize("shape,m", [((512, 512), 40), ((256, 512), 30), ((512, 128), 24),
                                     ((128, 128, 128), 16)])
def test_tma_column_shapes_match_fp64(gpu, shape, m):
    """Columns of 128, 256 and 512 points on the TMA column tiles (512-point
    lines move as two boxes of 256 rows), with shrinkwrap between stages."""
    _, support, intensity = triangle(shape, m)
    recipe = Recipe(HIO(6), Shrinkwrap(), RAAR(4), ER(4))
    ref, ours = run_both(intensity, support, recipe, starts=2, seed=4)
    for (r_obj, r_sup, r_err), run in zip(ref, ours, strict=True):
        np.testing.assert_allclose(run.errors, r_err, rtol=1e-4, atol=1e-7)
        assert fp64.relative_diff(run.object, r_obj) < 1e-4
        np.testing.assert_array_equal(run.support, r_sup)


@pytest.mark.parametrize("variant", ["batched", "plain"])
def test_given_start_matches_fp64(gpu, variant):
    """tests/test_cuda.cpp:104-119."""
    _, support, intensity = triangle((40, 36), 10)
    init = np.stack([random_field(40 * 36, 11).reshape(40, 36),
                     random_field(40 * 36, 12).reshape(40, 36)])
    recipe = Recipe(HIO(5), RAAR(5), ER(5))
    ref, ours = run_both(intensity, support, recipe, starts=2, init=init, variant=variant)
    for (r_obj, _, r_err), run in zip(ref, ours, strict=True):
        assert fp64.relative_diff(run.object, r_obj) < 1e-5
        assert abs(run.error - r_err[-1]) <= 1e-5 * r_err[-1] + 1e-7


def test_given_start_replaces_the_random_one(gpu):
    """tests/test_recover.cpp:32-46: the solution is a fixed point of ER."""
    obj, support, intensity = triangle((32, 24), 8)
    p = qpc.make_problem(intensity, support=support)
    start = np.stack([obj, random_field(32 * 24, 3).reshape(32, 24)])
    with qpc.Solver(p, starts=2, seed=1, init=start) as s:
        s.run(Recipe(ER(5)))
        a = s.results()
    with qpc.Solver(p, starts=2, seed=2, init=start) as s:
        s.run(Recipe(ER(5)))
        b = s.results()
    assert a[0].error < 1e-5
    assert np.abs(a[0].object - obj).max() < 1e-5
    np.testing.assert_array_equal(a[1].object, b[1].object)
    with pytest.raises(ValueError, match="init.shape"):
        qpc.Solver(p, starts=3, init=start)


def test_batched_equals_plain_and_pairs(gpu):
    """tests/test_cuda.cpp:160-180: every schedule gives the same reconstruction."""
    _, _, intensity = triangle((64, 64), 20)
    p = qpc.make_problem(intensity)
    recipe = Recipe(RAAR(40), repeat(3, HIO(20), Shrinkwrap(method="rms")), ER(20))
    runs = {}
    for name, kw in {"plain": dict(variant="plain"), "batched": dict(variant="batched"),
                     "pairs": dict(variant="batched", batch=2)}.items():
        with qpc.Solver(p, starts=4, seed=9, **kw) as s:
            s.run(recipe)
            runs[name] = s.results()
    for k in range(4):
        for other in ("batched", "pairs"):
            np.testing.assert_array_equal(runs[other][k].object, runs["plain"][k].object)
            np.testing.assert_array_equal(runs[other][k].support, runs["plain"][k].support)
            np.testing.assert_allclose(runs[other][k].errors, runs["plain"][k].errors, rtol=1e-6)


def test_progress_matches_the_error_history(gpu):
    """tests/test_cuda.cpp:121-137."""
    _, support, intensity = triangle((32, 32), 8)
    p = qpc.make_problem(intensity, support=support)
    seen, reported = [], []

    def progress(it, errors):
        seen.append(it)
        reported.append(errors[2])

    with qpc.Solver(p, starts=3, sync_every=5, progress=progress) as s:
        s.run(Recipe(HIO(7), ER(8)))
        runs = s.results()
    assert seen == [5, 10, 15]
    for it, e in zip(seen, reported):
        assert e == runs[2].errors[it - 1]


def test_run_continues_from_the_current_state(gpu):
    """tests/test_recover.cpp:97-107: split runs equal the whole run."""
    _, support, intensity = triangle((32, 32), 8)
    p = qpc.make_problem(intensity, support=support)
    with qpc.Solver(p) as s:
        s.run(Recipe(HIO(10)))
        s.run(Recipe(ER(5)))
        split = s.results()[0]
    with qpc.Solver(p) as s:
        s.run(Recipe(HIO(10), ER(5)))
        whole = s.results()[0]
    np.testing.assert_array_equal(split.object, whole.object)
    np.testing.assert_allclose(split.errors, whole.errors, rtol=1e-6)


def test_er_never_increases_the_error(gpu):
    """tests/test_recover.cpp:53-62."""
    _, support, intensity = triangle((64, 64), 20)
    run = qpc.reconstruct(intensity, support=support, recipe=Recipe(ER(100)))
    assert run.errors.shape == (100,)
    assert run.errors[-1] < run.errors[0]
    assert np.all(run.errors[1:] <= run.errors[:-1] * (1 + 1e-4))


def test_hio_then_er_recovers_2d(gpu):
    """tests/test_recover.cpp:48-51."""
    obj, support, intensity = triangle((64, 64), 20)
    runs = qpc.reconstruct(intensity, support=support, recipe=Recipe(HIO(300), ER(100)),
                           starts=4, seed=7)
    assert min(fp64.aligned_error(r.object, obj) for r in runs) < 1e-2


def test_raar_recovers_3d(gpu):
    """tests/test_recover.cpp:64-67 and test_cuda.cpp:139-148."""
    obj, support, intensity = triangle((24, 24, 24), 8)
    runs = qpc.reconstruct(intensity, support=support, recipe=Recipe(RAAR(300), ER(100)),
                           starts=2, seed=7)
    assert min(fp64.aligned_error(r.object, obj) for r in runs) < 1e-2


def test_default_recipe_without_support_matches_fp64(gpu, readme):
    """The README figure (config 1): default recipe, 8 starts, autocorrelation
    support. Best run < 1e-3 Fourier error and < 1e-2 aligned error
    (test_recover.cpp:69-76), and the final Fourier error and the object error
    of the best run agree with the FP64 oracle within 1e-4."""
    obj, _, intensity = readme
    ens = qpc.reconstruct(intensity, starts=8)
    assert isinstance(ens, qpc.Ensemble) and len(ens) == 8
    best = ens.best
    assert best.error < 1e-3
    ours_obj_err = fp64.aligned_error(best.object, obj)
    assert ours_obj_err < 1e-2
    ref = fp64.reconstruct(fp64.make_problem(intensity), fp64.default_recipe(), starts=8)
    ref_best = min(ref, key=lambda r: r[2][-1])
    assert abs(best.error - float(ref_best[2][-1])) < 1e-4
    assert abs(ours_obj_err - fp64.aligned_error(ref_best[0], obj)) < 1e-4
    assert ens.ranking[0] == min(range(8), key=lambda i: ens[i].error)


def test_mixed_storage_floor_3d(gpu):
    """FP16 amplitude storage converges to a floor set by the amplitude rounding."""
    obj, support, intensity = corner(32, 12)
    runs = qpc.reconstruct(intensity, support=support, recipe=Recipe(HIO(200), ER(100)),
                           starts=2, amp_storage="f16")
    best = min(runs, key=lambda r: r.error)
    assert best.error < 3e-3
    assert fp64.aligned_error(best.object, obj) < 1e-2


def test_engine_errors_surface_as_value_errors(gpu, readme):
    """python/tests/test_api.py:41-46."""
    _, support, intensity = readme
    with pytest.raises(ValueError):
        qpc.reconstruct(intensity, support=support, recipe=Recipe(ER(0)))
    with pytest.raises(ValueError):
        qpc.reconstruct(intensity, support=support, starts=4, batch=3)
    with pytest.raises(ValueError, match=r"support\.shape"):
        qpc.reconstruct(intensity, support=np.ones((3, 3), bool))
    with pytest.raises(ValueError):
        qpc.reconstruct(intensity, support=support, recipe=Recipe(detwin(ER(1), axis=2)))


def test_single_start_returns_a_reconstruction(gpu, readme):
    """python/tests/test_api.py:6-15."""
    obj, support, intensity = readme
    result = qpc.reconstruct(intensity, support=support, recipe=Recipe(HIO(30), ER(20)))
    assert isinstance(result, qpc.Reconstruction)
    assert result.object.shape == obj.shape and result.object.dtype == np.complex64
    assert result.support.dtype == bool
    assert result.errors.shape == (50,)
    assert result.error == result.errors[-1]


def test_negative_intensity_warns(gpu, readme):
    _, support, intensity = readme
    with pytest.warns(UserWarning, match="negative"):
        qpc.reconstruct(intensity - 0.5 * intensity.max(), support=support, recipe=Recipe(ER(1)))


@pytest.mark.parametrize("schedule", ["streamed", "resident"])
def test_reset_equals_a_fresh_solver(gpu, schedule):
    """Solver.reset keeps buffers and graphs; the next problem's results are
    those of a solver built for it."""
    _, s1, i1 = triangle((64, 64), 20)
    _, s2, i2 = triangle((64, 64), 14)
    p1 = qpc.make_problem(i1, support=s1)
    p2 = qpc.make_problem(i2, support=s2)
    recipe = Recipe(HIO(12), Shrinkwrap(), ER(8))
    with qpc.Solver(p1, starts=4, seed=1, sync_every=5, schedule=schedule) as s:
        s.run(recipe)
        s.reset(p2, seed=7)
        s.run(recipe)
        reused = s.results()
        with pytest.raises(ValueError, match="shape"):
            s.reset(qpc.make_problem(np.pad(i2, 2)), seed=1)
    with qpc.Solver(p2, starts=4, seed=7, sync_every=5, schedule=schedule) as s:
        s.run(recipe)
        fresh = s.results()
    for a, b in zip(reused, fresh, strict=True):
        np.testing.assert_array_equal(a.object, b.object)
        np.testing.assert_array_equal(a.support, b.support)
        np.testing.assert_allclose(a.errors, b.errors, rtol=1e-6)


def test_reconstruct_reuses_its_solver(gpu):
    """Two reconstruct() calls of one shape: the second loads into the first's
    solver and gives what a fresh solver gives."""
    _, s1, i1 = triangle((48, 40), 12)
    _, s2, i2 = triangle((48, 40), 10)
    recipe = Recipe(RAAR(10), ER(5))
    qpc.api.clear_cache()
    a = qpc.reconstruct(i1, support=s1, recipe=recipe, starts=2, seed=3)
    b = qpc.reconstruct(i2, support=s2, recipe=recipe, starts=2, seed=3)
    with qpc.Solver(qpc.make_problem(i2, support=s2), starts=2, seed=3) as s:
        s.run(recipe)
        fresh = s.results()
    for x, y in zip(b, fresh, strict=True):
        np.testing.assert_array_equal(x.object, y.object)
    assert not np.array_equal(a[0].object, b[0].object)
    qpc.api.clear_cache()


@pytest.mark.parametrize("shape,m", [((6, 32, 32), 4), ((8, 64, 64), 6), ((4, 128, 128), 4)])
def test_3d_register_passes_match_fp64(gpu, shape, m):
    """3D iterations through the register-resident passes on every axis
    (slices of side 32, 64, 128; z extents 4..8)."""
    _, support, intensity = triangle(shape, m)
    recipe = Recipe(HIO(8), Shrinkwrap(), RAAR(6), ER(6))
    ref, ours = run_both(intensity, support, recipe, starts=2, seed=5, sync_every=4)
    for (r_obj, r_sup, r_err), run in zip(ref, ours, strict=True):
        np.testing.assert_allclose(run.errors, r_err, rtol=1e-4, atol=1e-7)
        assert fp64.relative_diff(run.object, r_obj) < 1e-4
        np.testing.assert_array_equal(run.support, r_sup)


def test_profile_passes_times_every_pass(gpu):
    """Each pass of an iteration is timed from a captured graph of launches:
    two values in 2D, four in 3D, one for the resident kernel; on a caller's
    stream too. The timing leaves the solver as it was: a run that profiles
    between two recipes ends where the same run without the profile ends."""
    import torch

    _, support, intensity = triangle((64, 64), 20)
    p2 = qpc.make_problem(intensity, support=support)
    _, support3, intensity3 = triangle((32, 32, 32), 10)
    p3 = qpc.make_problem(intensity3, support=support3)
    stream = torch.cuda.Stream()
    cases = [(p2, dict(schedule="streamed", batch=2), 2), (p3, dict(schedule="streamed", batch=2), 4),
             (p2, dict(schedule="resident"), 1), (p2, dict(schedule="persistent"), 1),
             (p2, dict(schedule="streamed", batch=4, stream=stream.cuda_stream), 2)]
    for problem, kw, count in cases:
        with qpc.Solver(problem, starts=4, seed=1, sync_every=5, **kw) as s:
            s.run(Recipe(HIO(3)))
            before = qpc.kernel_launches()
            ms = s.profile_passes(4)
            assert len(ms) == count
            assert all(np.isfinite(m) and 0.0 < m < 10.0 for m in ms), ms
            assert qpc.kernel_launches() > before
            s.run(Recipe(ER(2)))
            runs = s.results()
        with qpc.Solver(problem, starts=4, seed=1, sync_every=5, **kw) as s:
            s.run(Recipe(HIO(3)))
            s.run(Recipe(ER(2)))
            plain = s.results()
        for r, q in zip(runs, plain, strict=True):
            assert r.errors.shape == (5,)
            assert np.all(np.isfinite(r.errors)) and np.all(r.errors > 0)
            np.testing.assert_allclose(r.errors, q.errors, rtol=1e-6)
            np.testing.assert_array_equal(r.object, q.object)
