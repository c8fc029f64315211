"""Many problems of uneven shapes in one batch (one graph per chunk, the
shapes as parallel branches) against the same problems run alone and against
the FP64 oracle."""

import numpy as np
import pytest

from oracle import fp64
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200 import workloads
from qoraphasecu_b200.recipe import ER, HIO, RAAR, Recipe, Shrinkwrap, repeat

pytestmark = pytest.mark.gpu

SHAPES = [((64, 64), 16), ((48, 40), 10), ((64, 64), 20), ((128, 128), 30), ((16, 16, 16), 6),
          ((48, 40), 12)]


def problems_of(shapes, masked=True):
    out = []
    for shape, m in shapes:
        _, support, intensity = triangle(shape, m)
        mask = None
        if masked:
            mask = np.zeros(shape, np.uint8)
            mask[tuple(n // 2 for n in shape)] = 1
        out.append((intensity, support, mask))
    return out


def test_batch_equals_problems_run_alone(gpu):
    """Same kernels, same per-problem starts: each problem's objects and
    supports are bit-identical to a solver of that problem alone."""
    data = problems_of(SHAPES)
    problems = [qpc.make_problem(i, support=s, mask=m) for i, s, m in data]
    recipe = Recipe(HIO(12), Shrinkwrap(method="rms"), RAAR(9), ER(7))
    with qpc.BatchSolver(problems, starts=2, seed=5, sync_every=5, schedule="streamed") as b:
        b.run(recipe)
        together = b.results()
    assert len(together) == len(problems)
    for p, runs in zip(problems, together, strict=True):
        with qpc.Solver(p, starts=2, seed=5, sync_every=5, schedule="streamed") as s:
            s.run(recipe)
            alone = s.results()
        for a, r in zip(alone, runs, strict=True):
            assert r.object.shape == p.shape
            np.testing.assert_array_equal(r.object, a.object)
            np.testing.assert_array_equal(r.support, a.support)
            np.testing.assert_allclose(r.errors, a.errors, rtol=1e-6)


def test_batch_reset_equals_a_new_batch(gpu):
    """BatchSolver.reset with new problems of the same shapes (several shape
    classes) gives what a new batch built on them gives, bit for bit."""
    first = [qpc.make_problem(i, support=s, mask=m) for i, s, m in problems_of(SHAPES)]
    second = [qpc.make_problem(i, support=s, mask=m)
              for i, s, m in problems_of([(shape, m + 2) for shape, m in SHAPES])]
    recipe = Recipe(HIO(8), Shrinkwrap(method="rms"), ER(6))
    with qpc.BatchSolver(first, starts=2, seed=5, sync_every=4, schedule="streamed") as b:
        b.run(recipe)
        b.reset(second, seed=9)
        b.run(recipe)
        reused = b.results()
    with qpc.BatchSolver(second, starts=2, seed=9, sync_every=4, schedule="streamed") as b:
        b.run(recipe)
        fresh = b.results()
    for runs_a, runs_b in zip(reused, fresh, strict=True):
        for a, r in zip(runs_a, runs_b, strict=True):
            assert len(a.errors) == recipe.iterations()
            np.testing.assert_array_equal(a.object, r.object)
            np.testing.assert_array_equal(a.support, r.support)
            np.testing.assert_allclose(a.errors, r.errors, rtol=1e-6)
    with qpc.BatchSolver(first, starts=2, seed=5) as b:
        with pytest.raises(ValueError):
            b.reset(second[:-1])
        with pytest.raises(ValueError):
            b.reset(second[::-1])


def test_reconstruct_batch_reuses_its_solver(gpu):
    qpc.api.clear_cache()
    data1 = problems_of(SHAPES[:4])
    data2 = problems_of([(shape, m + 2) for shape, m in SHAPES[:4]])
    recipe = Recipe(HIO(6), ER(4))

    def call(data):
        return qpc.reconstruct_batch([d[0] for d in data], supports=[d[1] for d in data],
                                     masks=[d[2] for d in data], recipe=recipe, starts=2, seed=3,
                                     sync_every=5)

    def batch_solvers():
        return [v for k, v in qpc.api._cached_solvers().items() if k[0] == "batch"]

    call(data1)
    kept = batch_solvers()
    assert len(kept) == 1
    second = call(data2)
    assert batch_solvers() == kept
    problems = [qpc.make_problem(i, support=s, mask=m) for i, s, m in data2]
    with qpc.BatchSolver(problems, starts=2, seed=3, sync_every=5) as b:
        b.run(recipe)
        fresh = b.results()
    for ens, runs in zip(second, fresh, strict=True):
        for x, y in zip(ens, runs, strict=True):
            np.testing.assert_array_equal(x.object, y.object)
            np.testing.assert_array_equal(x.support, y.support)
    qpc.api.clear_cache()
    assert batch_solvers() == []


def test_batch_matches_fp64(gpu):
    data = problems_of(SHAPES[:4])
    recipe = Recipe(HIO(10), Shrinkwrap(), ER(10))
    ours = qpc.reconstruct_batch([d[0] for d in data], supports=[d[1] for d in data],
                                 masks=[d[2] for d in data], recipe=recipe, starts=2, seed=3,
                                 sync_every=4)
    for (intensity, support, mask), ens in zip(data, ours, strict=True):
        ref = fp64.reconstruct(fp64.make_problem(intensity, support, mask), recipe.ops(),
                               starts=2, seed=3)
        for (r_obj, r_sup, r_err), run in zip(ref, ens, strict=True):
            np.testing.assert_allclose(run.errors, r_err, rtol=1e-4, atol=1e-7)
            assert fp64.relative_diff(run.object, r_obj) < 1e-4
            np.testing.assert_array_equal(run.support, r_sup)


def test_batch_progress_and_given_starts(gpu):
    data = problems_of(SHAPES[:3], masked=False)
    problems = [qpc.make_problem(i, support=s) for i, s, _ in data]
    init = [np.stack([random_field(int(np.prod(p.shape)), 10 * q + k).reshape(p.shape)
                      for k in range(2)]) for q, p in enumerate(problems)]
    seen = []
    with qpc.BatchSolver(problems, starts=2, init=init, sync_every=5,
                         progress=lambda it, e: seen.append((it, e))) as b:
        b.run(Recipe(HIO(10), ER(5)))
        runs = b.results()
    assert [it for it, _ in seen] == [5, 10, 15]
    for it, errors in seen:
        assert errors.shape == (6,)
        for q in range(3):
            for k in range(2):
                assert errors[2 * q + k] == runs[q][k].errors[it - 1]
    for q, (intensity, support, _) in enumerate(data):
        ref = fp64.reconstruct(fp64.make_problem(intensity, support), Recipe(HIO(10), ER(5)).ops(),
                               starts=2, start=init[q])
        for (r_obj, _, r_err), run in zip(ref, runs[q], strict=True):
            np.testing.assert_allclose(run.errors, r_err, rtol=1e-4, atol=1e-7)


def test_uneven_workload_er_never_increases(gpu):
    """The uneven-batch workload generator (sides 64..256 here, autotuned
    schedule per side), recipe repeat(2, HIO(50), Shrinkwrap(rms 0.3)), ER(50):
    once the final ER stage has put the iterate inside the support, no start of
    any problem raises its Fourier error (ER alternates two projections;
    tests/test_recover.cpp:53-62 allows the same 1e-4 of FP32 slack), and every
    error history is finite and has the recipe's length."""
    batch = workloads.uneven_batch(count=8, seed=2100, sizes=(64, 128, 256))
    recipe = Recipe(repeat(2, HIO(50), Shrinkwrap(0.3, 1.0, "rms")), ER(50))
    ens = qpc.reconstruct_batch([b[1] for b in batch], masks=[b[2] for b in batch], recipe=recipe,
                                starts=4, seed=1)
    assert len(ens) == len(batch)
    for (obj, _, _), e in zip(batch, ens, strict=True):
        assert len(e) == 4
        for run in e:
            assert run.object.shape == obj.shape
            assert run.errors.shape == (150,) and np.all(np.isfinite(run.errors))
            er = run.errors[101:]  # iterates from the second ER iteration on lie in S
            # 1e-6 absolute: a start that fits its noise reaches the FP32 floor
            assert np.all(er[1:] <= er[:-1] * (1 + 1e-4) + 1e-6)


def test_batch_rejects_bad_input(gpu):
    _, _, intensity = triangle((32, 32), 8)
    p = qpc.make_problem(intensity)
    with pytest.raises(ValueError):
        qpc.BatchSolver([], starts=2)
    with pytest.raises(ValueError, match="init"):
        qpc.BatchSolver([p, p], starts=1, init=[np.zeros((32, 32))])
    with qpc.BatchSolver([p, qpc.make_problem(np.pad(intensity, 8))], starts=1) as b:
        with pytest.raises(ValueError, match="one shape"):
            b.profile_passes(2)
    with qpc.BatchSolver([p, p], starts=2) as b:
        assert len(b.profile_passes(2)) == 2
