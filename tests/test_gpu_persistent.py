"""The persistent schedule: a chunk of iterations of every start as one launch.

The launch walks a work list of tiles (modulus tiles of 8 columns, update
tiles of whole rows), each tile waiting, with a bounded poll, only for the
tiles of its own start that it reads. The tiles run the same arithmetic as
the streamed passes, so the iterates are the streamed schedule's bit for bit
(the Fourier errors up to the order of their FP64 atomic sums), on square and
rectangular problems, with shrinkwrap and detwin between chunks, for single
problems and for several problems of one shape in one solver. The bounded
waits are exercised by starving the staged copies (QPB_TIMEOUT, the solver
recovers after a reset)."""

import numpy as np
import pytest

from oracle import fp64
from synthetic import triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200 import workloads
from qoraphasecu_b200.recipe import ER, HIO, RAAR, Recipe, Shrinkwrap, detwin

pytestmark = pytest.mark.gpu


def _runs(problem, recipe, schedule, **kw):
    with qpc.Solver(problem, schedule=schedule, **kw) as s:
        s.run(recipe)
        return s.results()


@pytest.mark.parametrize("shape,m", [((64, 64), 20), ((128, 256), 30), ((256, 64), 20),
                                     ((256, 256), 40)])
def test_persistent_equals_streamed(gpu, shape, m):
    _, support, intensity = triangle(shape, m)
    p = qpc.make_problem(intensity, support=support)
    recipe = Recipe(HIO(12), Shrinkwrap(), RAAR(9), detwin(HIO(4)), ER(7))
    kw = dict(starts=6, seed=3, sync_every=5)
    streamed = _runs(p, recipe, "streamed", batch=6, **kw)
    persistent = _runs(p, recipe, "persistent", **kw)
    for a, b in zip(streamed, persistent, strict=True):
        np.testing.assert_array_equal(b.object, a.object)
        np.testing.assert_array_equal(b.support, a.support)
        np.testing.assert_allclose(b.errors, a.errors, rtol=1e-6)


def test_persistent_matches_fp64_on_the_benchmark_problem(gpu):
    """Two RAAR iterations of 32 starts on the gaussians problem against the
    FP64 oracle at the single-operator bar."""
    _, intensity, mask = workloads.gaussians(256, seed=1000)
    support = qpc.autocorrelation_support(intensity)
    p = qpc.make_problem(intensity, support=support, mask=mask)
    ours = _runs(p, Recipe(RAAR(2, 0.9)), "persistent", starts=32, seed=0, sync_every=50)
    truth = fp64.reconstruct(fp64.make_problem(intensity, support, mask),
                             [fp64.op("raar", 2, 0.9)], starts=32, seed=0)
    for run, (obj, _, err) in zip(ours, truth, strict=True):
        assert float(np.max(np.abs(run.errors - err) / err)) < 1e-5
        assert fp64.relative_diff(run.object, obj) < 1e-5


def test_persistent_batches_several_problems(gpu):
    """Problems of one shape share the launch; each problem's starts give what
    the problem gives alone."""
    problems = []
    for m in (14, 18, 22):
        _, support, intensity = triangle((64, 128), m)
        problems.append(qpc.make_problem(intensity, support=support))
    recipe = Recipe(RAAR(10), Shrinkwrap(), ER(5))
    with qpc.BatchSolver(problems, starts=2, seed=1, sync_every=5,
                         schedule="persistent") as b:
        b.run(recipe)
        together = b.results()
    for q, p in enumerate(problems):
        alone = _runs(p, recipe, "streamed", starts=2, seed=1, sync_every=5, batch=2)
        for a, t in zip(alone, together[q], strict=True):
            np.testing.assert_array_equal(t.object, a.object)
            np.testing.assert_allclose(t.errors, a.errors, rtol=1e-6)


def test_persistent_rejects_other_shapes(gpu):
    _, support, intensity = triangle((48, 64), 12)
    with pytest.raises(ValueError, match="persistent"):
        qpc.Solver(qpc.make_problem(intensity, support=support), schedule="persistent")
    _, support, intensity = triangle((16, 32, 32), 6)
    with pytest.raises(ValueError, match="persistent"):
        qpc.Solver(qpc.make_problem(intensity, support=support), schedule="persistent")


def test_persistent_waits_time_out_and_recover(gpu):
    _, support, intensity = triangle((64, 64), 20)
    p = qpc.make_problem(intensity, support=support)
    recipe = Recipe(HIO(6), ER(4))
    with qpc.Solver(p, starts=4, seed=3, sync_every=5, schedule="persistent") as s:
        s.set_wait_limit(64, starve=True)
        with pytest.raises(TimeoutError):
            s.run(recipe)
        s.set_wait_limit(1 << 22, starve=False)
        s.reset(p, seed=3)
        s.run(recipe)
        recovered = s.results()
    fresh = _runs(p, recipe, "persistent", starts=4, seed=3, sync_every=5)
    for a, b in zip(recovered, fresh, strict=True):
        np.testing.assert_array_equal(a.object, b.object)
