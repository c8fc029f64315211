"""fp16 storage of the iterate and the wave: the half and mixed variants.

The reference's Variant::half keeps x and the wave as fp16 pairs and
Variant::mixed keeps the wave in fp16 for HIO and RAAR while x and ER stay in
FP32 (src/cuda/half.cu:14-83, cuda_solver.cu:74-86); both divide the
amplitude by its peak and need power-of-two extents. These tests follow its
tests/test_cuda.cpp:182-257: the extents are checked, a given start is taken
in the data's scale, half stalls at its fp16 floor (about 1e-3), mixed
converges past it in 2D and 3D, and ER under mixed is the FP32 path. The FP32
arithmetic of every pass is the same as in the complex64 variants, so after
one iteration the fp16 variants sit within fp16 rounding of the FP64 oracle.
"""

import numpy as np
import pytest

from oracle import fp64
from synthetic import corner, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200.recipe import ER, HIO, RAAR, Recipe, Shrinkwrap

pytestmark = pytest.mark.gpu


def test_half_and_mixed_reject_other_extents(gpu):
    """test_cuda.cpp:182-190."""
    _, support, intensity = triangle((48, 64), 12)
    p = qpc.make_problem(intensity, support=support)
    for variant in ("half", "mixed"):
        with pytest.raises(ValueError, match="power-of-two"):
            qpc.Solver(p, variant=variant)
    _, support, intensity = triangle((64, 64), 12)
    p = qpc.make_problem(intensity, support=support)
    with pytest.raises(ValueError):
        qpc.Solver(p, variant="half", amp_storage="f16")
    with pytest.raises(ValueError):
        qpc.Solver(p, variant="mixed", schedule="resident")


@pytest.mark.parametrize("variant", ["half", "mixed"])
def test_given_start_is_in_the_data_scale(gpu, variant):
    """test_cuda.cpp:192-205: the truth as the start stays (nearly) a fixed point."""
    obj, support, intensity = triangle((64, 64), 24)
    run = qpc.reconstruct(intensity, support=support, recipe=Recipe(ER(3)), init=obj,
                          variant=variant)
    assert run.error < 3e-3
    assert fp64.relative_diff(run.object, obj) < 5e-3


def test_half_recovers_to_its_precision_floor(gpu):
    """test_cuda.cpp:207-217."""
    obj, support, intensity = triangle((64, 64), 24)
    runs = qpc.reconstruct(intensity, support=support, recipe=Recipe(HIO(400), ER(100)),
                           starts=4, variant="half")
    best = runs.best
    assert best.error < 3e-3
    assert fp64.aligned_error(best.object, obj) < 5e-3


def test_mixed_converges_past_the_half_floor(gpu):
    """test_cuda.cpp:219-229."""
    obj, support, intensity = triangle((64, 64), 24)
    runs = qpc.reconstruct(intensity, support=support, recipe=Recipe(HIO(400), ER(100)),
                           starts=4, variant="mixed")
    best = runs.best
    assert best.error < 1e-5
    assert fp64.aligned_error(best.object, obj) < 1e-4


def test_mixed_converges_past_the_half_floor_3d(gpu):
    """test_cuda.cpp:231-241."""
    obj, support, intensity = corner(64, 24)
    runs = qpc.reconstruct(intensity, support=support, recipe=Recipe(HIO(400), ER(100)),
                           starts=4, variant="mixed")
    best = runs.best
    assert best.error < 1e-5
    assert fp64.aligned_error(best.object, obj) < 1e-5


def test_er_under_mixed_is_the_fp32_path(gpu):
    """test_cuda.cpp:243-257: ER runs in FP32 and differs from the complex64
    variant only by the amplitude scaling."""
    _, support, intensity = triangle((64, 32), 12)
    p = qpc.make_problem(intensity, support=support)
    recipe = Recipe(ER(30), Shrinkwrap(), ER(10))
    out = {}
    for variant in ("batched", "mixed"):
        with qpc.Solver(p, starts=2, seed=4, variant=variant) as s:
            s.run(recipe)
            out[variant] = s.results()
    for a, b in zip(out["batched"], out["mixed"], strict=True):
        assert fp64.relative_diff(b.object, a.object) < 1e-4
        assert abs(b.error - a.error) <= 1e-4 * a.error


@pytest.mark.parametrize("variant", ["half", "mixed"])
@pytest.mark.parametrize("shape,m", [((64, 64), 20), ((256, 256), 40), ((512, 512), 60),
                                     ((32, 64, 64), 10), ((128, 128, 128), 16)])
def test_one_iteration_is_within_fp16_rounding_of_fp64(gpu, variant, shape, m):
    """The first RAAR iteration from the oracle's random starts: the error
    within 1e-3 relative, the object within 5e-3 (fp16 keeps about three
    significant digits)."""
    _, support, intensity = triangle(shape, m)
    ref = fp64.reconstruct(fp64.make_problem(intensity, support), [fp64.op("raar", 1, 0.9)],
                           starts=2, seed=5)
    p = qpc.make_problem(intensity, support=support)
    with qpc.Solver(p, starts=2, seed=5, variant=variant) as s:
        s.run(Recipe(RAAR(1, 0.9)))
        ours = s.results()
    for (r_obj, _, r_err), run in zip(ref, ours, strict=True):
        assert abs(run.errors[0] - r_err[0]) <= 1e-3 * r_err[0]
        assert fp64.relative_diff(run.object, r_obj) < 5e-3


@pytest.mark.parametrize("variant", ["half", "mixed"])
def test_fp16_variants_batch_like_the_plain_start_loop(gpu, variant):
    """Start groups as graph branches give the same iterates as all starts in
    one launch."""
    _, support, intensity = triangle((64, 64), 20)
    p = qpc.make_problem(intensity, support=support)
    recipe = Recipe(HIO(10), Shrinkwrap(), RAAR(10), ER(5))
    runs = []
    for batch in (4, 2):
        with qpc.Solver(p, starts=4, seed=2, batch=batch, variant=variant, sync_every=5) as s:
            s.run(recipe)
            runs.append(s.results())
    for a, b in zip(*runs, strict=True):
        np.testing.assert_array_equal(a.object, b.object)
        np.testing.assert_allclose(a.errors, b.errors, rtol=1e-6)
