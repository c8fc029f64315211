"""Pins the oracles (CPU only).

* The FP64 restatement (oracle/fp64.py) against golden vectors produced by the
  reference's own compiled CPU path (tests/golden/*.npz, make_golden.py).
* The reference's known-answer and property tests, run on the FP64 oracle:
  test_operators.cpp, test_problem.cpp, test_recipe.cpp, test_recover.cpp.
* When oracle/_ref is built: its FFT shim against numpy.fft.
"""

from pathlib import Path

import numpy as np
import pytest

from oracle import fp64, ref
from synthetic import random_field, readme_triangle, triangle

GOLDEN = Path(__file__).resolve().parent / "golden"
SHAPES = [(32, 32), (17, 24), (16, 16, 16)]


def golden(name):
    return np.load(GOLDEN / f"{name}.npz")


# ------------------------------------------------------------ golden vectors
def test_fp64_modulus_projection_matches_the_reference():
    g = golden("operators")
    p = fp64.make_problem(g["mp_intensity"], g["mp_support"], g["mp_mask"])
    out, err = fp64.modulus_project(p, g["mp_x"])
    assert fp64.relative_diff(out, g["mp_out"]) < 1e-5
    assert abs(err - float(g["mp_err"])) <= 1e-5 * float(g["mp_err"])


def test_fp64_blur_matches_the_reference():
    g = golden("operators")
    out = fp64.gaussian_blur(g["blur_image"], float(g["blur_sigma"]))
    assert np.abs(out - g["blur_out"]).max() < 1e-5


def test_fp64_half_support_matches_the_reference_exactly():
    g = golden("operators")
    np.testing.assert_array_equal(fp64.half_support(g["half_support"], 0), g["half_axis0"])
    np.testing.assert_array_equal(fp64.half_support(g["half_support"], 1), g["half_axis1"])


def test_fp64_autocorrelation_support_matches_the_reference():
    g = golden("operators")
    ours = fp64.autocorrelation_support(g["ac_intensity"], 0.1)
    assert np.count_nonzero(ours != g["ac_support"]) <= 2


def test_fp64_short_recipe_matches_the_reference():
    g = golden("short_recipe")
    ops = [fp64.op("hio", 15, 0.9), fp64.op("shrinkwrap", threshold=0.3, sigma=1.0),
           fp64.op("raar", 10, 0.9), fp64.op("detwin_begin"), fp64.op("hio", 5, 0.9),
           fp64.op("detwin_end"), fp64.op("er", 10)]
    runs = fp64.reconstruct(fp64.make_problem(g["intensity"], g["support"]), ops, starts=2,
                            seed=3)
    for k, (obj, sup, err) in enumerate(runs):
        np.testing.assert_allclose(err, g["errors"][k], rtol=1e-4, atol=1e-7)
        assert fp64.relative_diff(obj, g["objects"][k]) < 1e-4
        np.testing.assert_array_equal(sup, g["supports"][k].astype(bool))


def test_fp64_default_recipe_matches_the_reference():
    """Whole recipe: final Fourier error and aligned object error of the best run
    within 1e-4 of the reference's."""
    g = golden("default_recipe")
    runs = fp64.reconstruct(fp64.make_problem(g["intensity"]), fp64.default_recipe(), starts=8)
    errors = np.array([r[2][-1] for r in runs])
    best = int(np.argmin(errors))
    assert abs(errors[best] - g["final_errors"].min()) < 1e-4
    assert abs(fp64.aligned_error(runs[best][0], g["truth"]) - float(g["best_aligned"])) < 1e-4


# ---------------------------------------------- the reference's property tests
@pytest.mark.parametrize("shape", SHAPES)
def test_modulus_projection_is_idempotent(shape):
    """test_operators.cpp:20-29."""
    _, support, intensity = triangle(shape, 8)
    p = fp64.make_problem(intensity, support)
    x = random_field(int(np.prod(shape)), 1).reshape(shape)
    once, _ = fp64.modulus_project(p, x)
    twice, err = fp64.modulus_project(p, once)
    assert err < 1e-5
    assert np.abs(twice - once).max() < 1e-5


@pytest.mark.parametrize("shape", SHAPES)
def test_masked_pixels_keep_their_computed_magnitude(shape):
    """test_operators.cpp:31-44."""
    _, support, intensity = triangle(shape, 8)
    mask = np.zeros(shape, np.uint8)
    mask.flat[0] = 1
    mask.flat[mask.size // 2] = 1
    x = random_field(int(np.prod(shape)), 2).reshape(shape)
    a, _ = fp64.modulus_project(fp64.make_problem(intensity, support, mask), x)
    b, _ = fp64.modulus_project(fp64.make_problem(intensity, support), x)
    assert np.abs(a - b).max() > 1e-4
    assert fp64.modulus_project(fp64.make_problem(intensity, support, mask), a)[1] < 1e-5


@pytest.mark.parametrize("shape", SHAPES)
def test_error_is_zero_at_the_true_object(shape):
    """test_operators.cpp:46-52."""
    obj, support, intensity = triangle(shape, 8)
    out, err = fp64.modulus_project(fp64.make_problem(intensity, support), obj)
    assert err < 1e-5
    assert np.abs(out - obj).max() < 1e-4


@pytest.mark.parametrize("shape", SHAPES)
def test_blur_preserves_the_sum(shape):
    """test_operators.cpp:68-75."""
    image = np.zeros(shape, np.float32)
    image.flat[image.size // 2 + 3] = 1.0
    blurred = fp64.gaussian_blur(image, 1.5)
    assert abs(blurred.sum() - 1.0) < 1e-5
    assert blurred.max() < 0.5


def test_layout_round_trips_and_moves_the_centre():
    """test_problem.cpp:13-27."""
    v = np.arange(5 * 4 * 7).reshape(5, 4, 7)
    there = fp64.to_fft_order(v)
    assert not np.array_equal(there, v)
    np.testing.assert_array_equal(fp64.to_centered(there), v)
    w = np.zeros((6, 5), int)
    w[3, 2] = 1
    assert fp64.to_fft_order(w)[0, 0] == 1


def test_make_problem_clips_and_rejects():
    """test_problem.cpp:29-46."""
    p = fp64.make_problem(np.array([[4.0, -1.0], [9.0, 0.0]], np.float32),
                          np.array([[1, 1], [0, 0]], np.uint8))
    np.testing.assert_array_equal(p.amplitude, [[2, 0], [3, 0]])
    four = np.ones((2, 2), np.float32)
    with pytest.raises(ValueError):
        fp64.make_problem(np.ones(4, np.float32))
    with pytest.raises(ValueError):
        fp64.make_problem(four, mask=np.ones((2, 2), np.uint8))
    bad = four.copy()
    bad[0, 1] = np.nan
    with pytest.raises(ValueError):
        fp64.make_problem(bad)


def test_autocorrelation_support_covers_the_object():
    """test_problem.cpp:48-60."""
    _, support, intensity = triangle((64, 64), 16)
    derived = fp64.autocorrelation_support(intensity, 0.1)
    inside = int(support.sum())
    assert int((support & derived).sum()) > inside // 2
    assert int(derived.sum()) > inside


def test_half_support_keeps_the_lower_half():
    """test_problem.cpp:62-77."""
    support = np.zeros((8, 4), np.uint8)
    support[2:6, :] = 1
    half = fp64.half_support(support, 0)
    expect = np.zeros((8, 4), np.uint8)
    expect[2:4, :] = 1
    np.testing.assert_array_equal(half, expect)
    columns = fp64.half_support(support, 1)
    assert columns[2, 1] == 1 and columns[2, 2] == 0


def test_recipe_expansion_count_and_validation():
    """test_recipe.cpp:8-31 on the op-list form."""
    assert fp64.iterations(fp64.default_recipe()) == 50 + 20 + 50 + 8 * 50 + 200
    fp64.validate(fp64.default_recipe())
    for bad in ([], [fp64.op("er", 0)], [fp64.op("detwin_begin"), fp64.op("er", 1)],
                [fp64.op("detwin_end")],
                [fp64.op("detwin_begin"), fp64.op("detwin_begin"), fp64.op("er", 1),
                 fp64.op("detwin_end"), fp64.op("detwin_end")],
                [fp64.op("shrinkwrap", threshold=0.0, sigma=1.0)]):
        with pytest.raises(ValueError):
            fp64.validate(bad)


def test_aligned_error_ignores_shift_phase_and_twin():
    """test_recover.cpp:18-30."""
    obj, _, _ = triangle((32, 32), 10)
    moved = np.empty_like(obj)
    rotation = np.complex64(np.exp(0.7j))
    for y in range(32):
        for x in range(32):
            moved[y, x] = rotation * np.conj(obj[(32 - y) % 32, (32 - x + 3) % 32])
    assert fp64.aligned_error(moved, obj) < 1e-5
    assert fp64.aligned_error(random_field(32 * 32, 4).reshape(32, 32), obj) > 0.5


def test_given_start_replaces_the_random_one():
    """test_recover.cpp:32-46."""
    obj, support, intensity = triangle((32, 24), 8)
    p = fp64.make_problem(intensity, support)
    start = np.stack([obj, random_field(32 * 24, 3).reshape(32, 24)])
    a = fp64.reconstruct(p, [fp64.op("er", 5)], starts=2, seed=1, start=start)
    b = fp64.reconstruct(p, [fp64.op("er", 5)], starts=2, seed=2, start=start)
    assert a[0][2][-1] < 1e-5
    assert np.abs(a[0][0] - obj).max() < 1e-5
    np.testing.assert_array_equal(a[1][0], b[1][0])


def test_er_never_increases_the_error():
    """test_recover.cpp:53-62."""
    _, support, intensity = triangle((64, 64), 20)
    err = fp64.reconstruct(fp64.make_problem(intensity, support), [fp64.op("er", 100)])[0][2]
    assert err[-1] < err[0]
    assert np.all(err[1:] <= err[:-1] * (1 + 1e-4))


def test_default_recipe_without_support_recovers():
    """test_recover.cpp:69-76 and python/tests/test_api.py:17-24."""
    obj, _, intensity = readme_triangle()
    runs = fp64.reconstruct(fp64.make_problem(intensity), fp64.default_recipe(), starts=8)
    best = min(runs, key=lambda r: r[2][-1])
    assert best[2][-1] < 1e-3
    assert fp64.aligned_error(best[0], obj) < 1e-2


def test_progress_fires_every_sync_interval():
    """test_recover.cpp:78-89."""
    _, support, intensity = triangle((32, 32), 8)
    seen = []
    s = fp64.Solver(fp64.make_problem(intensity, support), starts=2, sync_every=4,
                    progress=lambda it, e: seen.append((it, len(e))))
    s.run([fp64.op("hio", 6, 0.9), fp64.op("er", 6)])
    assert seen == [(4, 2), (8, 2), (12, 2)]


def test_run_continues_from_the_current_state():
    """test_recover.cpp:97-107: bit-identical."""
    _, support, intensity = triangle((32, 32), 8)
    p = fp64.make_problem(intensity, support)
    s = fp64.Solver(p)
    s.run([fp64.op("hio", 10, 0.9)])
    s.run([fp64.op("er", 5)])
    whole = fp64.reconstruct(p, [fp64.op("hio", 10, 0.9), fp64.op("er", 5)])[0]
    split = s.results()[0]
    np.testing.assert_array_equal(split[0], whole[0])
    np.testing.assert_array_equal(split[2], whole[2])


def test_uniform_is_the_reference_counter_rng():
    """pointwise.hpp:19-32: spot values of splitmix64 and the 24-bit uniform."""
    assert int(fp64.mix64(np.uint64(0))) == 0xE220A8397B1DCDAF
    u = fp64.uniform(0, 0, np.arange(4, dtype=np.uint64))
    assert u.dtype == np.float32 and np.all((u >= 0) & (u < 1))
    # every value is a multiple of 2^-24
    assert np.all((u * 2**24) == np.floor(u * 2**24))


# ------------------------------------------------------------- the FFT shim
@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("shape", [(32, 32), (17, 24), (16, 16, 16), (96, 250), (21, 15)])
def test_fft_shim_matches_numpy(shape):
    rng = np.random.default_rng(0)
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    for forward, numpy_fn in ((True, np.fft.fftn), (False, np.fft.ifftn)):
        got = ref.fft(a, forward)
        want = numpy_fn(a.astype(np.complex128), norm="ortho")
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-6
