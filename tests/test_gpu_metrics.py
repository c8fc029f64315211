"""Device scoring and set-up against the FP64 oracle: aligned_error
(src/core/metrics.cpp:17-86) and simulate_intensity (src/core/problem.cpp:90-99)."""

import numpy as np
import pytest

from oracle import fp64
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc

pytestmark = pytest.mark.gpu

SHAPES = [(64, 48), (256, 256), (21, 15), (16, 20, 12)]


@pytest.mark.parametrize("shape", SHAPES)
def test_simulate_intensity_matches_fp64(gpu, shape):
    obj, _, _ = triangle(shape, 6)
    obj = obj + 0.1 * random_field(int(np.prod(shape)), 3).reshape(shape)
    ours = qpc.simulate_intensity(obj)
    ref = fp64.simulate_intensity(obj)
    assert ours.dtype == np.float32 and ours.shape == shape
    rel = np.linalg.norm(ours.astype(np.float64) - ref) / np.linalg.norm(ref)
    assert rel < 1e-5


@pytest.mark.parametrize("shape", SHAPES)
def test_aligned_error_matches_fp64(gpu, shape):
    """Unrelated objects, a shifted and rotated copy with noise, and a shifted
    twin: the device error agrees with the oracle's to 1e-5 (relative, or
    absolute below 1e-5)."""
    n = int(np.prod(shape))
    ref = random_field(n, 1).reshape(shape)
    rng = np.random.default_rng(2)
    shift = tuple(int(rng.integers(0, s)) for s in shape)
    noise = 1e-3 * random_field(n, 4).reshape(shape)
    moved = (np.roll(ref, shift, axis=tuple(range(len(shape)))) * np.exp(0.7j) + noise)
    twin = np.conj(np.flip(ref, axis=tuple(range(len(shape)))))
    twin = np.roll(twin, shift, axis=tuple(range(len(shape)))).astype(np.complex64)
    cases = [random_field(n, 7).reshape(shape), moved.astype(np.complex64), twin]
    ours = qpc.aligned_error(np.stack(cases), ref)
    for a, e in zip(cases, ours, strict=True):
        expected = fp64.aligned_error(a, ref)
        assert abs(e - expected) <= 1e-5 * max(expected, 1.0), (e, expected)
    assert ours[1] < 2e-3 and ours[2] < 1e-5
    assert qpc.aligned_error(cases[1], ref) == pytest.approx(float(ours[1]), rel=1e-6)


def test_aligned_error_scores_reconstructions(gpu):
    """The README triangle reconstructed from 4 starts: the device scores every
    start as the oracle does."""
    obj, support, intensity = triangle((64, 64), 20)
    runs = qpc.reconstruct(intensity, support=support, starts=4, seed=2)
    ours = qpc.aligned_error(np.stack([r.object for r in runs]), obj)
    for r, e in zip(runs, ours, strict=True):
        expected = fp64.aligned_error(r.object, obj)
        assert abs(e - expected) <= 1e-5 * max(expected, 1.0)


def test_shape_mismatch_is_a_value_error(gpu):
    with pytest.raises(ValueError, match="shapes differ"):
        qpc.aligned_error(np.zeros((8, 8), np.complex64), np.zeros((8, 9), np.complex64))


def numpy_align(a, ref):
    """The translation, twin and phase of src/core/metrics.cpp:17-86, applied
    with numpy complex128 (the same steps as the oracle's aligned_error)."""
    axes = tuple(range(ref.ndim))
    best = None
    for cand in (a, np.roll(np.conj(np.flip(a, axis=axes)), 1, axis=axes)):
        cand = cand.astype(np.complex128)
        cc = np.fft.ifftn(np.fft.fftn(ref) * np.conj(np.fft.fftn(cand)))
        shift = np.unravel_index(int(np.argmax(np.abs(cc) ** 2)), ref.shape)
        moved = np.roll(cand, shift, axis=axes)
        overlap = np.sum(ref * np.conj(moved))
        moved = moved * (overlap / abs(overlap))
        err = np.linalg.norm(moved - ref) / np.linalg.norm(ref)
        if best is None or err < best[1]:
            best = (moved, err)
    return best


@pytest.mark.parametrize("shape", [(64, 48), (21, 15), (16, 20, 12)])
def test_align_moves_every_object_onto_the_reference(gpu, shape):
    n = int(np.prod(shape))
    axes = tuple(range(len(shape)))
    ref = random_field(n, 1).reshape(shape)
    rng = np.random.default_rng(3)
    objs = []
    for k in range(4):
        shift = tuple(int(rng.integers(0, s)) for s in shape)
        o = np.roll(ref, shift, axis=axes) * np.exp(1j * rng.uniform(-3, 3))
        if k % 2:
            o = np.conj(np.flip(o, axis=axes))
        objs.append((o + 1e-3 * random_field(n, 10 + k).reshape(shape)).astype(np.complex64))
    stack = np.stack(objs)
    aligned, mean, errors = qpc.align(stack, ref)
    np.testing.assert_allclose(errors, qpc.aligned_error(stack, ref), rtol=1e-6)
    for a, o in zip(aligned, objs, strict=True):
        expected, err = numpy_align(o, ref.astype(np.complex128))
        assert fp64.relative_diff(a, expected) < 1e-5
        assert fp64.relative_diff(a, ref) < 2e-3
    assert fp64.relative_diff(mean, np.mean(aligned.astype(np.complex128), axis=0)) < 1e-6
    assert fp64.relative_diff(mean, ref) < 1e-3


def test_ensemble_average(gpu):
    obj, support, intensity = triangle((64, 64), 20)
    ens = qpc.reconstruct(intensity, support=support, starts=4, seed=2)
    mean, errors = ens.average()
    assert mean.shape == obj.shape and errors.shape == (4,)
    assert errors[0] < 1e-6  # the best run against itself
    one, e1 = ens.average(runs=1)
    np.testing.assert_allclose(one, ens.best.object, rtol=0, atol=1e-6)
