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
