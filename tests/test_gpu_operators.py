"""Single operators on the device against the FP64 oracle.

Tolerances: 1e-5 relative L2 for FP32 operators (modulus projection, blur);
exact for the support cut and the detwin half support; autocorrelation
support exact except for pixels within 1e-6 (relative to the level) of the
threshold. Shapes follow the reference's tests (test_operators.cpp:77-78,
test_cuda.cpp:26-54) plus the benchmark sizes.
"""

import numpy as np
import pytest

from oracle import fp64
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc

pytestmark = pytest.mark.gpu

SHAPES = [(32, 32), (17, 24), (16, 16, 16), (48, 40), (21, 15), (16, 20, 12), (64, 64),
          (128, 128), (256, 256), (512, 512), (64, 64, 64), (1, 64), (96, 250)]


def pair(intensity, support=None, mask=None):
    return (fp64.make_problem(intensity, support, mask),
            qpc.make_problem(intensity, support=support, mask=mask))


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_modulus_projection_matches_fp64(gpu, shape):
    obj, support, intensity = triangle(shape, min(8, min(shape)))
    mask = np.zeros(shape, np.uint8)
    mask.flat[5] = 1
    mask.flat[mask.size // 2] = 1
    ref_p, p = pair(intensity, support, mask)
    x = random_field(int(np.prod(shape)), 5).reshape(shape)
    ref, ref_err = fp64.modulus_project(ref_p, x)
    out, err = qpc.modulus_project(p, x)
    assert fp64.relative_diff(out, ref) < 1e-5
    assert abs(err - ref_err) <= 1e-5 * ref_err
    # idempotent up to float rounding: the projection lands on the modulus set
    _, again = qpc.modulus_project(p, out)
    assert again < 1e-5


_GENERIC_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import qoraphasecu_b200 as qpc
from synthetic import random_field, triangle
out = {{}}
for shape in {shapes!r}:
    _, support, intensity = triangle(shape, 8)
    p = qpc.make_problem(intensity, support=support)
    x = random_field(int(np.prod(shape)), 7).reshape(shape)
    out["x".join(map(str, shape))] = qpc.modulus_project(p, x)[0]
    out["blur" + "x".join(map(str, shape))] = qpc.gaussian_blur(np.abs(x), 1.3)
np.savez({path!r}, **out)
"""


def test_register_resident_passes_match_the_generic_passes(gpu, tmp_path):
    """The power-of-two kernels and the generic mixed-radix kernels compute the
    same transforms (to FP32 rounding); the generic ones run in a child process
    with QPB_GENERIC_PASSES=1."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    tests = Path(__file__).resolve().parent
    shapes = [(16, 16), (32, 64), (64, 64), (128, 128), (256, 256), (512, 256), (1024, 16),
              (16, 32, 64), (64, 64, 64)]
    path = tmp_path / "generic.npz"
    script = _GENERIC_SCRIPT.format(root=str(tests.parent), tests=str(tests), shapes=shapes,
                                    path=str(path))
    env = dict(os.environ, QPB_GENERIC_PASSES="1")
    subprocess.run([sys.executable, "-c", script], check=True, env=env, timeout=600)
    generic = np.load(path)
    for shape in shapes:
        _, support, intensity = triangle(shape, 8)
        p = qpc.make_problem(intensity, support=support)
        x = random_field(int(np.prod(shape)), 7).reshape(shape)
        key = "x".join(map(str, shape))
        assert fp64.relative_diff(qpc.modulus_project(p, x)[0], generic[key]) < 2e-6, shape
        blur = qpc.gaussian_blur(np.abs(x), 1.3)
        assert np.abs(blur - generic["blur" + key]).max() < 1e-5 * np.abs(blur).max(), shape


def test_error_is_zero_at_the_true_object(gpu):
    obj, support, intensity = triangle((32, 32), 8)
    _, p = pair(intensity, support)
    out, err = qpc.modulus_project(p, obj)
    assert err < 1e-5
    assert np.abs(out - obj).max() < 1e-4


def test_masked_pixels_keep_their_computed_magnitude(gpu):
    obj, support, intensity = triangle((32, 32), 8)
    mask = np.zeros((32, 32), np.uint8)
    mask.flat[0] = 1
    mask.flat[512] = 1
    p_masked = qpc.make_problem(intensity, support=support, mask=mask)
    p_plain = qpc.make_problem(intensity, support=support)
    x = random_field(32 * 32, 2).reshape(32, 32)
    a, _ = qpc.modulus_project(p_masked, x)
    b, _ = qpc.modulus_project(p_plain, x)
    assert np.abs(a - b).max() > 1e-4
    assert qpc.modulus_project(p_masked, a)[1] < 1e-5


@pytest.mark.parametrize("storage,tol", [("f16", 2e-3), ("bf16", 1e-2)])
def test_low_precision_amplitude_storage(gpu, storage, tol):
    """FP16/BF16 amplitude storage with FP32 arithmetic: error vs the FP64 oracle
    is bounded by the storage rounding of the amplitude."""
    obj, support, intensity = triangle((64, 64), 16)
    ref_p, p = pair(intensity, support)
    x = random_field(64 * 64, 9).reshape(64, 64)
    ref, ref_err = fp64.modulus_project(ref_p, x)
    out, err = qpc.modulus_project(p, x, amp_storage=storage)
    rel = fp64.relative_diff(out, ref)
    print(f"{storage}: relative L2 vs FP64 {rel:.2e}, error {err:.6e} vs {ref_err:.6e}")
    assert rel < tol
    assert abs(err - ref_err) <= tol * ref_err


@pytest.mark.parametrize("shape", [(32, 32), (17, 24), (16, 16, 16), (16, 20, 12), (256, 256)],
                         ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("sigma", [0.0, 1.0, 1.5, 4.0])
def test_gaussian_blur_matches_fp64(gpu, shape, sigma):
    rng = np.random.default_rng(3)
    image = rng.random(shape).astype(np.float32)
    ref = fp64.gaussian_blur(image, sigma)
    out = qpc.gaussian_blur(image, sigma)
    rel = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert rel < 1e-5
    assert np.abs(out - ref).max() < 1e-5 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("shape", [(32, 32), (17, 24), (16, 16, 16)])
def test_blur_preserves_the_sum(gpu, shape):
    image = np.zeros(shape, np.float32)
    image.flat[image.size // 2 + 3] = 1.0
    blurred = qpc.gaussian_blur(image, 1.5)
    assert abs(blurred.astype(np.float64).sum() - 1.0) < 1e-5
    assert blurred.max() < 0.5


def test_support_projection_is_exact(gpu):
    obj, support, _ = triangle((16, 20, 12), 6)
    x = random_field(16 * 20 * 12, 6).reshape(16, 20, 12)
    out = qpc.support_project(support, x)
    np.testing.assert_array_equal(out, fp64.support_project(support, x).astype(np.complex64))
    np.testing.assert_array_equal(qpc.support_project(support, out), out)


def test_half_support_keeps_the_lower_half(gpu):
    """tests/test_problem.cpp:62-77."""
    support = np.zeros((8, 4), bool)
    support[2:6, :] = True
    half = qpc.half_support(support, 0)
    expect = np.zeros((8, 4), bool)
    expect[2:4, :] = True
    np.testing.assert_array_equal(half, expect)
    columns = qpc.half_support(support, 1)
    assert columns[2, 1] and not columns[2, 2]


@pytest.mark.parametrize("shape,axis", [((64, 48), 0), ((64, 48), 1), ((17, 24), 1),
                                        ((16, 20, 12), 2), ((16, 20, 12), 0)])
def test_half_support_matches_fp64(gpu, shape, axis):
    _, support, _ = triangle(shape, 9)
    rng = np.random.default_rng(1)
    support = support | (rng.random(shape) < 0.05)
    np.testing.assert_array_equal(qpc.half_support(support, axis),
                                  fp64.half_support(support, axis).astype(bool))


def _band_mismatch(ours, ref_values, level, threshold, band=1e-6):
    cut = threshold * level
    differ = ours != (ref_values > cut)
    near = np.abs(ref_values - cut) <= band * level
    return np.count_nonzero(differ & ~near)


@pytest.mark.parametrize("shape", [(64, 64), (17, 24), (16, 16, 16), (256, 256)])
def test_autocorrelation_support_matches_fp64(gpu, shape):
    _, _, intensity = triangle(shape, min(16, min(shape) // 2))
    ours = qpc.autocorrelation_support(intensity, 0.1)
    buf = fp64.to_fft_order(intensity).astype(np.complex128)
    ac = fp64.to_centered(np.abs(fp64.Fft(len(shape)).inverse(buf)))
    assert _band_mismatch(ours, ac, ac.max(), 0.1) == 0
    ref = fp64.autocorrelation_support(intensity, 0.1).astype(bool)
    assert ours.sum() > 0 and np.count_nonzero(ours != ref) <= 2


def test_make_problem_clips_and_rejects(gpu):
    """tests/test_problem.cpp:29-46."""
    p = qpc.make_problem(np.array([[4.0, -1.0], [9.0, 0.0]], np.float32),
                         support=np.array([[1, 1], [0, 0]], bool))
    np.testing.assert_array_equal(p.amplitude, [[2, 0], [3, 0]])
    np.testing.assert_array_equal(p.mask, 0)
    four = np.ones((2, 2), np.float32)
    with pytest.raises(ValueError):
        qpc.make_problem(four, mask=np.ones((2, 2), bool))
    bad = four.copy()
    bad[0, 1] = np.nan
    with pytest.raises(ValueError):
        qpc.make_problem(bad)
    with pytest.raises(ValueError):
        qpc.make_problem(np.ones(4, np.float32))
