"""The amplitude-loss adjoint kernel behind torch.autograd.

Checks, against the FP64 oracle: the loss value; the gradient against the
identity 2 (x - P_M x) built from the oracle's modulus projection
(src/cpu/kernels.cpp:25-42 of the reference); the gradient against complex128
central finite differences on 32 x 32 crops; the autograd wiring; and that
Adam with the support projection converges.
"""

import numpy as np
import pytest

from oracle import fp64
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200 import autograd as qad

pytestmark = pytest.mark.gpu


def fp64_loss(problem, x_centred):
    """sum over usable pixels of (|F x| - A)^2, complex128."""
    fft = fp64.Fft(x_centred.ndim)
    y = fft.forward(fp64.to_fft_order(np.asarray(x_centred, np.complex128)))
    amp = fp64.to_fft_order(problem.amplitude).astype(np.float64)
    usable = fp64.to_fft_order(problem.mask) == 0
    return float(np.sum(np.where(usable, (np.abs(y) - amp) ** 2, 0.0)))


def device_loss_grad(problem_q, x_centred):
    import torch

    model = qad.AmplitudeModel(problem_q)
    nd = x_centred.ndim
    x = torch.from_numpy(np.ascontiguousarray(np.fft.ifftshift(x_centred)).astype(np.complex64)).cuda()
    loss, grad = qad._loss_and_grad(x[None], model.signed, model.shape)
    torch.cuda.synchronize()
    g = np.fft.fftshift(grad[0].cpu().numpy(), axes=tuple(range(-nd, 0)))
    return float(loss[0].item()), g


@pytest.mark.parametrize("shape", [(64, 64), (48, 40), (16, 16, 16), (256, 256)])
def test_loss_and_gradient_match_fp64(gpu, shape):
    _, support, intensity = triangle(shape, 8)
    mask = np.zeros(shape, np.uint8)
    mask.flat[7] = 1
    ref_p = fp64.make_problem(intensity, support, mask)
    p = qpc.make_problem(intensity, support=support, mask=mask)
    x = random_field(int(np.prod(shape)), 13).reshape(shape)
    loss, grad = device_loss_grad(p, x)
    ref_loss = fp64_loss(ref_p, x)
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    projected, _ = fp64.modulus_project(ref_p, x)
    identity = 2.0 * (x.astype(np.complex128) - projected)
    assert fp64.relative_diff(grad, identity) < 1e-5


def test_gradient_matches_complex128_finite_differences(gpu):
    """Central differences of the FP64 loss along random complex directions on
    32 x 32 crops (the central crop of a 64 x 64 object, with its own intensity)."""
    obj, support, _ = triangle((64, 64), 20)
    crop = obj[16:48, 16:48].astype(np.complex64)
    intensity = fp64.simulate_intensity(crop)
    p = qpc.make_problem(intensity, support=support[16:48, 16:48])
    ref_p = fp64.make_problem(intensity, support[16:48, 16:48])
    rng = np.random.default_rng(5)
    x = (crop + 0.3 * (rng.standard_normal(crop.shape) + 1j * rng.standard_normal(crop.shape))
         ).astype(np.complex64)
    _, grad = device_loss_grad(p, x)
    x128 = x.astype(np.complex128)
    h = 1e-4
    for _ in range(6):
        v = rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape)
        v /= np.linalg.norm(v)
        fd = (fp64_loss(ref_p, x128 + h * v) - fp64_loss(ref_p, x128 - h * v)) / (2 * h)
        analytic = float(np.real(np.vdot(grad.astype(np.complex128), v)))
        # The directional derivative of a unit direction is at most ||grad||;
        # the gradient itself is FP32, good to 1e-5 of its norm.
        assert abs(fd - analytic) <= 1e-5 * np.linalg.norm(grad), (fd, analytic)


def test_autograd_backward_scales_the_gradient(gpu):
    import torch

    _, support, intensity = triangle((32, 32), 8)
    p = qpc.make_problem(intensity, support=support)
    model = qad.AmplitudeModel(p)
    x0 = np.stack([np.fft.ifftshift(random_field(1024, s).reshape(32, 32)) for s in (1, 2)])
    x = torch.from_numpy(x0.astype(np.complex64)).cuda().requires_grad_(True)
    losses = qad.amplitude_loss(x, model)
    assert losses.shape == (2,)
    (3.0 * losses[0] + 0.5 * losses[1]).backward()
    _, g0 = qad._loss_and_grad(x.detach(), model.signed, model.shape)
    expected = g0.clone()
    expected[0] *= 3.0
    expected[1] *= 0.5
    torch.testing.assert_close(x.grad, expected, rtol=1e-6, atol=1e-6)


def test_adam_with_support_projection_converges(gpu):
    obj, support, intensity = triangle((64, 64), 20)
    p = qpc.make_problem(intensity, support=support)
    runs = qad.adam_reconstruct(p, starts=2, steps=300, lr=1e-2, seed=3)
    for run in runs:
        assert run.errors.shape == (300,)
        assert run.errors[-1] < 0.5 * run.errors[0]
        assert np.all(run.object[~support.astype(bool)] == 0)


def test_adam_magnitude_bound_keeps_masked_directions_in_check(gpu):
    """Under a beamstop the loss leaves the masked Fourier components free;
    the per-pixel bound keeps every start's object within `bound` RMS
    amplitudes of the support, and the bounded run converges as far as the
    unbounded one."""
    from qoraphasecu_b200 import workloads

    obj = workloads.square(128, seed=5)
    intensity = np.abs(np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(obj), norm="ortho"))) ** 2
    mask = workloads.beamstop(obj.shape, 4.0)
    support = qpc.autocorrelation_support(intensity)
    p = qpc.make_problem(intensity.astype(np.float32), support=support, mask=mask)
    bounded = qad.adam_reconstruct(p, starts=4, steps=400, lr=2e-2, seed=1, bound=8.0)
    free = qad.adam_reconstruct(p, starts=4, steps=400, lr=2e-2, seed=1, bound=None)
    usable = mask == 0
    inside = max(int(np.count_nonzero(support)), 1)
    rms = np.sqrt(np.sum(intensity[usable].astype(np.float64)) / inside)
    for b, f in zip(bounded, free, strict=True):
        assert np.all(np.isfinite(b.object))
        assert float(np.max(np.abs(b.object))) <= 8.0 * rms * (1 + 1e-5)
        assert np.all(b.object[~support.astype(bool)] == 0)
        assert b.errors[-1] <= f.errors[-1] * 1.25 + 1e-3


def test_adam_graph_replay_equals_eager_steps(gpu):
    """The captured step replays the eager step's arithmetic: identical
    objects, per-step errors equal up to the FP64 sums' order."""
    obj, support, intensity = triangle((64, 64), 20)
    p = qpc.make_problem(intensity, support=support)
    eager = qad.adam_reconstruct(p, starts=3, steps=40, lr=1e-2, seed=2, graph=False)
    replayed = qad.adam_reconstruct(p, starts=3, steps=40, lr=1e-2, seed=2, graph=True)
    for a, b in zip(eager, replayed, strict=True):
        assert b.errors.shape == (40,)
        np.testing.assert_array_equal(b.object, a.object)
        np.testing.assert_allclose(b.errors, a.errors, rtol=1e-6)


def test_project_support_bound_matches_the_elementwise_formula(gpu):
    """The fused projection after an Adam step against the element-wise torch
    formula it replaces (x * support, then x * min(1, bound / |x|)): two
    elements a thread (even sizes) and one (odd sizes), batches of objects,
    magnitudes on both sides of the bound, and the support alone."""
    import torch

    for shape, batch in (((64, 48), 3), ((15, 17), 2), ((8, 8, 9), 1)):
        g = torch.Generator(device="cuda").manual_seed(5)
        x = torch.randn((batch, *shape), dtype=torch.complex64, device="cuda", generator=g) * 4
        support = torch.rand(shape, device="cuda", generator=g) > 0.3
        inside = support.expand_as(x)
        for bound in (3.0, None):
            want = x * support
            if bound is not None:
                want = want * torch.clamp(bound / torch.abs(want).clamp_min(1e-30), max=1.0)
            got = qad.project_support_bound(x.clone(), support, bound)
            torch.testing.assert_close(got, want, rtol=1e-6, atol=0.0)
            assert torch.all(got[~inside] == 0)
            below = inside & (torch.abs(x) <= (bound if bound is not None else float("inf")))
            assert torch.equal(got[below], x[below])
            if bound is not None:
                assert float(torch.abs(got).max()) <= bound * (1 + 1e-6)
                assert bool(torch.any(~below & inside))  # some pixels were scaled


def test_adam_reconstruction_matches_the_same_algorithm_in_fp64(gpu):
    """adam_reconstruct (FP32 line passes, torch's fused Adam on the objects'
    real view, the fused support-and-bound projection, graph replay) against
    the same algorithm in FP64 on the host (torch complex128, torch.fft),
    from the same starts: per-step Fourier errors and final objects within
    1e-5 relative after 60 steps."""
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from precision_report import _adam_fp64

    from qoraphasecu_b200 import workloads

    rng = np.random.default_rng(41)
    obj = workloads.square(256, seed=41)
    intensity = workloads.poisson(workloads.simulate_intensity(obj), 1e7, rng)
    p = qpc.make_problem(intensity, mask=workloads.beamstop((256, 256), 6))
    with qpc.Solver(p, starts=2, seed=0) as drawn:
        first = drawn.results()
    x0 = np.stack([np.fft.ifftshift(r.object) for r in first]).astype(np.complex128)
    amp = np.fft.ifftshift(np.asarray(p.amplitude, np.float64))
    usable = np.fft.ifftshift(np.asarray(p.mask)) == 0
    support = np.fft.ifftshift(np.asarray(p.support)) != 0
    energy = float(np.sum(np.where(usable, amp ** 2, 0.0)))
    scale = float(np.sqrt(energy / max(int(support.sum()), 1)))
    ours = qad.adam_reconstruct(p, starts=2, steps=60, lr=1e-2, seed=0, bound=16.0)
    x, errors = _adam_fp64(x0, scale, amp, usable, support, 60, 1e-2, 16.0)
    for run, e, xs in zip(ours, errors, x, strict=True):
        np.testing.assert_allclose(run.errors, e, rtol=1e-5)
        assert fp64.relative_diff(run.object, np.fft.fftshift(xs)) < 1e-5
