"""Device-resident inputs and outputs: CUDA torch tensors in, CUDA torch
tensors out, the same numbers as the host path."""

import numpy as np
import pytest

from oracle import fp64
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200.recipe import ER, HIO, Recipe, Shrinkwrap

pytestmark = pytest.mark.gpu


def test_make_problem_on_the_device_equals_the_host(gpu):
    import torch

    _, support, intensity = triangle((64, 48), 14)
    intensity = intensity.copy()
    intensity[3, 5] = -2.0  # clipped to zero amplitude
    mask = np.zeros(intensity.shape, np.uint8)
    mask[32, 24] = 1
    host = qpc.make_problem(intensity, mask=mask)
    dev = qpc.make_problem(torch.from_numpy(intensity).cuda(), mask=torch.from_numpy(mask).cuda())
    assert dev.on_device and not host.on_device
    np.testing.assert_array_equal(dev.amplitude.cpu().numpy(), host.amplitude)
    np.testing.assert_array_equal(dev.mask.cpu().numpy(), host.mask)
    # autocorrelation support: the same device transform, the same threshold
    np.testing.assert_array_equal(dev.support.cpu().numpy(), host.support)
    ref = fp64.autocorrelation_support(intensity)
    assert np.mean(dev.support.cpu().numpy() != ref) < 1e-3
    given = qpc.make_problem(torch.from_numpy(intensity).cuda(),
                             support=torch.from_numpy(support).cuda())
    np.testing.assert_array_equal(given.support.cpu().numpy(), support != 0)


def test_device_errors_are_value_errors(gpu):
    import torch

    bad = torch.zeros((16, 16), device="cuda")
    bad[2, 2] = float("nan")
    with pytest.raises(ValueError, match="NaN"):
        qpc.make_problem(bad)
    with pytest.raises(ValueError, match="every pixel"):
        qpc.make_problem(torch.ones((16, 16), device="cuda"),
                         mask=torch.ones((16, 16), dtype=torch.uint8, device="cuda"))


@pytest.mark.parametrize("shape,m", [((64, 64), 20), ((40, 36), 10), ((16, 16, 16), 6)])
def test_reconstruct_on_the_device_equals_the_host(gpu, shape, m):
    import torch

    _, support, intensity = triangle(shape, m)
    recipe = Recipe(HIO(20), Shrinkwrap(), ER(10))
    host = qpc.reconstruct(intensity, support=support, recipe=recipe, starts=3, seed=4)
    dev = qpc.reconstruct(torch.from_numpy(intensity).cuda(),
                          support=torch.from_numpy(support).cuda(), recipe=recipe, starts=3,
                          seed=4)
    for h, d in zip(host, dev, strict=True):
        assert d.object.is_cuda and d.support.is_cuda
        np.testing.assert_array_equal(d.object.cpu().numpy(), h.object)
        np.testing.assert_array_equal(d.support.cpu().numpy(), h.support)
        np.testing.assert_allclose(d.errors, h.errors, rtol=1e-6)
        assert torch.allclose(d.amplitude, torch.from_numpy(np.abs(h.object)).cuda())


def test_device_init(gpu):
    import torch

    _, support, intensity = triangle((32, 24), 8)
    init = np.stack([random_field(32 * 24, 5).reshape(32, 24), random_field(32 * 24, 6).reshape(32, 24)])
    recipe = Recipe(HIO(5), ER(5))
    host = qpc.reconstruct(intensity, support=support, recipe=recipe, starts=2, init=init)
    dev = qpc.reconstruct(torch.from_numpy(intensity).cuda(),
                          support=torch.from_numpy(support).cuda(), recipe=recipe, starts=2,
                          init=torch.from_numpy(init.astype(np.complex64)).cuda())
    for h, d in zip(host, dev, strict=True):
        np.testing.assert_array_equal(d.object.cpu().numpy(), h.object)
    with pytest.raises(ValueError, match="CUDA tensor"):
        qpc.reconstruct(torch.from_numpy(intensity).cuda(), recipe=recipe, starts=2, init=init)
