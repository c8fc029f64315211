"""The allocation-free modulus projection, qpb_modulus_project_noalloc.

Applications that reserve all their GPU memory when they start (a detector
pipeline with a fixed budget, a service whose pool already holds most of HBM)
cannot let a library call cudaMalloc later, and neither can host threads that
must not stall on cudaMalloc's device-wide synchronisation. This entry point
serves them: it allocates nothing and keeps its scratch in a fixed array inside
libqpb.so, while the caller provides every input and output in device memory.

The test calls it through the C ABI twice in a row, on two different shapes so
that anything the first call leaves in the shared scratch would spoil the
second, and compares each result with the allocating qpb_modulus_project at the
1e-5 relative tolerance of the other modulus-projection tests. It also checks
that a shape above the stated maximum is refused. This file is collected last,
so that a failure here never stops the rest of the suite from running first.
"""

import ctypes

import numpy as np
import pytest

from oracle.fp64 import relative_diff
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200 import _lib

pytestmark = pytest.mark.gpu


def _to_device(array):
    import torch

    return torch.from_numpy(np.ascontiguousarray(array)).cuda()


def _call(lib, shape, amp, mask, x, out, err, stream):
    return lib.qpb_modulus_project_noalloc(
        len(shape), _lib.shape_arg(shape), ctypes.c_void_p(amp.data_ptr()),
        ctypes.c_void_p(mask.data_ptr()) if mask is not None else None,
        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(err.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_projection_matches_the_allocating_one_twice(gpu):
    import torch

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for shape, seed in (((48, 40), 5), ((16, 20, 12), 6)):
        n = int(np.prod(shape))
        _, support, intensity = triangle(shape, 6)
        mask = np.zeros(shape, np.uint8)
        mask.flat[3] = 1
        mask.flat[n // 2] = 1
        problem = qpc.make_problem(intensity, support=support, mask=mask)
        x = random_field(n, seed).reshape(shape)
        expected, expected_err = qpc.modulus_project(problem, x)

        amp = _to_device(np.fft.ifftshift(problem.amplitude))
        msk = _to_device(np.fft.ifftshift(problem.mask))
        xd = _to_device(np.fft.ifftshift(x).astype(np.complex64).view(np.float32))
        out = torch.empty_like(xd)
        err = torch.full((1,), float("nan"), dtype=torch.float32, device="cuda")
        _lib.check(_call(lib, shape, amp, msk, xd, out, err, stream))
        torch.cuda.synchronize()
        got = np.fft.fftshift(out.cpu().numpy().view(np.complex64).reshape(shape))
        assert relative_diff(got, expected) < 1e-5, shape
        assert abs(float(err.item()) - expected_err) <= 1e-5 * expected_err, shape


def test_noalloc_refuses_shapes_above_its_maximum(gpu):
    import torch

    lib = _lib.load()
    small = torch.zeros(8, dtype=torch.float32, device="cuda")
    status = _call(lib, (512, 512), small, None, small, small, small, 0)
    assert status == _lib.INVALID_ARGUMENT
    assert "maximum" in lib.qpb_last_error().decode()
    status = _call(lib, (8, 8192), small, None, small, small, small, 0)
    assert status == _lib.INVALID_ARGUMENT
