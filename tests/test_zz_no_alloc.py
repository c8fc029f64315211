"""The allocation-free modulus projection, qpb_modulus_project_noalloc.

Applications that reserve all their GPU memory when they start (a detector
pipeline with a fixed budget, a service whose pool already holds most of HBM)
cannot let a library call cudaMalloc later, and neither can host threads that
must not stall on cudaMalloc's device-wide synchronisation. This entry point
serves them: it allocates nothing and keeps its scratch in a fixed array inside
libqpb.so, while the caller provides every input and output in device memory.

The test calls it through the C ABI several times in a row, on shapes that run
every kind of line pass it can reach: the generic mixed-radix passes (48 x 40,
16 x 20 x 12, the 4096-point rows of 16 x 4096), the register-resident
power-of-two passes with bulk-copied row tiles and the stage-major twiddle
slots (256 x 256, its maximum, and 64 x 32 x 32), then a shape it already ran
(whose twiddle tables it reuses) and an in-place call (out == x). Each result
is compared with the allocating qpb_modulus_project and with the FP64 oracle at
the 1e-5 relative tolerance of the other modulus-projection tests. It also
checks that a shape above the stated maximum and a misaligned pointer are
refused before anything is launched. This file is collected last, so that a
failure here never stops the rest of the suite from running first.
"""

import ctypes

import numpy as np
import pytest

from oracle import fp64
from oracle.fp64 import relative_diff
from synthetic import random_field, triangle

import qoraphasecu_b200 as qpc
from qoraphasecu_b200 import _lib

pytestmark = pytest.mark.gpu

# (shape, triangle side, seed of the iterate)
CASES = (
    ((48, 40), 12, 5),
    ((16, 20, 12), 6, 6),
    ((256, 256), 40, 7),
    ((64, 32, 32), 10, 8),
    ((16, 4096), 8, 9),
    ((48, 40), 10, 10),
)


def _to_device(array):
    import torch

    return torch.from_numpy(np.ascontiguousarray(array)).cuda()


def _call(lib, shape, amp, mask, x, out, err, stream):
    return lib.qpb_modulus_project_noalloc(
        len(shape), _lib.shape_arg(shape), ctypes.c_void_p(amp.data_ptr()),
        ctypes.c_void_p(mask.data_ptr()) if mask is not None else None,
        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(err.data_ptr()), ctypes.c_void_p(stream))


def _case(shape, m, seed):
    n = int(np.prod(shape))
    _, support, intensity = triangle(shape, m)
    mask = np.zeros(shape, np.uint8)
    mask.flat[3] = 1
    mask.flat[n // 2] = 1
    problem = qpc.make_problem(intensity, support=support, mask=mask)
    oracle_problem = fp64.make_problem(intensity, support, mask)
    x = random_field(n, seed).reshape(shape)
    return problem, oracle_problem, x


def _check(shape, problem, oracle_problem, x, got, err):
    expected, expected_err = qpc.modulus_project(problem, x)
    assert relative_diff(got, expected) < 1e-5, shape
    assert abs(err - expected_err) <= 1e-5 * expected_err, shape
    ref_out, ref_err = fp64.modulus_project(oracle_problem, x)
    assert relative_diff(got, ref_out) < 1e-5, shape
    assert abs(err - ref_err) <= 1e-5 * ref_err, shape


def test_noalloc_projection_matches_the_allocating_one(gpu):
    import torch

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for shape, m, seed in CASES:
        problem, oracle_problem, x = _case(shape, m, seed)
        amp = _to_device(np.fft.ifftshift(problem.amplitude))
        msk = _to_device(np.fft.ifftshift(problem.mask))
        xd = _to_device(np.fft.ifftshift(x).astype(np.complex64).view(np.float32))
        out = torch.empty_like(xd)
        err = torch.full((1,), float("nan"), dtype=torch.float32, device="cuda")
        _lib.check(_call(lib, shape, amp, msk, xd, out, err, stream))
        torch.cuda.synchronize()
        got = np.fft.fftshift(out.cpu().numpy().view(np.complex64).reshape(shape))
        _check(shape, problem, oracle_problem, x, got, float(err.item()))


def test_noalloc_projection_in_place(gpu):
    import torch

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for shape, m, seed in (((256, 256), 40, 11), ((64, 32, 32), 10, 12), ((48, 40), 12, 13)):
        problem, oracle_problem, x = _case(shape, m, seed)
        amp = _to_device(np.fft.ifftshift(problem.amplitude))
        msk = _to_device(np.fft.ifftshift(problem.mask))
        xd = _to_device(np.fft.ifftshift(x).astype(np.complex64).view(np.float32))
        err = torch.full((1,), float("nan"), dtype=torch.float32, device="cuda")
        _lib.check(_call(lib, shape, amp, msk, xd, xd, err, stream))
        torch.cuda.synchronize()
        got = np.fft.fftshift(xd.cpu().numpy().view(np.complex64).reshape(shape))
        _check(shape, problem, oracle_problem, x, got, float(err.item()))


def test_noalloc_refuses_shapes_above_its_maximum(gpu):
    import torch

    lib = _lib.load()
    small = torch.zeros(8, dtype=torch.float32, device="cuda")
    status = _call(lib, (512, 512), small, None, small, small, small, 0)
    assert status == _lib.INVALID_ARGUMENT
    assert "maximum" in lib.qpb_last_error().decode()
    status = _call(lib, (8, 8192), small, None, small, small, small, 0)
    assert status == _lib.INVALID_ARGUMENT


def test_noalloc_refuses_misaligned_arrays(gpu):
    """A complex64 view that starts at an odd element is 8-byte aligned only;
    the bulk copies that move x and out need 16 bytes, so the call refuses it
    before launching anything."""
    import torch

    lib = _lib.load()
    shape = (16, 16)
    buf = torch.zeros(2 * (256 + 1), dtype=torch.float32, device="cuda")
    odd = buf[2:]  # one complex64 element in: 8 bytes past a 16-byte boundary
    assert odd.data_ptr() % 16 == 8
    amp = torch.ones(256, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.float32, device="cuda")
    before = qpc.api.kernel_launches()
    status = _call(lib, shape, amp, None, odd, buf[:512], err, 0)
    assert status == _lib.INVALID_ARGUMENT
    assert "aligned" in lib.qpb_last_error().decode()
    status = _call(lib, shape, amp, None, buf[:512], odd, err, 0)
    assert status == _lib.INVALID_ARGUMENT
    assert qpc.api.kernel_launches() == before
