"""The point-wise step's quotient and square root (qpb::divide and
qpb::square_root in projection.cuh) against the correctly rounded IEEE
operations.

The reference evaluates |y| = sqrtf(re^2 + im^2) and target / (|y| + eps)
with the IEEE square root and division (src/cuda/device.cuh:20-27,
src/cpu/kernels.cpp:32-39). The kernels refine the hardware's approximate
reciprocal and reciprocal square root by Newton-Raphson steps with FMA
residuals (Markstein's methods), which have no slow path. Over the operand
ranges the step meets (amplitudes and magnitudes from 0 to 1e7, denominators
|y| + 1e-12, squared magnitudes down to subnormals) every result must be within
one ulp of numpy's correctly rounded float32 result, and nearly all of them
equal to it."""

import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("divide") / "libdivide_check.so"
    subprocess.run(
        ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++20",
         "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared",
         "-I", str(ROOT / "include"), "-I", str(ROOT / "qoraphasecu_b200" / "csrc"),
         str(Path(__file__).with_name("divide_check.cu")), "-o", str(out)],
        check=True)
    lib = ctypes.CDLL(str(out))
    lib.divide_on_device.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_longlong]
    return lib


def _divide(lib, a, b=None):
    a = np.ascontiguousarray(a, np.float32)
    bp = None
    if b is not None:
        b = np.ascontiguousarray(b, np.float32)
        bp = b.ctypes.data
    q = np.empty_like(a)
    rc = lib.divide_on_device(a.ctypes.data, bp, q.ctypes.data, a.size)
    assert rc == 0, f"CUDA error {rc}"
    return q


def _ulps(x, y):
    """Distance in units in the last place between float32 arrays of one sign."""
    xi = x.view(np.int32).astype(np.int64)
    yi = y.view(np.int32).astype(np.int64)
    return np.abs(xi - yi)


def test_divide_matches_ieee_division(gpu, harness):
    rng = np.random.default_rng(7)
    n = 1 << 24
    mag = (10.0 ** rng.uniform(-8, 7, n)).astype(np.float32)
    amp = (10.0 ** rng.uniform(-8, 7, n)).astype(np.float32)
    amp[rng.random(n) < 0.05] = 0.0
    den = (mag + np.float32(1e-12)).astype(np.float32)
    for num in (amp, mag):  # target = A on usable pixels, |y| on masked ones
        q = _divide(harness, num, den)
        exact = num / den
        assert np.all(np.isfinite(q))
        assert int(_ulps(q, exact).max()) <= 1
        assert float(np.mean(q != exact)) < 1e-4


def test_divide_edge_operands(gpu, harness):
    den = np.array([1e-12, 1e-12, 1.0, 3.0, 7.0, 1e7, 16777215.0, 1.9999999], np.float32)
    num = np.array([0.0, 1e6, 1.0, 1.0, 21.0, 1e7, 16777215.0, 1.0], np.float32)
    q = _divide(harness, num, den)
    exact = num / den
    assert int(_ulps(q, exact).max()) <= 1
    assert q[0] == 0.0 and q[2] == 1.0 and q[4] == 3.0 and q[5] == 1.0 and q[6] == 1.0


def test_square_root_matches_ieee_sqrt(gpu, harness):
    rng = np.random.default_rng(11)
    n = 1 << 24
    re = (10.0 ** rng.uniform(-8, 7, n) * rng.choice([-1.0, 1.0], n)).astype(np.float32)
    im = (10.0 ** rng.uniform(-8, 7, n) * rng.choice([-1.0, 1.0], n)).astype(np.float32)
    x = (re * re + im * im).astype(np.float32)
    x = x[np.isfinite(x)]
    q = _divide(harness, x)
    exact = np.sqrt(x)
    assert int(_ulps(q, exact).max()) <= 1
    assert float(np.mean(q != exact)) < 1e-4


def test_square_root_edge_operands(gpu, harness):
    x = np.array([0.0, 1e-45, 1e-40, 1.1754942e-38, 1e-30, 2.0**-64, 2.0**-65, 1.0, 4.0, 2.0,
                  16777216.0, 3.4e38], np.float32)
    q = _divide(harness, x)
    exact = np.sqrt(x)
    assert int(_ulps(q, exact).max()) <= 1
    assert q[0] == 0.0 and q[7] == 1.0 and q[8] == 2.0 and q[10] == 4096.0
