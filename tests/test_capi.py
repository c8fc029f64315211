"""The C-ABI library loads and exports every symbol include/qpb.h declares, and
its host-side validation answers without a GPU (no compute call is made)."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from qoraphasecu_b200 import _lib
import qoraphasecu_b200 as qpc

HEADER = Path(__file__).resolve().parent.parent / "include" / "qpb.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(qpb_[a-z_]+)\s*\(", text)) - {"qpb_progress_fn"})


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.EXPORTS)


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors have the C compiler's sizes and field offsets."""
    structs = {"qpb_problem": _lib.Problem, "qpb_options": _lib.Options, "qpb_op": _lib.Op}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    import subprocess

    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        cname, field, value = line.split()
        py = structs[cname]
        expect = ctypes.sizeof(py) if field == "size" else getattr(py, field).offset
        assert int(value) == expect, line


def test_last_error_starts_empty():
    assert _lib.load().qpb_last_error() in (b"",)


def test_create_validates_before_touching_a_device():
    lib = _lib.load()
    amp = np.ones((8, 8), np.float32)
    sup = np.ones((8, 8), np.uint8)
    p = qpc.api.Problem(amp, np.zeros((8, 8), np.uint8), sup)
    handle = ctypes.c_void_p()
    for field, value, message in (("starts", 0, "starts must be >= 1"),
                                  ("sync_every", 0, "sync_every must be >= 1"),
                                  ("batch", 3, "batch must divide starts")):
        o = _lib.Options(starts=4, batch=0, seed=0, start=None, sync_every=10, variant=0,
                         amp_storage=0, device=-1, stream=None)
        setattr(o, field, value)
        status = lib.qpb_create(ctypes.byref(p._c()), ctypes.byref(o), ctypes.byref(handle))
        assert status == _lib.INVALID_ARGUMENT
        assert message in lib.qpb_last_error().decode()
        with pytest.raises(ValueError):
            _lib.check(status)


def test_create_batch_validates_before_touching_a_device():
    lib = _lib.load()
    amp = np.ones((8, 8), np.float32)
    sup = np.ones((8, 8), np.uint8)
    p = qpc.api.Problem(amp, np.zeros((8, 8), np.uint8), sup)
    views = (_lib.Problem * 2)(p._c(), p._c())
    handle = ctypes.c_void_p()
    o = _lib.Options(starts=2, batch=0, seed=0, start=None, sync_every=10, variant=0,
                     amp_storage=0, device=-1, stream=None, schedule=0)
    assert lib.qpb_create_batch(views, 0, ctypes.byref(o), ctypes.byref(handle)) == \
        _lib.INVALID_ARGUMENT
    assert "no problems" in lib.qpb_last_error().decode()
    o.schedule = 7
    assert lib.qpb_create_batch(views, 2, ctypes.byref(o), ctypes.byref(handle)) == \
        _lib.INVALID_ARGUMENT
    assert "unknown schedule" in lib.qpb_last_error().decode()
    o.schedule = 0
    views[1].ndim = 4
    assert lib.qpb_create_batch(views, 2, ctypes.byref(o), ctypes.byref(handle)) == \
        _lib.INVALID_ARGUMENT
    assert handle.value is None


def test_metrics_validate_before_touching_a_device():
    lib = _lib.load()
    a = np.zeros((4, 4), np.complex64)
    out = np.zeros(1, np.float32)
    shape = _lib.shape_arg((4, 4))
    assert lib.qpb_aligned_error(_lib.ptr(a), None, 2, shape, 1, _lib.ptr(out)) == \
        _lib.INVALID_ARGUMENT
    assert lib.qpb_aligned_error(_lib.ptr(a), _lib.ptr(a), 4, shape, 1, _lib.ptr(out)) == \
        _lib.INVALID_ARGUMENT
    assert lib.qpb_aligned_error(_lib.ptr(a), _lib.ptr(a), 2, shape, 0, _lib.ptr(out)) == \
        _lib.INVALID_ARGUMENT
    assert lib.qpb_simulate_intensity(_lib.ptr(a), 1, shape, _lib.ptr(out)) == \
        _lib.INVALID_ARGUMENT
    with pytest.raises(ValueError, match="shapes differ"):
        qpc.aligned_error(a, np.zeros((4, 5), np.complex64))


def test_support_bound_projection_validates_before_touching_a_device():
    lib = _lib.load()
    x = np.zeros(8, np.complex64)
    s = np.ones(8, np.uint8)
    args = (_lib.ptr(s),)
    assert lib.qpb_project_support_bound(8, 1, *args, 0.0, _lib.ptr(x), None) == _lib.INVALID_ARGUMENT
    assert lib.qpb_project_support_bound(8, 1, *args, float("nan"), _lib.ptr(x), None) == \
        _lib.INVALID_ARGUMENT
    assert lib.qpb_project_support_bound(0, 1, *args, 1.0, _lib.ptr(x), None) == _lib.INVALID_ARGUMENT
    assert lib.qpb_project_support_bound(8, 0, *args, 1.0, _lib.ptr(x), None) == _lib.INVALID_ARGUMENT
    assert lib.qpb_project_support_bound(8, 1, None, 1.0, _lib.ptr(x), None) == _lib.INVALID_ARGUMENT
    misaligned = x.view(np.uint8)[4:].ctypes.data
    assert lib.qpb_project_support_bound(4, 1, *args, 1.0, misaligned, None) == \
        _lib.INVALID_ARGUMENT


def test_run_rejects_null_solver_and_bad_recipes():
    lib = _lib.load()
    ops = (_lib.Op * 1)(_lib.Op(0, 0, 0, 0, 0, 0, 0))
    assert lib.qpb_run(None, ops, 1) == _lib.INVALID_ARGUMENT


def test_no_device_is_a_runtime_error_not_a_fallback():
    if qpc.cuda_available():
        pytest.skip("a device is present")
    with pytest.raises(RuntimeError):
        qpc.make_problem(np.ones((8, 8), np.float32))
