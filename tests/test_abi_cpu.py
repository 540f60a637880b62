"""The C ABI library without a GPU: it loads, exports every function include/bfvm.h declares, and
fails with a status (never a crash) when no device is present."""

import ctypes
import subprocess

import pytest

from parabiofvm_b200 import _abi


def test_library_exports_every_declared_function():
    lib = _abi.load()
    declared = _abi.header_functions()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, f"declared in include/bfvm.h but not exported: {missing}"
    # and the ctypes table covers the header exactly
    assert sorted(_abi.SIGNATURES) == declared


def test_exports_are_plain_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in _abi.header_functions():
        assert name in syms, name


def test_status_strings_and_version():
    lib = _abi.load()
    assert lib.bfvm_status_string(0) == b"ok"
    assert lib.bfvm_status_string(6) == b"agent outside the mesh"
    assert lib.bfvm_version() >= 10000


def test_create_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _abi.load()
    h = ctypes.c_void_p()
    i3 = (ctypes.c_int32 * 3)
    D = (ctypes.c_float * 1)(1.0)
    st = lib.bfvm_create(ctypes.byref(h), 0, 3, i3(0, 0, 0), i3(100, 100, 100), i3(20, 20, 20), 1, 0.01, D, D, 0)
    assert st == 4  # BFVM_ERR_NO_DEVICE
    assert h.value is None
    assert b"device" in lib.bfvm_last_error()


def test_invalid_mesh_rejected_before_device_lookup():
    lib = _abi.load()
    h = ctypes.c_void_p()
    i3 = (ctypes.c_int32 * 3)
    D = (ctypes.c_float * 1)(1.0)
    assert lib.bfvm_create(ctypes.byref(h), 0, 5, i3(0, 0, 0), i3(100, 100, 100), i3(20, 20, 20), 1, 0.01, D, D, 0) == 1
    assert lib.bfvm_create(ctypes.byref(h), 0, 3, i3(0, 0, 0), i3(100, 100, 100), i3(20, 0, 20), 1, 0.01, D, D, 0) == 1
    assert lib.bfvm_create(ctypes.byref(h), 0, 3, i3(0, 0, 0), i3(100000, 100, 100), i3(20, 20, 20), 1, 0.01, D, D,
                           0) == 1
    assert lib.bfvm_destroy(None) == 0
