"""C ABI checks that need no GPU: the library loads, exports every entry point declared in
include/mhd_b200.h, and reports a missing device through its status codes."""

import ctypes as C
import os
import re

import pytest

from mhd_gpu_solver_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    text = open(os.path.join(ROOT, "include", "mhd_b200.h")).read()
    return sorted(set(re.findall(r"\b(mhdb_[a-z_0-9]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_entry_points() == sorted(_capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_capi.LIB_PATH)
    for name in declared_entry_points():
        assert hasattr(lib, name), name


@pytest.mark.skipif(_capi.cuda_available(), reason="checks the no-device path")
def test_no_device_is_reported_not_faulted():
    g = _capi.Grid(8, 8, 2, 0.0, 1.0, 0.0, 1.0)
    h = C.c_void_p()
    assert _capi.lib.mhdb_create(C.byref(g), 0, C.byref(h)) == _capi.NO_DEVICE
    assert h.value is None
    assert b"no device" in _capi.lib.mhdb_last_error(None)
    with pytest.raises(RuntimeError, match="no device"):
        _capi.DeviceSolver(8, 8)


def test_argument_errors_before_any_device_work():
    h = C.c_void_p()
    g = _capi.Grid(8, 8, 1, 0.0, 1.0, 0.0, 1.0)
    assert _capi.lib.mhdb_create(C.byref(g), 0, C.byref(h)) == _capi.INVALID_ARGUMENT
    assert _capi.lib.mhdb_last_error(None) == b"CUDA solver requires grid.ng >= 2"
    g = _capi.Grid(0, 8, 2, 0.0, 1.0, 0.0, 1.0)
    assert _capi.lib.mhdb_create(C.byref(g), 0, C.byref(h)) == _capi.INVALID_ARGUMENT
    g = _capi.Grid(8, 8, 2, 0.0, 1.0, 0.0, 1.0)
    assert _capi.lib.mhdb_create(C.byref(g), 7, C.byref(h)) == _capi.INVALID_ARGUMENT
    assert _capi.lib.mhdb_create(None, 0, C.byref(h)) == _capi.INVALID_ARGUMENT
    # NULL handles are rejected, never dereferenced
    assert _capi.lib.mhdb_configure(None, 0, 0, None, 0, 1) == _capi.INVALID_ARGUMENT
    assert _capi.lib.mhdb_precision(None) == -1
    assert _capi.lib.mhdb_launch_count(None) == 0
    _capi.lib.mhdb_destroy(None)


def test_kernel_kind_names_match_the_header():
    """MHDB_KERNEL_* values in include/mhd_b200.h and the names the Python layer gives them."""
    import os
    import re

    from mhd_gpu_solver_b200 import _capi

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(root, "include", "mhd_b200.h")) as f:
        text = f.read()
    kinds = {int(v): k for k, v in re.findall(r"MHDB_KERNEL_(\w+) = (\d+)", text)}
    assert {v: n.lower() for v, n in kinds.items()} == _capi.KERNEL_KINDS
