"""The allocation-free solve (mhdb_solve_steps_noalloc_f64) against the handle-based one.

Callers that cannot allocate device memory (code inside another framework's memory pool or
under a fixed budget) get a fixed-step FP64 solve whose scratch is a file-scope device array of
the library. This test calls it through the C ABI on two different solves in a row, so the
second call runs on scratch left over from the first, and compares each result with
mhdb_solve_steps on a handle (relative L1 <= 1e-12 per component, equal step count and time).
It also checks that a grid beyond the scratch limit is refused.
"""

import ctypes as C

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200 import workloads as wl
from mhd_gpu_solver_b200.mhd_solver import apply_boundary_conditions

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _state(nx, ny, bc, seed):
    U = wl.embed(wl.to_conservative(wl.fourier_state(nx, ny, seed), 5.0 / 3.0))
    apply_boundary_conditions(U, nx, ny, 2, bc[0], bc[1])
    return U


def _with_handle(U, nx, ny, bc, params, nsteps):
    dev = _capi.DeviceSolver(nx, ny)
    try:
        dev.configure(bc[0], bc[1])
        dev.upload(U)
        r = dev.solve_steps(params, nsteps)
        out = dev.download()
    finally:
        dev.close()
    return out[:, 2:-2, 2:-2], r


def _no_alloc(U, nx, ny, bc, params, nsteps, in_place):
    import torch

    interior = np.ascontiguousarray(U[:, 2:-2, 2:-2])
    u_in = torch.from_numpy(interior).cuda()
    u_out = u_in if in_place else torch.empty_like(u_in)
    torch.cuda.synchronize()
    g = _capi.Grid(nx, ny, 2, 0.0, 1.0, 0.0, 1.0)
    r = _capi.Result()
    rc = _capi.lib.mhdb_solve_steps_noalloc_f64(
        C.byref(g), bc[0], bc[1], C.byref(params), nsteps, C.c_void_p(u_in.data_ptr()),
        C.c_void_p(u_out.data_ptr()), C.byref(r), None)
    _capi.raise_for(rc, None)
    return u_out.cpu().numpy(), r


def _rel_l1(a, b):
    num = np.abs(a - b).reshape(9, -1).sum(axis=1)
    den = np.abs(b).reshape(9, -1).sum(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


def test_no_alloc_solve_matches_handle_solve_twice_in_a_row():
    if not _capi.cuda_available():
        pytest.fail("no CUDA device")
    cases = [
        # nx, ny, bc, params, steps, in_place
        (96, 80, (_capi.BC_PERIODIC, _capi.BC_PERIODIC),
         _capi.make_params(limiter=_capi.VANLEER), 25, False),
        (131, 67, (_capi.BC_OUTFLOW, _capi.BC_PERIODIC),
         _capi.make_params(limiter=_capi.MC, ohmic=True, hall=True, ambipolar=True,
                           eta_ohm=1e-3, eta_hall=1e-2, eta_ambipolar=1e-3), 17, True),
    ]
    for seed, (nx, ny, bc, params, steps, in_place) in enumerate(cases):
        U = _state(nx, ny, bc, seed)
        ref, r_ref = _with_handle(U, nx, ny, bc, params, steps)
        got, r = _no_alloc(U, nx, ny, bc, params, steps, in_place)
        assert r.steps == r_ref.steps == steps
        assert abs(r.t - r_ref.t) <= 1e-12 * r_ref.t
        assert abs(r.c_h - r_ref.c_h) <= 1e-12 * r_ref.c_h
        err = _rel_l1(got, ref)
        assert np.all(err <= TOL), err


def test_no_alloc_refuses_grids_beyond_its_scratch():
    g = _capi.Grid(1024, 1024, 2, 0.0, 1.0, 0.0, 1.0)
    r = _capi.Result()
    p = _capi.make_params()
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = _capi.lib.mhdb_solve_steps_noalloc_f64(C.byref(g), 0, 0, C.byref(p), 1, dummy, dummy,
                                                C.byref(r), None)
    assert rc == _capi.INVALID_ARGUMENT
    assert b"exceeds the 233016-cell limit" in _capi.lib.mhdb_last_error(None)


def test_no_alloc_refuses_partly_overlapping_state_buffers():
    """u_out must equal u_in or lie wholly apart from it. Both pointers here lie inside one
    allocation twice the state's size, so even an unchecked copy would stay in bounds."""
    import torch

    if not _capi.cuda_available():
        pytest.fail("no CUDA device")
    nx, ny = 40, 30
    buf = torch.zeros(2 * 9 * nx * ny, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    g = _capi.Grid(nx, ny, 2, 0.0, 1.0, 0.0, 1.0)
    r = _capi.Result()
    p = _capi.make_params()
    base = buf.data_ptr()
    rc = _capi.lib.mhdb_solve_steps_noalloc_f64(C.byref(g), 0, 0, C.byref(p), 1,
                                                C.c_void_p(base), C.c_void_p(base + 8 * nx),
                                                C.byref(r), None)
    assert rc == _capi.INVALID_ARGUMENT
    assert b"must equal u_in or not overlap it" in _capi.lib.mhdb_last_error(None)
