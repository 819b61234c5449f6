"""The bounded bulk-copy waits of the TMA strip marches: a wait that runs out is reported, not
spun on, and leaves the device usable.

mhdb_debug_stall_copies arms the first row copy of the strip at the grid's origin for more
transaction bytes than its boxes deliver: a phase that nothing completes (the copies themselves
are well-formed and land). The kernel's wait gives up after its 0.5 s limit, records the timeout
in the Ctrl block, waits (bounded) for its copies in flight and stops; the solve then returns
MHDB_CUDA_ERROR with the single-solve message, as the reference maps CUDA failures to
std::runtime_error("CUDA: ...") (src/cuda/cuda_solver.cu:23-30). A batched solve reports the same
through mhdb_batch_status while the other solves of the batch finish with their own results, and
a fresh handle on the same context then runs clean against the oracle.
"""

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200 import workloads as wl
from mhd_gpu_solver_b200.batch import BatchSolver
from oracle import oracle as orc
from tests.helpers import assert_components, initial_state

pytestmark = pytest.mark.gpu

MESSAGE = "bulk-copy wait exceeded its limit"


@pytest.fixture(scope="module", autouse=True)
def _need_device():
    if not _capi.cuda_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")


def _config(precision, kind):
    return next(c["config"] for c in _capi.tile_configs(precision) if c["kind"] == kind)


@pytest.mark.parametrize("precision,kind", [(_capi.FP32, "march_tma_delta"),
                                            (_capi.FP32, "march_tma_pair"),
                                            (_capi.FP32, "march_tma"),
                                            (_capi.FP64, "march_tma")])
def test_single_solve_reports_a_wait_that_ran_out(precision, kind):
    n = 96
    U0 = initial_state(wl.fourier_state(n, n, 3), 5.0 / 3.0)
    cp = _capi.make_params(limiter=_capi.VANLEER)
    dev = _capi.DeviceSolver(n, n, precision=precision)
    try:
        dev.set_tile_config(_config(precision, kind))
        dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
        dev.upload(U0)
        dev.debug_stall_copies(16)
        with pytest.raises(RuntimeError, match=MESSAGE) as e:
            dev.solve_steps(cp, 4)
        assert e.value.code == _capi.CUDA_ERROR
        # the same handle, hook off, state re-uploaded: a clean solve
        dev.debug_stall_copies(0)
        dev.upload(U0)
        r = dev.solve_steps(cp, 4)
        again = dev.download()
    finally:
        dev.close()
    assert r.steps == 4
    p = orc.Params(limiter=orc.VANLEER, max_steps=4, fixed_steps=True)
    ref, _, steps, c_h = orc.solve(U0, orc.Grid(n, n), p)
    tol = 1e-12 if precision == _capi.FP64 else 1e-6
    assert_components(again, ref, tol, c_h)
    # a fresh handle on the same context
    dev = _capi.DeviceSolver(n, n, precision=precision)
    try:
        dev.set_tile_config(_config(precision, kind))
        dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
        dev.upload(U0)
        r = dev.solve_steps(cp, 4)
        fresh = dev.download()
    finally:
        dev.close()
    assert r.steps == steps and np.array_equal(fresh, again)


def test_batch_reports_a_wait_that_ran_out():
    """Three 128^2 solves on the increment-form TMA batch kernel, the second with the hook on.
    Each step launch has far more CTAs than work items (20 per solve), so every CTA runs one item
    and the stalled warp runs no item of another solve: the other two finish their 6 steps with
    the values they have alone (the persistent kernels are bit-identical alone and in a mix)."""
    n = 128
    states = [initial_state(wl.fourier_state(n, n, 20 + i), 5.0 / 3.0) for i in range(3)]

    def fixed():
        return _capi.make_params(limiter=_capi.VANLEER, max_steps=6)

    b = BatchSolver(_capi.FP32)
    try:
        ids = [b.add(U, fixed(), (orc.PERIODIC, orc.PERIODIC), fixed_steps=True) for U in states]
        b.debug_stall_copies(ids[1], 16)
        while b.step(6) > 0:
            pass
        with pytest.raises(RuntimeError, match=MESSAGE) as e:
            b.status(ids[1])
        assert e.value.code == _capi.CUDA_ERROR
        got = {}
        for i in (0, 2):
            r, fin = b.status(ids[i])
            assert fin and r.steps == 6
            got[i] = b.download(ids[i])
    finally:
        b.close()
    for i in (0, 2):
        alone = BatchSolver(_capi.FP32)
        try:
            sid = alone.add(states[i], fixed(), (orc.PERIODIC, orc.PERIODIC), fixed_steps=True)
            alone.step(6)
            assert np.array_equal(alone.download(sid), got[i])
        finally:
            alone.close()
