"""Strip decomposition on the GPU (mhd_gpu_solver_b200/strips.py): a grid split into 2-3 strips,
each a solver on the same GPU with its own stream, stepped through the deferred C entry points
(mhdb_strip_*) with the combined CFL reduction and the overlap-row copies on the device. The
split result is held to the whole-grid solve on the GPU and to the FP64 oracle at the parity
tolerances (FP64 relative L1 1e-12, FP32-mixed 1e-6)."""

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi, strips
from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc

from gpu_util import gpu_solve, to_c_params
from helpers import initial_state, interior

pytestmark = pytest.mark.gpu

TOL = {_capi.FP64: 1e-12, _capi.FP32: 1e-6}
CORE = [0, 1, 2, 4, 5, 6]


def psi_l1(a: np.ndarray, b: np.ndarray, c_h: float) -> float:
    """L1 of the psi difference on psi's own scale in the GLM system, c_h |B|: psi starts at
    zero and its sources (c_h^2 div B, a cancellation of O(c_h^2 |B|) terms) leave it at the
    rounding level of that scale, so its relative L1 measures rounding, not agreement."""
    scale = c_h * np.abs(b[5:8]).sum()
    return float(np.abs(a[8] - b[8]).sum() / scale)


def check(got, want, c_h, precision):
    e = rel_l1(got, want)
    assert np.all(e[CORE] <= TOL[precision]), e
    for c in (3, 7):  # mz and bz stay zero in these 2D states: absolute L1
        assert e[c] <= TOL[precision], e
    assert psi_l1(got, want, c_h) <= TOL[precision], psi_l1(got, want, c_h)


def rel_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-component relative L1 of interior arrays (9, ny, nx)."""
    num = np.abs(a - b).reshape(9, -1).sum(axis=1)
    den = np.abs(b).reshape(9, -1).sum(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


def _case(nx, ny, bc, masked, ni, steps, limiter=orc.VANLEER, t_end=None):
    prim = wl.fourier_state(nx, ny, seed=2)
    mask = None
    if masked:
        mask = wl.circles_and_rectangles(nx, ny, seed=4, n_circles=4, n_rects=2).copy()
        if bc[1] == orc.PERIODIC:
            mask[:strips.SEAM_ROWS] = 1
            mask[-strips.SEAM_ROWS:] = 1
    kw = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2,
              eta_ambipolar=1e-3) if ni else {}
    if t_end is None:
        p = orc.Params(limiter=limiter, max_steps=steps, fixed_steps=True, **kw)
    else:
        p = orc.Params(t_end=t_end, limiter=limiter, **kw)
    U0 = initial_state(prim, p.gamma, bc, mask)
    return orc.Grid(nx, ny), p, U0, mask


def _split(grid, p, U0, bc, mask, count, precision, tile_config=-1):
    with strips.StripSolver(grid.nx, grid.ny, precision, strips=count, bc=bc, mask=mask,
                            tile_config=tile_config) as ss:
        ss.upload(U0)
        cp = to_c_params(p)
        res = ss.solve_steps(cp, p.max_steps) if p.fixed_steps else ss.solve(cp)
        return ss.gather(), res, ss.diagnostics(cp)


SMALL = [
    ("periodic", 64, 96, (orc.PERIODIC, orc.PERIODIC), False, False),
    ("masked_nonideal_outflow_x", 72, 90, (orc.OUTFLOW, orc.PERIODIC), True, True),
    ("masked_outflow", 60, 70, (orc.OUTFLOW, orc.OUTFLOW), True, False),
]


@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
@pytest.mark.parametrize("count", [2, 3])
@pytest.mark.parametrize("name,nx,ny,bc,masked,ni", SMALL, ids=[c[0] for c in SMALL])
def test_strips_match_oracle_and_whole_grid(name, nx, ny, bc, masked, ni, count, precision):
    grid, p, U0, mask = _case(nx, ny, bc, masked, ni, steps=12)
    got, res, _ = _split(grid, p, U0, bc, mask, count, precision)
    want, t, steps, c_h = orc.solve(U0, grid, p, bc, mask)
    assert res[1] == steps == 12
    check(got, interior(want), c_h, precision)
    whole, wt, wsteps, wc_h = gpu_solve(U0, grid, p, bc, mask, precision=precision)
    assert res[1] == wsteps
    check(got, interior(whole), c_h, precision)
    assert abs(res[0] - wt) <= 1e-12 * wt and abs(res[2] - wc_h) <= TOL[precision] * wc_h


@pytest.mark.parametrize("precision,tile_config", [(_capi.FP64, -1), (_capi.FP32, 13)])
def test_time_based_strips_stop_with_the_whole_grid(precision, tile_config):
    """Time-based strip solves (the host steps in batches and may launch steps past the end,
    which do nothing on the device), also on the increment form whose state buffers alternate."""
    bc = (orc.OUTFLOW, orc.OUTFLOW)
    grid, p, U0, mask = _case(48, 64, bc, True, False, steps=0, t_end=0.01)
    got, res, _ = _split(grid, p, U0, bc, mask, 2, precision, tile_config)
    want, t, steps, c_h = orc.solve(U0, grid, p, bc, mask)
    assert res[1] == steps and abs(res[0] - t) <= TOL[precision] * t
    check(got, interior(want), c_h, precision)


def test_strip_diagnostics_combine_to_the_whole_grid():
    bc = (orc.PERIODIC, orc.PERIODIC)
    grid, p, U0, mask = _case(64, 80, bc, False, False, steps=6)
    _, _, diag = _split(grid, p, U0, bc, mask, 2, _capi.FP64)
    dev = _capi.DeviceSolver(grid.nx, grid.ny, precision=_capi.FP64)
    try:
        dev.configure(bc[0], bc[1])
        dev.upload(np.ascontiguousarray(U0))
        cp = to_c_params(p)
        dev.solve_steps(cp, p.max_steps)
        want = dev.diagnostics(cp)
    finally:
        dev.close()
    for k in ("mass", "energy", "div_b_l2"):
        assert abs(diag[k] - want[k]) <= 1e-12 * abs(want[k]), k
    for k in ("div_b_max", "rho_min", "p_min"):
        assert abs(diag[k] - want[k]) <= 1e-12 * abs(want[k]), k
    assert diag["finite"] == want["finite"] is True


@pytest.mark.parametrize("precision,tile_config", [(_capi.FP64, 7), (_capi.FP32, 11),
                                                   (_capi.FP32, 13)])
def test_strips_on_the_strip_march(precision, tile_config):
    """Strips on the TMA strip march against the FP64 oracle and the whole grid."""
    n = 512
    bc = (orc.PERIODIC, orc.PERIODIC)
    grid, p, U0, mask = _case(n, n, bc, False, False, steps=20)
    got, res, _ = _split(grid, p, U0, bc, mask, 2, precision, tile_config)
    want, t, steps, c_h = orc.solve(U0, grid, p, bc, mask)
    whole, wt, wsteps, _ = gpu_solve(U0, grid, p, bc, mask, precision=precision,
                                     tile_config=tile_config)
    assert res[1] == wsteps == steps
    check(got, interior(want), c_h, precision)
    check(got, interior(whole), c_h, precision)
    print("psi on the c_h |B| scale: strips vs oracle", psi_l1(got, interior(want), c_h),
          "whole grid vs oracle", psi_l1(interior(whole), interior(want), c_h))


def test_strip_call_order_is_checked():
    dev = _capi.DeviceSolver(16, 16, precision=_capi.FP64)
    try:
        with pytest.raises(_capi.MhdbValueError):
            dev.strip_step()
        with pytest.raises(_capi.MhdbValueError):
            dev.set_reduce_rows(4, 4)
        with pytest.raises(_capi.MhdbValueError):
            dev.set_cell_size(0.0, 1.0)
        dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
        dev.upload(np.ascontiguousarray(initial_state(wl.four_quadrant(16, 16), 5.0 / 3.0)))
        cp = _capi.make_params(limiter=_capi.MC)
        dev.strip_begin(cp, 2)
        with pytest.raises(_capi.MhdbValueError):
            dev.strip_step()  # the reduction of begin awaits its finish
        dev.strip_finish()
        with pytest.raises(_capi.MhdbValueError):
            dev.strip_finish()
        for _ in range(2):
            dev.strip_step()
            dev.strip_finish()
        done, steps, _ = dev.strip_poll()
        assert done and steps == 2
        assert dev.strip_end().steps == 2
    finally:
        dev.close()
