"""GPU-side helpers of the test suite: run the CUDA backend through the C ABI on a state built
for the oracle."""

from __future__ import annotations

import numpy as np

from mhd_gpu_solver_b200 import _capi
from oracle import oracle as orc


def to_c_params(p: orc.Params) -> _capi.Params:
    return _capi.make_params(t_end=p.t_end, cfl=p.cfl, gamma=p.gamma, glm_alpha=p.glm_alpha,
                             limiter=p.limiter, ohmic=p.ohmic, hall=p.hall, ambipolar=p.ambipolar,
                             eta_ohm=p.eta_ohm, eta_hall=p.eta_hall,
                             eta_ambipolar=p.eta_ambipolar, max_steps=p.max_steps)


def gpu_solve(U0: np.ndarray, grid: orc.Grid, p: orc.Params, bc=(orc.PERIODIC, orc.PERIODIC),
              mask=None, walls: bool = True, precision: int = _capi.FP64, tile_config: int = -1):
    dev = _capi.DeviceSolver(grid.nx, grid.ny, grid.x_min, grid.x_max, grid.y_min, grid.y_max,
                             grid.ng, precision)
    try:
        dev.set_tile_config(tile_config)
        dev.configure(bc[0], bc[1], mask, walls)
        dev.upload(np.ascontiguousarray(U0))
        cp = to_c_params(p)
        r = dev.solve_steps(cp, p.max_steps) if p.fixed_steps else dev.solve(cp)
        out = dev.download()
        return out, r.t, r.steps, r.c_h
    finally:
        dev.close()
