"""Invariants on the GPU, every precision form and every kernel configuration: a uniform state
stays uniform bit for bit (the face fluxes cancel exactly; the FP32-mixed state holds the
uploaded values to its 48 bits), and a periodic solve conserves its totals of mass, momentum,
energy and B (each face flux is evaluated once and enters both of its cells), as the reference's
operator and integrator tests require (tests/test_mhd_operator.cpp:111-159,
tests/test_time_integrator.cpp:69-129)."""

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200 import workloads as wl
from tests.helpers import initial_state, interior

pytestmark = pytest.mark.gpu

NI = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2, eta_ambipolar=1e-3)


def run(U0, n, precision, config, steps, **kw):
    dev = _capi.DeviceSolver(n, n, precision=precision)
    try:
        dev.set_tile_config(config)
        dev.configure(0, 0)
        dev.upload(U0)
        r = dev.solve_steps(_capi.make_params(limiter=_capi.VANLEER, **kw), steps)
        return dev.download(), r
    finally:
        dev.close()


@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
def test_uniform_state_stays_uniform(precision):
    n = 60
    prim = {k: np.full((n, n), v) for k, v in dict(rho=1.3, vx=0.4, vy=-0.2, vz=0.1, p=0.8,
                                                   bx=0.7, by=-0.3, bz=0.2, psi=0.0).items()}
    U0 = initial_state(prim, 5.0 / 3.0)
    start = interior(U0).reshape(9, -1)[:, 0]
    tol = 0.0 if precision == _capi.FP64 else 2.0 ** -46
    for cfg in _capi.tile_configs(precision):
        for kw in ({}, NI):
            out, r = run(U0, n, precision, cfg["config"], 10, **kw)
            assert r.steps == 10
            cells = interior(out).reshape(9, -1)
            assert np.all(cells == cells[:, :1]), (cfg, kw)  # every cell alike, bit for bit
            assert np.all(np.abs(cells[:, 0] - start) <= tol * np.abs(start)), (cfg, kw)


@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
def test_periodic_solve_conserves_totals(precision):
    n = 64
    U0 = initial_state(wl.fourier_state(n, n, 8), 5.0 / 3.0)
    a = interior(U0).reshape(9, -1).sum(axis=1)
    # components that start at zero (vz, Bz) are held to the scale of one unit per cell
    scale = np.maximum(np.abs(interior(U0)).reshape(9, -1).sum(axis=1), float(n * n))
    tol = 1e-12 if precision == _capi.FP64 else 1e-9
    for cfg in _capi.tile_configs(precision):
        for kw in ({}, NI):
            out, _ = run(U0, n, precision, cfg["config"], 20, **kw)
            b = interior(out).reshape(9, -1).sum(axis=1)
            assert np.all(np.abs(b - a)[:8] <= tol * scale[:8]), (cfg, kw, (b - a)[:8] / scale[:8])
