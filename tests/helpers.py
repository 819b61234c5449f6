"""Shared helpers of the test suite: initial states in the reference layout and error norms."""

from __future__ import annotations

import numpy as np

from mhd_gpu_solver_b200 import workloads as wl
from mhd_gpu_solver_b200.accuracy import component_l1
from oracle import oracle as orc


def initial_state(prim: dict, gamma: float, bc=(orc.PERIODIC, orc.PERIODIC), mask=None,
                  walls: bool = True, ng: int = 2) -> np.ndarray:
    """Ghosted state as MHDSolver.set_primitives leaves it: to_conservative on the interior,
    ghost fill, then the wall fill when a mask with solid cells is set
    (include/mhd/solver_api.hpp:243-274 of the reference)."""
    ny, nx = prim["rho"].shape
    U = wl.embed(wl.to_conservative(prim, gamma), ng)
    grid = orc.Grid(nx, ny, ng)
    U = orc.apply_bc(U, grid, bc)
    if mask is not None and walls and not np.all(mask != 0):
        U = orc.wall_fill(U, grid, mask, gamma)
    return U


def interior(U: np.ndarray, ng: int = 2) -> np.ndarray:
    return U[:, ng:U.shape[1] - ng, ng:U.shape[2] - ng]


def rel_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-component relative L1 of a vs b over the interior (absolute where b is all zero)."""
    ai, bi = interior(a), interior(b)
    num = np.abs(ai - bi).reshape(9, -1).sum(axis=1)
    den = np.abs(bi).reshape(9, -1).sum(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


def signal_speed(U: np.ndarray, gamma: float = 5.0 / 3.0, ng: int = 2) -> float:
    """Maximum signal speed of a state (the GLM speed c_h its next step would take)."""
    ny, nx = U.shape[1] - 2 * ng, U.shape[2] - 2 * ng
    return orc.cfl(U, orc.Grid(nx, ny, ng), orc.Params(gamma=gamma))[1]


def component_errors(a: np.ndarray, b: np.ndarray, c_h: float | None = None,
                     gamma: float = 5.0 / 3.0, vector_scale: bool = False) -> np.ndarray:
    """Per-component L1 error of a against b over the interior, every component held
    (mhd_gpu_solver_b200.accuracy.component_l1: relative L1, absolute where b is identically
    zero, psi on the scale max(sum|psi|, c_h sum|B|); with vector_scale the components of m and B
    on their vector's scale). c_h defaults to the maximum signal speed of b (the speed of its
    next step)."""
    if c_h is None:
        c_h = signal_speed(b, gamma)
    return component_l1(a, b, c_h, vector_scale=vector_scale)


FP32_MIXED_BAR = 1e-6


def assert_components(a: np.ndarray, b: np.ndarray, tol: float, c_h: float | None = None,
                      gamma: float = 5.0 / 3.0, what=None) -> np.ndarray:
    """component_errors(a, b) <= tol for all nine components; returns the errors. The FP32-mixed
    bar (tol >= FP32_MIXED_BAR) holds the components of m and B on their vector's scale (see
    mhd_gpu_solver_b200.accuracy); tighter bars (FP64) hold every component on its own."""
    err = component_errors(a, b, c_h, gamma, vector_scale=tol >= FP32_MIXED_BAR)
    assert np.all(err <= tol), (what, err)
    return err


def rel_linf(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ai, bi = interior(a), interior(b)
    num = np.abs(ai - bi).reshape(9, -1).max(axis=1)
    den = np.abs(bi).reshape(9, -1).max(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)
