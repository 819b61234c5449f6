"""Seeded synthetic initial states and masks (host side, numpy, FP64).

Every generator returns interior primitive arrays of shape (ny, nx) as a dict with keys
rho, vx, vy, vz, p, bx, by, bz, psi (the argument order of MHDSolver.set_primitives), evaluated
at cell centres x_i = x_min + (i + 1/2) dx (Grid2D::get_x, include/grid/grid.hpp:185-193 of the
reference). Random draws use numpy's PCG64 generator, whose streams are stable across numpy
versions.

* four_quadrant: piecewise-constant quadrants split at x = y = 0.5 (the 128^2 outflow case).
* fourier_state: smooth periodic field from random Fourier modes with integer wavevectors,
  1 <= |k| <= 8, amplitude |k|^-2, uniform phases; v scaled to rms 1, B = curl(A_z) scaled to
  rms 1 (div B = 0 in the continuum), rho = 1 + clip(0.2 f1), p = 1 + clip(0.1 f2) with the
  perturbations clipped to [-0.2, 0.2].
* circles_and_rectangles: uint8 fluid mask (1 = fluid) of 12 circles with radius U[0.02, 0.08]
  and 6 axis-aligned rectangles, rasterised at cell centres with inclusive tests, later shapes
  painting over earlier ones (the rule of the reference GUI's rasteriser, gui/geometry.py:22-38,
  130-156).
* orszag_tang, sod, brio_wu, ohmic_sine_bz: the named presets of the reference
  (include/initial_condition/inititial_condition.hpp:56-101; tests/test_regression_golden.cpp:
  82-101) used by the parity tests.
"""

from __future__ import annotations

import math

import numpy as np

FIELDS = ("rho", "vx", "vy", "vz", "p", "bx", "by", "bz", "psi")


def cell_centers(nx: int, ny: int, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0):
    dx = (x_max - x_min) / nx
    dy = (y_max - y_min) / ny
    xs = x_min + (np.arange(nx, dtype=np.float64) + 0.5) * dx
    ys = y_min + (np.arange(ny, dtype=np.float64) + 0.5) * dy
    return xs, ys


def _empty(nx: int, ny: int) -> dict:
    return {k: np.zeros((ny, nx), dtype=np.float64) for k in FIELDS}


def four_quadrant(nx: int, ny: int, seed: int = 0) -> dict:
    """rho, p ~ U[0.1, 2]; vx, vy ~ U[-1, 1]; By ~ U[-1, 1]; Bx = 0.75; vz = Bz = psi = 0.
    Quadrants are drawn in the order (x<0.5,y<0.5), (x>=0.5,y<0.5), (x<0.5,y>=0.5),
    (x>=0.5,y>=0.5), five draws each in the order rho, p, vx, vy, By."""
    rng = np.random.Generator(np.random.PCG64(seed))
    xs, ys = cell_centers(nx, ny)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    out = _empty(nx, ny)
    out["bx"][:] = 0.75
    quads = [(X < 0.5) & (Y < 0.5), (X >= 0.5) & (Y < 0.5), (X < 0.5) & (Y >= 0.5),
             (X >= 0.5) & (Y >= 0.5)]
    for q in quads:
        rho = rng.uniform(0.1, 2.0)
        p = rng.uniform(0.1, 2.0)
        vx = rng.uniform(-1.0, 1.0)
        vy = rng.uniform(-1.0, 1.0)
        by = rng.uniform(-1.0, 1.0)
        out["rho"][q] = rho
        out["p"][q] = p
        out["vx"][q] = vx
        out["vy"][q] = vy
        out["by"][q] = by
    return out


def _modes(kmax: int = 8):
    """Half-plane integer wavevectors with 1 <= |k| <= kmax (kx > 0, or kx == 0 and ky > 0)."""
    ks = []
    for kx in range(0, kmax + 1):
        for ky in range(-kmax, kmax + 1):
            if kx == 0 and ky <= 0:
                continue
            kk = math.hypot(kx, ky)
            if 1.0 <= kk <= kmax:
                ks.append((kx, ky, kk))
    return ks


def _synth(coef: np.ndarray, ex: np.ndarray, ey: np.ndarray) -> np.ndarray:
    """Re(sum_k coef[ky, kx] exp(i 2 pi (kx x + ky y))) on the cell-centre grid."""
    return np.real(ey.T @ coef @ ex)


def fourier_coefficients(seed: int = 0, kmax: int = 8) -> np.ndarray:
    """The five seeded spectra (vx, vy, A_z, f1, f2) of fourier_state as a complex array of shape
    (5, 2 kmax + 1, kmax + 1), row ky + kmax, column kx: the input of the device generator."""
    rng = np.random.Generator(np.random.PCG64(seed))
    modes = _modes(kmax)
    out = np.zeros((5, 2 * kmax + 1, kmax + 1), dtype=np.complex128)
    for q in range(5):
        phases = rng.uniform(0.0, 2.0 * np.pi, size=len(modes))
        for (kx, ky, kk), ph in zip(modes, phases):
            out[q, ky + kmax, kx] = kk ** -2.0 * np.exp(1j * ph)
    return out


def quadrant_values(seed: int = 0) -> np.ndarray:
    """(4, 5) array of (rho, p, vx, vy, By) per quadrant as four_quadrant draws them."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.array([[rng.uniform(0.1, 2.0), rng.uniform(0.1, 2.0), rng.uniform(-1.0, 1.0),
                      rng.uniform(-1.0, 1.0), rng.uniform(-1.0, 1.0)] for _ in range(4)])


def fourier_state(nx: int, ny: int, seed: int = 0, kmax: int = 8, x_min=0.0, x_max=1.0,
                  y_min=0.0, y_max=1.0) -> dict:
    rng = np.random.Generator(np.random.PCG64(seed))
    modes = _modes(kmax)
    xs, ys = cell_centers(nx, ny, x_min, x_max, y_min, y_max)
    lx, ly = x_max - x_min, y_max - y_min
    kxs = np.arange(0, kmax + 1)
    kys = np.arange(-kmax, kmax + 1)
    ex = np.exp(2j * np.pi * np.outer(kxs, (xs - x_min) / lx))      # (kmax+1, nx)
    ey = np.exp(2j * np.pi * np.outer(kys, (ys - y_min) / ly))      # (2kmax+1, ny)

    def coefficients():
        phases = rng.uniform(0.0, 2.0 * np.pi, size=len(modes))
        c = np.zeros((len(kys), len(kxs)), dtype=np.complex128)
        for (kx, ky, kk), ph in zip(modes, phases):
            c[ky + kmax, kx] = kk ** -2.0 * np.exp(1j * ph)
        return c

    cvx, cvy, caz, cf1, cf2 = (coefficients() for _ in range(5))
    vx = _synth(cvx, ex, ey)
    vy = _synth(cvy, ex, ey)
    vs = 1.0 / math.sqrt(float(np.mean(vx * vx + vy * vy)))
    vx *= vs
    vy *= vs
    # B = curl(A_z z^): Bx = dA/dy, By = -dA/dx (analytic derivatives of the modes).
    KX = (2j * np.pi / lx) * kxs[None, :]
    KY = (2j * np.pi / ly) * kys[:, None]
    bx = _synth(caz * KY, ex, ey)
    by = -_synth(caz * KX, ex, ey)
    bs = 1.0 / math.sqrt(float(np.mean(bx * bx + by * by)))
    bx *= bs
    by *= bs
    f1 = _synth(cf1, ex, ey)
    f2 = _synth(cf2, ex, ey)
    f1 /= math.sqrt(float(np.mean(f1 * f1)))
    f2 /= math.sqrt(float(np.mean(f2 * f2)))
    out = _empty(nx, ny)
    out["rho"] = 1.0 + np.clip(0.2 * f1, -0.2, 0.2)
    out["p"] = 1.0 + np.clip(0.1 * f2, -0.2, 0.2)
    out["vx"] = vx
    out["vy"] = vy
    out["bx"] = bx
    out["by"] = by
    return out


CIRCLE, RECTANGLE = 0, 1  # shape kinds of the C ABI (mhdb_shape)


def circles_and_rectangles_shapes(seed: int = 0, n_circles: int = 12,
                                  n_rects: int = 6) -> list[tuple]:
    """The seeded shapes of the masked workload as (kind, solid, a, b, c, d) tuples, painted in
    order: circles (centre (a, b) ~ U[0,1]^2, radius c ~ U[0.02, 0.08]), then rectangles (lower
    left corner (a, b) ~ U[0,1]^2, upper right corner (a + w, b + h), w and h ~ U[0.02, 0.15]),
    all solid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shapes = []
    for _ in range(n_circles):
        cx, cy = rng.uniform(0.0, 1.0, size=2)
        r = rng.uniform(0.02, 0.08)
        shapes.append((CIRCLE, 1, float(cx), float(cy), float(r), 0.0))
    for _ in range(n_rects):
        x0, y0 = rng.uniform(0.0, 1.0, size=2)
        w, h = rng.uniform(0.02, 0.15, size=2)
        shapes.append((RECTANGLE, 1, float(x0), float(y0), float(x0 + w), float(y0 + h)))
    return shapes


def rasterize(shapes, nx: int, ny: int, x_min=0.0, x_max=1.0, y_min=0.0,
              y_max=1.0) -> np.ndarray:
    """Interior fluid mask (ny, nx), 1 = fluid, by the rule of the reference's geometry helpers
    (gui/geometry.py:22-38, :130-156): all fluid, then each shape in order paints the cells whose
    centre it contains (inclusive tests), later shapes overwriting earlier ones."""
    xs, ys = cell_centers(nx, ny, x_min, x_max, y_min, y_max)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    mask = np.ones((ny, nx), dtype=np.uint8)
    for kind, solid, a, b, c, d in shapes:
        if kind == CIRCLE:
            hit = (X - a) ** 2 + (Y - b) ** 2 <= c * c
        else:
            xa, xb = sorted((a, c))
            ya, yb = sorted((b, d))
            hit = (X >= xa) & (X <= xb) & (Y >= ya) & (Y <= yb)
        mask[hit] = 0 if solid else 1
    return mask


def circles_and_rectangles(nx: int, ny: int, seed: int = 0, n_circles: int = 12,
                           n_rects: int = 6) -> np.ndarray:
    """Circles: centre ~ U[0,1]^2, radius ~ U[0.02, 0.08]; rectangles: lower-left corner
    ~ U[0,1]^2, width and height ~ U[0.02, 0.15]. Circles first, then rectangles."""
    return rasterize(circles_and_rectangles_shapes(seed, n_circles, n_rects), nx, ny)


def orszag_tang(nx: int, ny: int) -> dict:
    xs, ys = cell_centers(nx, ny)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    out = _empty(nx, ny)
    out["rho"][:] = 25.0 / (36.0 * np.pi)
    out["vx"] = -np.sin(2.0 * np.pi * Y)
    out["vy"] = np.sin(2.0 * np.pi * X)
    out["p"][:] = 5.0 / (12.0 * np.pi)
    out["bx"] = -np.sin(2.0 * np.pi * Y)
    out["by"] = np.sin(4.0 * np.pi * X)
    return out


def sod(nx: int, ny: int, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0) -> dict:
    xs, _ = cell_centers(nx, ny, x_min, x_max, y_min, y_max)
    X = np.broadcast_to(xs[None, :], (ny, nx))
    out = _empty(nx, ny)
    left = X < 0.5
    out["rho"] = np.where(left, 1.0, 0.125)
    out["p"] = np.where(left, 1.0, 0.1)
    return out


def brio_wu(nx: int, ny: int) -> dict:
    xs, _ = cell_centers(nx, ny)
    X = np.broadcast_to(xs[None, :], (ny, nx))
    out = _empty(nx, ny)
    left = X < 0.5
    out["bx"][:] = 0.75
    out["rho"] = np.where(left, 1.0, 0.125)
    out["p"] = np.where(left, 1.0, 0.1)
    out["by"] = np.where(left, 1.0, -1.0)
    return out


def ohmic_sine_bz(nx: int, ny: int) -> dict:
    xs, _ = cell_centers(nx, ny)
    X = np.broadcast_to(xs[None, :], (ny, nx))
    out = _empty(nx, ny)
    out["rho"][:] = 1.0
    out["p"][:] = 1.0
    out["bz"] = np.sin(2.0 * np.pi * X)
    return out


def to_conservative(prim: dict, gamma: float) -> np.ndarray:
    """include/mhd/mhd_physics.hpp:41-57, elementwise: returns (9, ny, nx)."""
    rho, vx, vy, vz = prim["rho"], prim["vx"], prim["vy"], prim["vz"]
    p, bx, by, bz, psi = prim["p"], prim["bx"], prim["by"], prim["bz"], prim["psi"]
    e_kin = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    e_mag = 0.5 * (bx * bx + by * by + bz * bz)
    E = p / (gamma - 1.0) + e_kin + e_mag
    return np.stack([rho, rho * vx, rho * vy, rho * vz, E, bx, by, bz, psi])


def embed(cons: np.ndarray, ng: int = 2) -> np.ndarray:
    """Interior (9, ny, nx) -> ghosted (9, ny + 2 ng, nx + 2 ng) with zero ghosts."""
    _, ny, nx = cons.shape
    out = np.zeros((9, ny + 2 * ng, nx + 2 * ng), dtype=np.float64)
    out[:, ng:ng + ny, ng:ng + nx] = cons
    return out
