"""Python surface of the reference's ``mhd_solver`` module, backed by the B200 CUDA backend.

Names, arguments, defaults and exception types follow the reference pybind module
(python/mhd_pybind.cpp:166-309) and the MHDSolver class it wraps
(include/mhd/solver_api.hpp:22-452). Differences:

* The only execution backend is ``"cuda"`` (this package ships no CPU solver);
  ``set_backend("cpu")`` and ``set_backend("metal")`` raise RuntimeError("Backend not
  available: ..."), the reference's error for a backend that is not present.
* ``precision="fp32"`` selects the FP32-mixed form (FP32 arithmetic, compensated hi/lo state).
* ``SlopeLimiter.VanLeer`` and ``set_limiter_vanleer()`` are added.
* Additive calls: ``solve_steps(n)`` (exactly n steps), ``diagnostics()`` (FP64 on-device
  mass, energy, div-B max/L2, min rho/p, finiteness).
* The state stays resident on the GPU between runs. The host copy is downloaded only when it is
  read (``field``, ``max_div_b``, ...) and re-uploaded only after it was changed on the host, so
  a sequence of ``run`` calls moves no data; results are the same as uploading and downloading
  around every run, which is what the reference does.

Host-side state preparation (``set_primitives``, ``set_mask``, ``initialize``) is done on the
host with numpy, as the reference does it on the host: to_conservative, ghost fill and the
reflective wall fill.
"""

from __future__ import annotations

import enum

import numpy as np

from . import _capi
from . import workloads as _wl

_COMPONENTS = ("rho", "mx", "my", "mz", "energy", "bx", "by", "bz", "psi")

_thread_count = 0


def set_num_threads(n: int) -> None:
    """Accepted for compatibility; the CUDA backend uses no host worker threads."""
    global _thread_count
    _thread_count = max(0, int(n))


def num_threads() -> int:
    return 1


def set_simd_enabled(enabled: bool) -> None:
    """Accepted for compatibility; there are no host SIMD kernels in this package."""


def simd_enabled() -> bool:
    return False


def simd_backend() -> str:
    return "scalar"


def simd_width() -> int:
    return 1


def metal_available() -> bool:
    return False


def cuda_available() -> bool:
    return _capi.cuda_available()


def available_backends() -> list[str]:
    return ["cuda"] if cuda_available() else []


class SlopeLimiter(enum.IntEnum):
    Minmod = 0
    MC = 1
    VanLeer = 2


class BoundaryConditionType(enum.IntEnum):
    Periodic = 0
    Reflective = 1
    Outflow = 2


class NonIdealConfig:
    """include/physics_config/mhd_config.hpp:13-111."""

    def __init__(self):
        self.ohmic = False
        self.hall = False
        self.ambipolar = False
        self.eta_ohm = 0.0
        self.eta_hall = 0.0
        self.eta_ambipolar = 0.0

    @staticmethod
    def ideal() -> "NonIdealConfig":
        return NonIdealConfig()

    @staticmethod
    def with_ohmic(eta: float) -> "NonIdealConfig":
        return NonIdealConfig().enable_ohmic(eta)

    @staticmethod
    def with_hall(eta: float) -> "NonIdealConfig":
        return NonIdealConfig().enable_hall(eta)

    @staticmethod
    def with_ambipolar(eta: float) -> "NonIdealConfig":
        return NonIdealConfig().enable_ambipolar(eta)

    def enable_ohmic(self, eta: float) -> "NonIdealConfig":
        self.ohmic, self.eta_ohm = True, float(eta)
        return self

    def enable_hall(self, eta: float) -> "NonIdealConfig":
        self.hall, self.eta_hall = True, float(eta)
        return self

    def enable_ambipolar(self, eta: float) -> "NonIdealConfig":
        self.ambipolar, self.eta_ambipolar = True, float(eta)
        return self

    def disable_ohmic(self) -> "NonIdealConfig":
        self.ohmic = False
        return self

    def disable_hall(self) -> "NonIdealConfig":
        self.hall = False
        return self

    def disable_ambipolar(self) -> "NonIdealConfig":
        self.ambipolar = False
        return self

    def any(self) -> bool:
        return ((self.ohmic and self.eta_ohm != 0.0) or (self.hall and self.eta_hall != 0.0)
                or (self.ambipolar and self.eta_ambipolar != 0.0))

    def copy(self) -> "NonIdealConfig":
        c = NonIdealConfig()
        c.__dict__.update(self.__dict__)
        return c


class SolveParams:
    """include/mhd/solve_types.hpp:8-16 (same defaults)."""

    def __init__(self):
        self.t_end = 0.0
        self.cfl = 0.4
        self.gamma = 5.0 / 3.0
        self.glm_alpha = 0.1
        self.limiter = SlopeLimiter.MC
        self.nonideal = NonIdealConfig.ideal()
        self.max_steps = 1_000_000

    def to_c(self, t_end: float | None = None) -> _capi.Params:
        ni = self.nonideal
        return _capi.make_params(
            t_end=self.t_end if t_end is None else t_end, cfl=self.cfl, gamma=self.gamma,
            glm_alpha=self.glm_alpha, limiter=int(self.limiter), ohmic=ni.ohmic, hall=ni.hall,
            ambipolar=ni.ambipolar, eta_ohm=ni.eta_ohm, eta_hall=ni.eta_hall,
            eta_ambipolar=ni.eta_ambipolar, max_steps=self.max_steps)

    def copy(self) -> "SolveParams":
        p = SolveParams()
        p.__dict__.update(self.__dict__)
        p.nonideal = self.nonideal.copy()
        return p


class SolveResult:
    """include/mhd/solve_types.hpp:18-22."""

    def __init__(self, t: float = 0.0, steps: int = 0, c_h: float = 0.0):
        self._t, self._steps, self._c_h = float(t), int(steps), float(c_h)

    t = property(lambda self: self._t)
    steps = property(lambda self: self._steps)
    c_h = property(lambda self: self._c_h)

    def __repr__(self) -> str:
        return f"SolveResult(t={self._t!r}, steps={self._steps}, c_h={self._c_h!r})"


# ------------------------------------------------------------------ host-side state helpers


def _map_index(x: np.ndarray, n: int, bc: int) -> np.ndarray:
    """Boundary rule as an index map onto the interior
    (include/boundary_conditions/boundary_conditions.hpp:26-88)."""
    if bc == BoundaryConditionType.Periodic:
        return np.mod(x, n)
    return np.clip(x, 0, n - 1)


def apply_boundary_conditions(U: np.ndarray, nx: int, ny: int, ng: int, bc_x: int,
                              bc_y: int) -> None:
    """Ghost fill of a ghosted (9, ny+2ng, nx+2ng) state in place: x ghosts, then y ghosts over
    the full x range, which makes ghost (i, j) = interior (map_x(i), map_y(j))."""
    if bc_x == BoundaryConditionType.Reflective or bc_y == BoundaryConditionType.Reflective:
        raise ValueError("Reflective boundary conditions are not implemented yet")
    ix = _map_index(np.arange(nx + 2 * ng) - ng, nx, bc_x) + ng
    jy = _map_index(np.arange(ny + 2 * ng) - ng, ny, bc_y) + ng
    inner = U[:, ng:ng + ny, ng:ng + nx].copy()
    full = U[:, jy][:, :, ix]
    U[...] = full
    U[:, ng:ng + ny, ng:ng + nx] = inner


def apply_solid_wall_fill(U: np.ndarray, mask: np.ndarray, ng: int, gamma: float) -> None:
    """Reflective fill of solid interior cells in place (include/mhd/mask.hpp:85-149): first
    fluid interior neighbour in the order +x, -x, +y, -y; to_primitive with divisions, negate
    the normal velocity, floor rho and p at 1e-12, to_conservative; no fluid neighbour ->
    rho = p = 1 at rest. Vectorised over solid cells; the result does not depend on order
    because only fluid cells are read."""
    ny, nx = mask.shape
    solid = mask == 0
    if not solid.any():
        return
    jj, ii = np.nonzero(solid)
    done = np.zeros(jj.shape, dtype=bool)
    fluid = mask != 0
    inner = U[:, ng:ng + ny, ng:ng + nx]
    out = np.empty((9, jj.size), dtype=np.float64)
    for di, dj, axis in ((1, 0, 0), (-1, 0, 0), (0, 1, 1), (0, -1, 1)):
        ni, nj = ii + di, jj + dj
        ok = (~done) & (ni >= 0) & (ni < nx) & (nj >= 0) & (nj < ny)
        sel = np.nonzero(ok)[0]
        sel = sel[fluid[nj[sel], ni[sel]]]
        if sel.size == 0:
            continue
        s = inner[:, nj[sel], ni[sel]]
        rho, mx, my, mz, E, bx, by, bz, psi = s
        vx, vy, vz = mx / rho, my / rho, mz / rho
        e_kin = 0.5 * (mx * mx + my * my + mz * mz) / rho
        e_mag = 0.5 * (bx * bx + by * by + bz * bz)
        p = (gamma - 1.0) * (E - e_kin - e_mag)
        if axis == 0:
            vx = -vx
        else:
            vy = -vy
        r = np.where(rho < 1e-12, 1e-12, rho)
        p = np.where(p < 1e-12, 1e-12, p)
        ek = 0.5 * r * (vx * vx + vy * vy + vz * vz)
        em = 0.5 * (bx * bx + by * by + bz * bz)
        out[:, sel] = np.stack([r, r * vx, r * vy, r * vz, p / (gamma - 1.0) + ek + em, bx, by,
                                bz, psi])
        done[sel] = True
    rest = np.nonzero(~done)[0]
    if rest.size:
        out[:, rest] = 0.0
        out[0, rest] = 1.0
        out[4, rest] = 1.0 / (gamma - 1.0)
    inner[:, jj, ii] = out


def max_abs_div_b(U: np.ndarray, nx: int, ny: int, ng: int, dx: float, dy: float) -> float:
    """include/initial_condition/inititial_condition.hpp:273-287 on a ghosted host state."""
    bx, by = U[5], U[6]
    dbx = (bx[ng:ng + ny, ng + 1:ng + nx + 1] - bx[ng:ng + ny, ng - 1:ng + nx - 1]) * (0.5 / dx)
    dby = (by[ng + 1:ng + ny + 1, ng:ng + nx] - by[ng - 1:ng + ny - 1, ng:ng + nx]) * (0.5 / dy)
    return float(np.max(np.abs(dbx + dby)))


_PRESETS = {
    "uniform": "uniform", "Uniform": "uniform", "sine": "sine", "SineWave": "sine",
    "orszag_tang": "orszag_tang", "OrszagTang": "orszag_tang", "sod": "sod", "Sod": "sod",
    "brio_wu": "brio_wu", "BrioWu": "brio_wu",
}


class MHDSolver:
    """include/mhd/solver_api.hpp:22-452 with the CUDA backend selected."""

    def __init__(self, nx: int, ny: int, x_min: float = 0.0, x_max: float = 1.0,
                 y_min: float = 0.0, y_max: float = 1.0, ng: int = 2):
        if ng < 2:
            raise ValueError("MHDSolver requires ng >= 2")
        self._nx, self._ny, self._ng = int(nx), int(ny), int(ng)
        self._x_min, self._x_max = float(x_min), float(x_max)
        self._y_min, self._y_max = float(y_min), float(y_max)
        self._dx = (self._x_max - self._x_min) / self._nx
        self._dy = (self._y_max - self._y_min) / self._ny
        self._bc = (BoundaryConditionType.Periodic, BoundaryConditionType.Periodic)
        self._U = np.zeros((9, self._ny + 2 * ng, self._nx + 2 * ng), dtype=np.float64)
        self._mask = np.ones((self._ny, self._nx), dtype=np.uint8)
        self._params = SolveParams()
        self._t = 0.0
        self._steps = 0
        self._c_h = 0.0
        self._walls = True
        self._precision = _capi.FP64
        self._dev: _capi.DeviceSolver | None = None
        self._host_valid = True     # host copy holds the current state
        self._device_valid = False  # device copy holds the current state
        self._configured = None

    # ---- configuration (solver_api.hpp:80-145)
    def set_periodic_bc(self):
        self._sync_host()
        self._bc = (BoundaryConditionType.Periodic, BoundaryConditionType.Periodic)

    def set_outflow_bc(self):
        self._sync_host()
        self._bc = (BoundaryConditionType.Outflow, BoundaryConditionType.Outflow)

    def set_bc(self, type_x, type_y):
        self._sync_host()
        self._bc = (BoundaryConditionType(int(type_x)), BoundaryConditionType(int(type_y)))

    def set_gamma(self, gamma: float):
        self._params.gamma = float(gamma)

    def set_cfl(self, cfl: float):
        self._params.cfl = float(cfl)

    def set_glm_alpha(self, alpha: float):
        self._params.glm_alpha = float(alpha)

    def set_limiter_minmod(self):
        self._params.limiter = SlopeLimiter.Minmod

    def set_limiter_mc(self):
        self._params.limiter = SlopeLimiter.MC

    def set_limiter_vanleer(self):
        self._params.limiter = SlopeLimiter.VanLeer

    def set_ideal(self):
        self._params.nonideal = NonIdealConfig.ideal()

    def enable_ohmic(self, eta: float):
        self._params.nonideal.enable_ohmic(eta)

    def enable_hall(self, eta: float):
        self._params.nonideal.enable_hall(eta)

    def enable_ambipolar(self, eta: float):
        self._params.nonideal.enable_ambipolar(eta)

    def disable_ohmic(self):
        self._params.nonideal.disable_ohmic()

    def disable_hall(self):
        self._params.nonideal.disable_hall()

    def disable_ambipolar(self):
        self._params.nonideal.disable_ambipolar()

    # ---- mask (solver_api.hpp:148-154)
    def set_mask(self, mask):
        m = np.asarray(mask)
        if m.ndim != 2:
            raise ValueError("set_mask expects a 2D array (ny, nx)")
        if m.shape != (self._ny, self._nx):
            raise ValueError("set_mask shape must be (ny, nx)")
        self._sync_host()
        self._mask = np.ascontiguousarray(m, dtype=np.uint8).copy()
        if self._walls:
            apply_solid_wall_fill(self._U, self._mask, self._ng, self._params.gamma)
        self._host_changed()

    def get_mask(self) -> np.ndarray:
        return self._mask.copy()

    def clear_mask(self):
        self._sync_host()
        self._mask = np.ones((self._ny, self._nx), dtype=np.uint8)
        self._host_changed()

    def set_walls_reflective(self, enabled: bool):
        self._sync_host()
        self._walls = bool(enabled)
        self._host_changed()

    @property
    def walls_reflective(self) -> bool:
        return self._walls

    # ---- state (solver_api.hpp:211-292)
    def set_field(self, name: str, array):
        a = np.asarray(array, dtype=np.float64)
        if a.ndim != 2:
            raise ValueError("set_field expects a 2D array")
        c = self._component(name)
        self._sync_host()
        if a.shape == (self.size_y, self.size_x):
            self._U[c] = a
        elif a.shape == (self._ny, self._nx):
            ng = self._ng
            self._U[c, ng:ng + self._ny, ng:ng + self._nx] = a
        else:
            raise ValueError("set_field shape must be full (size_y, size_x) or interior (ny, nx)")
        self._host_changed()

    def set_primitives(self, rho, vx, vy, vz, pressure, bx, by, bz, psi=None):
        arrs = {}
        for label, a in (("rho", rho), ("vx", vx), ("vy", vy), ("vz", vz), ("pressure", pressure),
                         ("bx", bx), ("by", by), ("bz", bz)):
            a = np.asarray(a, dtype=np.float64)
            if a.ndim != 2:
                raise ValueError(f"{label} must be 2D")
            arrs[label] = a
        if arrs["rho"].shape != (self._ny, self._nx):
            raise ValueError("primitive arrays must have shape (ny, nx)")
        for a in arrs.values():
            if a.shape != arrs["rho"].shape:
                raise ValueError("primitive arrays must share the same shape")
        if psi is None:
            psi_a = np.zeros((self._ny, self._nx))
        else:
            psi_a = np.asarray(psi, dtype=np.float64)
            if psi_a.ndim != 2:
                raise ValueError("psi must be 2D")
            if psi_a.shape != arrs["rho"].shape:
                raise ValueError("primitive arrays must share the same shape")
        self._sync_host()
        prim = {"rho": arrs["rho"], "vx": arrs["vx"], "vy": arrs["vy"], "vz": arrs["vz"],
                "p": arrs["pressure"], "bx": arrs["bx"], "by": arrs["by"], "bz": arrs["bz"],
                "psi": psi_a}
        ng = self._ng
        self._U[:, ng:ng + self._ny, ng:ng + self._nx] = _wl.to_conservative(
            prim, self._params.gamma)
        apply_boundary_conditions(self._U, self._nx, self._ny, ng, self._bc[0], self._bc[1])
        if self._walls and not bool(np.all(self._mask != 0)):
            apply_solid_wall_fill(self._U, self._mask, ng, self._params.gamma)
        self._host_changed()

    def initialize(self, name: str):
        key = _PRESETS.get(name)
        if key is None:
            raise ValueError("Unknown initial condition: " + name)
        if key == "sod":
            self._params.gamma = 1.4
        elif key == "brio_wu":
            self._params.gamma = 2.0
        nx, ny = self._nx, self._ny
        if key == "orszag_tang":
            prim = _wl.orszag_tang(nx, ny)
        elif key == "sod":
            prim = _wl.sod(nx, ny, self._x_min, self._x_max, self._y_min, self._y_max)
        elif key == "brio_wu":
            prim = _wl.brio_wu(nx, ny)
        else:
            prim = {k: np.zeros((ny, nx)) for k in _wl.FIELDS}
            prim["rho"][:] = 1.0
            prim["p"][:] = 1.0
            if key == "sine":
                xs, _ = _wl.cell_centers(nx, ny, self._x_min, self._x_max, self._y_min,
                                         self._y_max)
                prim["rho"] = np.broadcast_to(1.0 + 0.1 * np.sin(2.0 * np.pi * xs), (ny, nx)).copy()
        self._sync_host()
        ng = self._ng
        self._U[:, ng:ng + ny, ng:ng + nx] = _wl.to_conservative(prim, self._params.gamma)
        apply_boundary_conditions(self._U, nx, ny, ng, self._bc[0], self._bc[1])
        if self._walls and not bool(np.all(self._mask != 0)):
            apply_solid_wall_fill(self._U, self._mask, ng, self._params.gamma)
        self._t = 0.0
        self._steps = 0
        self._host_changed()

    # ---- backend (solver_api.hpp:169-184, 394-400)
    def set_backend(self, backend: str, precision: str = "fp64"):
        if backend not in ("cpu", "CPU", "cuda", "CUDA", "metal", "Metal"):
            raise ValueError("Unknown backend: " + backend + " (expected cpu, cuda or metal)")
        name = backend.lower()
        if name != "cuda" or not cuda_available():
            raise RuntimeError("Backend not available: " + name)
        self._sync_host()
        self._precision = _capi.FP32 if precision == "fp32" else _capi.FP64
        if self._dev is not None:
            self._dev.close()
        self._dev = None
        self._device_valid = False
        self._configured = None

    @property
    def backend(self) -> str:
        return "cuda"

    def backend_device(self) -> str:
        return self._device().device_name()

    # ---- time integration (solver_api.hpp:294-329)
    def run(self, t_end: float) -> SolveResult:
        if t_end < 0.0:
            raise ValueError("run: t_end must be non-negative")
        dev = self._prepare_device()
        try:
            r = dev.solve(self._params.to_c(float(t_end)))
        except Exception:
            # As in the reference, a failed run leaves the host state as it was before the run.
            self._device_valid = False
            raise
        return self._account(r)

    def advance_to(self, t_abs: float) -> SolveResult:
        if t_abs < self._t:
            raise ValueError("advance_to: target time is earlier than current time")
        return self.run(t_abs - self._t)

    def solve_steps(self, nsteps: int) -> SolveResult:
        """Additive: exactly nsteps SSP-RK2 steps (no t_end limit)."""
        if nsteps < 0:
            raise ValueError("solve_steps: nsteps must be non-negative")
        dev = self._prepare_device()
        try:
            r = dev.solve_steps(self._params.to_c(0.0), int(nsteps))
        except Exception:
            self._device_valid = False
            raise
        return self._account(r)

    def diagnostics(self) -> dict:
        """Additive: FP64 diagnostics computed on the device."""
        dev = self._prepare_device()
        return dev.diagnostics(self._params.to_c(0.0))

    @property
    def time(self) -> float:
        return self._t

    @property
    def steps(self) -> int:
        return self._steps

    @property
    def c_h(self) -> float:
        return self._c_h

    def max_div_b(self) -> float:
        self._sync_host()
        return max_abs_div_b(self._U, self._nx, self._ny, self._ng, self._dx, self._dy)

    def field(self, name: str) -> np.ndarray:
        c = self._component(name)
        self._sync_host()
        return self._U[c].copy()

    # ---- geometry
    nx = property(lambda self: self._nx)
    ny = property(lambda self: self._ny)
    ng = property(lambda self: self._ng)
    size_x = property(lambda self: self._nx + 2 * self._ng)
    size_y = property(lambda self: self._ny + 2 * self._ng)
    x_min = property(lambda self: self._x_min)
    x_max = property(lambda self: self._x_max)
    y_min = property(lambda self: self._y_min)
    y_max = property(lambda self: self._y_max)

    @property
    def params(self) -> SolveParams:
        return self._params

    @params.setter
    def params(self, p: SolveParams):
        self._params = p.copy()

    # ---- internals
    def _component(self, name: str) -> int:
        try:
            return _COMPONENTS.index(name)
        except ValueError:
            raise ValueError("Unknown field: " + name) from None

    def _device(self) -> _capi.DeviceSolver:
        if self._dev is None:
            if not cuda_available():
                raise RuntimeError("Backend not available: cuda")
            self._dev = _capi.DeviceSolver(self._nx, self._ny, self._x_min, self._x_max,
                                           self._y_min, self._y_max, self._ng, self._precision)
        return self._dev

    def _host_changed(self):
        self._host_valid = True
        self._device_valid = False

    def _sync_host(self):
        if not self._host_valid:
            self._dev.download(self._U)
            self._host_valid = True

    def _prepare_device(self) -> _capi.DeviceSolver:
        dev = self._device()
        key = (int(self._bc[0]), int(self._bc[1]), self._walls, self._mask.tobytes())
        if self._configured != key:
            all_fluid = bool(np.all(self._mask != 0))
            dev.configure(int(self._bc[0]), int(self._bc[1]), None if all_fluid else self._mask,
                          self._walls)
            self._configured = key
        if not self._device_valid:
            dev.upload(self._U)
            self._device_valid = True
        return dev

    def _account(self, r) -> SolveResult:
        self._host_valid = False
        self._t += r.t
        self._steps += r.steps
        self._c_h = r.c_h
        return SolveResult(self._t, self._steps, self._c_h)
