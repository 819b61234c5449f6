"""ctypes front end of the CPU oracle — test infrastructure only.

Two implementations sit behind the same structs (oracle/mhd_oracle.h):

* ``impl="oracle"``: the plain-C restatement in ``mhd_oracle.c`` (always available);
* ``impl="ref"``: the reference CPU solver compiled from its own headers into
  ``oracle/_ref`` (SIMD + threads; minmod and MC only).

States are numpy float64 arrays of shape (9, ny + 2 ng, nx + 2 ng) in the reference's
StateField layout and component order (rho, mx, my, mz, E, bx, by, bz, psi).
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

MINMOD, MC, VANLEER = 0, 1, 2
PERIODIC, REFLECTIVE, OUTFLOW = 0, 1, 2
OK, EINVAL, EMAXSTEPS = 0, 1, 2


class _Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("ng", C.c_int), ("x_min", C.c_double),
                ("x_max", C.c_double), ("y_min", C.c_double), ("y_max", C.c_double)]


class _Params(C.Structure):
    _fields_ = [("t_end", C.c_double), ("cfl", C.c_double), ("gamma", C.c_double),
                ("glm_alpha", C.c_double), ("limiter", C.c_int), ("ohmic", C.c_int),
                ("hall", C.c_int), ("ambipolar", C.c_int), ("eta_ohm", C.c_double),
                ("eta_hall", C.c_double), ("eta_ambipolar", C.c_double),
                ("max_steps", C.c_int), ("fixed_steps", C.c_int)]


class _Result(C.Structure):
    _fields_ = [("t", C.c_double), ("steps", C.c_int), ("c_h", C.c_double)]


class _Diag(C.Structure):
    _fields_ = [("mass", C.c_double), ("energy", C.c_double), ("div_b_max", C.c_double),
                ("div_b_l2", C.c_double), ("rho_min", C.c_double), ("p_min", C.c_double),
                ("finite", C.c_int)]


@dataclass
class Grid:
    nx: int
    ny: int
    ng: int = 2
    x_min: float = 0.0
    x_max: float = 1.0
    y_min: float = 0.0
    y_max: float = 1.0

    @property
    def shape(self) -> tuple[int, int, int]:
        return (9, self.ny + 2 * self.ng, self.nx + 2 * self.ng)

    def c(self) -> _Grid:
        return _Grid(self.nx, self.ny, self.ng, self.x_min, self.x_max, self.y_min, self.y_max)


@dataclass
class Params:
    t_end: float = 0.0
    cfl: float = 0.4
    gamma: float = 5.0 / 3.0
    glm_alpha: float = 0.1
    limiter: int = MC
    ohmic: bool = False
    hall: bool = False
    ambipolar: bool = False
    eta_ohm: float = 0.0
    eta_hall: float = 0.0
    eta_ambipolar: float = 0.0
    max_steps: int = 1_000_000
    fixed_steps: bool = False

    def c(self) -> _Params:
        return _Params(self.t_end, self.cfl, self.gamma, self.glm_alpha, int(self.limiter),
                       int(self.ohmic), int(self.hall), int(self.ambipolar), self.eta_ohm,
                       self.eta_hall, self.eta_ambipolar, int(self.max_steps),
                       int(self.fixed_steps))


_PD = C.POINTER(C.c_double)
_PU8 = C.POINTER(C.c_uint8)
_libs: dict[str, C.CDLL] = {}


def _cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return " avx512f" in f.read()
    except OSError:
        return False


def ref_library_path() -> str | None:
    isa = "avx512" if _cpu_has_avx512() else "avx2"
    path = os.path.join(HERE, "_ref", f"libmhd_ref_{isa}.so")
    return path if os.path.exists(path) else None


def _lib(impl: str) -> C.CDLL:
    if impl in _libs:
        return _libs[impl]
    if impl == "oracle":
        path = os.path.join(HERE, "libmhd_oracle.so")
        if not os.path.exists(path):
            from oracle.build_oracle import build_oracle
            build_oracle()
        lib = C.CDLL(path)
        prefix = "mhdo_"
    elif impl == "ref":
        path = ref_library_path()
        if path is None:
            raise FileNotFoundError("reference CPU library not built (oracle/_ref)")
        lib = C.CDLL(path)
        prefix = "mhdr_"
        lib.mhdr_set_threads.argtypes = [C.c_int]
        lib.mhdr_set_threads.restype = C.c_int
        lib.mhdr_simd_backend.restype = C.c_char_p
        lib.mhdr_last_loop_seconds.restype = C.c_double
    else:
        raise ValueError(impl)
    solve = getattr(lib, prefix + "solve")
    solve.argtypes = [C.POINTER(_Grid), C.POINTER(_Params), C.c_int, C.c_int, _PU8, C.c_int,
                      _PD, C.POINTER(_Result)]
    solve.restype = C.c_int
    rhs = getattr(lib, prefix + "rhs")
    rhs.argtypes = [C.POINTER(_Grid), C.POINTER(_Params), _PU8, C.c_double, _PD, _PD]
    rhs.restype = C.c_int
    if impl == "oracle":
        lib.mhdo_apply_bc.argtypes = [C.POINTER(_Grid), C.c_int, C.c_int, _PD]
        lib.mhdo_wall_fill.argtypes = [C.POINTER(_Grid), _PU8, C.c_double, _PD]
        lib.mhdo_cfl.argtypes = [C.POINTER(_Grid), C.POINTER(_Params), _PU8, _PD, _PD, _PD]
        lib.mhdo_nonideal_e.argtypes = [_PD, _PD, C.POINTER(_Params), _PD]
        lib.mhdo_nonideal_e.restype = None
        lib.mhdo_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.mhdo_limiter.restype = C.c_double
        lib.mhdo_face_flux.argtypes = [C.c_int, _PD, _PD, _PD, _PD, C.c_double, C.c_double, _PD]
        lib.mhdo_face_flux.restype = None
        lib.mhdo_diagnostics.argtypes = [C.POINTER(_Grid), C.c_double, _PD, C.POINTER(_Diag)]
    _libs[impl] = lib
    return lib


def _pd(a: np.ndarray):
    return a.ctypes.data_as(_PD)


def _mask_ptr(mask):
    if mask is None:
        return None, None
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    return m, m.ctypes.data_as(_PU8)


class OracleError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: oracle status {code}")
        self.code = code


def solve(U: np.ndarray, grid: Grid, params: Params, bc=(PERIODIC, PERIODIC), mask=None,
          walls: bool = True, impl: str = "oracle"):
    """Advance a copy of U; returns (U_out, t, steps, c_h). Raises OracleError on failure."""
    lib = _lib(impl)
    out = np.ascontiguousarray(U, dtype=np.float64).copy()
    assert out.shape == grid.shape, (out.shape, grid.shape)
    m, mp = _mask_ptr(mask)
    res = _Result()
    fn = lib.mhdo_solve if impl == "oracle" else lib.mhdr_solve
    g, p = grid.c(), params.c()
    rc = fn(C.byref(g), C.byref(p), int(bc[0]), int(bc[1]), mp, int(walls), _pd(out),
            C.byref(res))
    if rc != OK:
        raise OracleError(rc, "solve")
    return out, res.t, res.steps, res.c_h


def rhs(U: np.ndarray, grid: Grid, params: Params, c_h: float, mask=None, impl: str = "oracle"):
    lib = _lib(impl)
    Uc = np.ascontiguousarray(U, dtype=np.float64)
    R = np.zeros_like(Uc)
    m, mp = _mask_ptr(mask)
    fn = lib.mhdo_rhs if impl == "oracle" else lib.mhdr_rhs
    g, p = grid.c(), params.c()
    rc = fn(C.byref(g), C.byref(p), mp, float(c_h), _pd(Uc), _pd(R))
    if rc != OK:
        raise OracleError(rc, "rhs")
    return R


def apply_bc(U: np.ndarray, grid: Grid, bc=(PERIODIC, PERIODIC)) -> np.ndarray:
    out = np.ascontiguousarray(U, dtype=np.float64).copy()
    g = grid.c()
    rc = _lib("oracle").mhdo_apply_bc(C.byref(g), int(bc[0]), int(bc[1]), _pd(out))
    if rc != OK:
        raise OracleError(rc, "apply_bc")
    return out


def wall_fill(U: np.ndarray, grid: Grid, mask, gamma: float) -> np.ndarray:
    out = np.ascontiguousarray(U, dtype=np.float64).copy()
    m, mp = _mask_ptr(mask)
    g = grid.c()
    _lib("oracle").mhdo_wall_fill(C.byref(g), mp, float(gamma), _pd(out))
    return out


def cfl(U: np.ndarray, grid: Grid, params: Params, mask=None) -> tuple[float, float]:
    Uc = np.ascontiguousarray(U, dtype=np.float64)
    m, mp = _mask_ptr(mask)
    dt, ch = C.c_double(), C.c_double()
    g, p = grid.c(), params.c()
    rc = _lib("oracle").mhdo_cfl(C.byref(g), C.byref(p), mp, _pd(Uc), C.byref(dt), C.byref(ch))
    if rc != OK:
        raise OracleError(rc, "cfl")
    return dt.value, ch.value


def limiter(kind: int, a: float, b: float) -> float:
    return _lib("oracle").mhdo_limiter(int(kind), float(a), float(b))


def nonideal_e(J, B, params: Params) -> np.ndarray:
    """E = eta_O J + eta_H J x B / |B| + eta_A (J x B) x B / |B|^2 of the enabled terms."""
    j = np.ascontiguousarray(J, dtype=np.float64)
    b = np.ascontiguousarray(B, dtype=np.float64)
    e = np.zeros(3)
    p = params.c()
    _lib("oracle").mhdo_nonideal_e(_pd(j), _pd(b), C.byref(p), _pd(e))
    return e


def face_flux(kind: int, wmm, wm, w0, wp, gamma: float, c_h: float) -> np.ndarray:
    arrs = [np.ascontiguousarray(w, dtype=np.float64) for w in (wmm, wm, w0, wp)]
    out = np.zeros(9)
    _lib("oracle").mhdo_face_flux(int(kind), *[_pd(a) for a in arrs], float(gamma), float(c_h),
                                  _pd(out))
    return out


def diagnostics(U: np.ndarray, grid: Grid, gamma: float) -> dict:
    Uc = np.ascontiguousarray(U, dtype=np.float64)
    d = _Diag()
    g = grid.c()
    _lib("oracle").mhdo_diagnostics(C.byref(g), float(gamma), _pd(Uc), C.byref(d))
    return {"mass": d.mass, "energy": d.energy, "div_b_max": d.div_b_max,
            "div_b_l2": d.div_b_l2, "rho_min": d.rho_min, "p_min": d.p_min,
            "finite": bool(d.finite)}


def ref_set_threads(n: int) -> int:
    return _lib("ref").mhdr_set_threads(int(n))


def ref_last_loop_seconds() -> float:
    """Step-loop seconds of the last impl="ref" solve (copies and allocation excluded)."""
    return float(_lib("ref").mhdr_last_loop_seconds())


def ref_simd_backend() -> str:
    return _lib("ref").mhdr_simd_backend().decode()


def to_conservative(rho, vx, vy, vz, p, bx, by, bz, psi, gamma: float) -> np.ndarray:
    """include/mhd/mhd_physics.hpp:41-57, vectorised (interior arrays, shape (ny, nx))."""
    e_kin = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    e_mag = 0.5 * (bx * bx + by * by + bz * bz)
    E = p / (gamma - 1.0) + e_kin + e_mag
    return np.stack([rho, rho * vx, rho * vy, rho * vz, E, bx, by, bz, psi])
