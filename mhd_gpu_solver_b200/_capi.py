"""ctypes binding of the C ABI in ``include/mhd_b200.h``.

The CUDA library is required: importing this module loads ``libmhd_b200.so`` and raises
``ImportError`` if it has not been built. Status codes become the exception types the reference
pybind module raises for the same C++ exceptions (std::invalid_argument -> ValueError,
std::runtime_error -> RuntimeError).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmhd_b200.so")

OK, INVALID_ARGUMENT, MAX_STEPS, CUDA_ERROR, NO_DEVICE, BAD_TIMESTEP = range(6)
FP64, FP32 = 0, 1
BC_PERIODIC, BC_REFLECTIVE, BC_OUTFLOW = 0, 1, 2
MINMOD, MC, VANLEER = 0, 1, 2

# Every entry point declared in include/mhd_b200.h.
EXPORTS = (
    "mhdb_cuda_available", "mhdb_create", "mhdb_destroy", "mhdb_last_error", "mhdb_device_name",
    "mhdb_precision", "mhdb_configure", "mhdb_upload", "mhdb_download", "mhdb_solve",
    "mhdb_solve_steps", "mhdb_diagnostics", "mhdb_stream", "mhdb_set_profiling",
    "mhdb_profile_read", "mhdb_launch_count", "mhdb_tile_config_count", "mhdb_tile_config_info",
    "mhdb_tile_config_kind", "mhdb_set_tile_config", "mhdb_solve_steps_noalloc_f64",
    "mhdb_batch_create", "mhdb_batch_destroy", "mhdb_batch_last_error", "mhdb_batch_add",
    "mhdb_batch_remove", "mhdb_batch_step", "mhdb_batch_status", "mhdb_batch_download",
    "mhdb_batch_info", "mhdb_batch_stream", "mhdb_generate", "mhdb_batch_add_generated",
    "mhdb_batch_launch", "mhdb_batch_poll", "mhdb_batch_config_count", "mhdb_batch_config_info",
    "mhdb_batch_set_config", "mhdb_set_cell_size", "mhdb_set_reduce_rows", "mhdb_strip_view", "mhdb_strip_begin",
    "mhdb_strip_step", "mhdb_strip_finish", "mhdb_strip_poll", "mhdb_strip_end",
    "mhdb_debug_stall_copies", "mhdb_batch_debug_stall_copies", "mhdb_configure_shapes",
    "mhdb_get_mask",
)


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("ng", C.c_int), ("x_min", C.c_double),
                ("x_max", C.c_double), ("y_min", C.c_double), ("y_max", C.c_double)]


class Params(C.Structure):
    _fields_ = [("t_end", C.c_double), ("cfl", C.c_double), ("gamma", C.c_double),
                ("glm_alpha", C.c_double), ("limiter", C.c_int), ("ohmic", C.c_int),
                ("hall", C.c_int), ("ambipolar", C.c_int), ("eta_ohm", C.c_double),
                ("eta_hall", C.c_double), ("eta_ambipolar", C.c_double),
                ("max_steps", C.c_int)]


def nonideal_any(p: Params) -> bool:
    """Whether the non-ideal terms are on: a flag set and its coefficient non-zero
    (include/physics_config/mhd_config.hpp:90-94)."""
    return bool((p.ohmic and p.eta_ohm != 0.0) or (p.hall and p.eta_hall != 0.0)
                or (p.ambipolar and p.eta_ambipolar != 0.0))


class Result(C.Structure):
    _fields_ = [("t", C.c_double), ("steps", C.c_int), ("c_h", C.c_double)]


class Diag(C.Structure):
    _fields_ = [("mass", C.c_double), ("energy", C.c_double), ("div_b_max", C.c_double),
                ("div_b_l2", C.c_double), ("rho_min", C.c_double), ("p_min", C.c_double),
                ("finite", C.c_int)]


class Shape(C.Structure):
    """mhdb_shape: kind 0 circle (centre (a, b), radius c), 1 rectangle (corners (a, b),
    (c, d)); solid 1 paints contained cells solid, 0 fluid."""
    _fields_ = [("kind", C.c_int), ("solid", C.c_int), ("a", C.c_double), ("b", C.c_double),
                ("c", C.c_double), ("d", C.c_double)]


class StripState(C.Structure):
    _fields_ = [("state", C.c_void_p), ("ch_bits", C.c_void_p), ("pitch", C.c_longlong),
                ("plane", C.c_longlong), ("planes", C.c_int), ("elem_bytes", C.c_int)]


class Init(C.Structure):
    _fields_ = [("kind", C.c_int), ("kmax", C.c_int), ("coef", C.POINTER(C.c_double)),
                ("quad", (C.c_double * 5) * 4)]


INIT_FOURIER, INIT_QUADRANTS = 0, 1

_PD = C.POINTER(C.c_double)
_PPD = C.POINTER(_PD)


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA backend first "
            "(python mhd_gpu_solver_b200/build.py or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    h = C.c_void_p
    sig = {
        "mhdb_cuda_available": ([], C.c_int),
        "mhdb_create": ([C.POINTER(Grid), C.c_int, C.POINTER(h)], C.c_int),
        "mhdb_destroy": ([h], None),
        "mhdb_last_error": ([h], C.c_char_p),
        "mhdb_device_name": ([h, C.c_char_p, C.c_size_t], C.c_int),
        "mhdb_precision": ([h], C.c_int),
        "mhdb_configure": ([h, C.c_int, C.c_int, C.POINTER(C.c_uint8), C.c_size_t, C.c_int],
                           C.c_int),
        "mhdb_upload": ([h, _PPD, C.c_size_t], C.c_int),
        "mhdb_download": ([h, _PPD, C.c_size_t], C.c_int),
        "mhdb_solve": ([h, C.POINTER(Params), C.POINTER(Result)], C.c_int),
        "mhdb_solve_steps": ([h, C.POINTER(Params), C.c_int, C.POINTER(Result)], C.c_int),
        "mhdb_diagnostics": ([h, C.POINTER(Params), C.POINTER(Diag)], C.c_int),
        "mhdb_stream": ([h], C.c_void_p),
        "mhdb_set_profiling": ([h, C.c_int], C.c_int),
        "mhdb_profile_read": ([h, _PD, C.POINTER(C.c_int), _PD, C.POINTER(C.c_int), C.c_int],
                              C.c_int),
        "mhdb_launch_count": ([h], C.c_longlong),
        "mhdb_tile_config_count": ([C.c_int], C.c_int),
        "mhdb_tile_config_info": ([C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "mhdb_tile_config_kind": ([C.c_int, C.c_int], C.c_int),
        "mhdb_set_tile_config": ([h, C.c_int], C.c_int),
        "mhdb_debug_stall_copies": ([h, C.c_int], C.c_int),
        "mhdb_configure_shapes": ([h, C.c_int, C.c_int, C.POINTER(Shape), C.c_int, C.c_int],
                                  C.c_int),
        "mhdb_get_mask": ([h, C.POINTER(C.c_uint8), C.c_size_t], C.c_int),
        "mhdb_solve_steps_noalloc_f64": ([C.POINTER(Grid), C.c_int, C.c_int, C.POINTER(Params),
                                          C.c_int, C.c_void_p, C.c_void_p, C.POINTER(Result),
                                          C.c_void_p], C.c_int),
    }
    b = C.c_void_p
    sig.update({
        "mhdb_batch_create": ([C.c_int, C.POINTER(b)], C.c_int),
        "mhdb_batch_destroy": ([b], None),
        "mhdb_batch_last_error": ([b], C.c_char_p),
        "mhdb_batch_add": ([b, C.POINTER(Grid), C.POINTER(Params), C.c_int, C.c_int, _PPD,
                            C.c_size_t, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "mhdb_batch_remove": ([b, C.c_int], C.c_int),
        "mhdb_batch_step": ([b, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "mhdb_batch_launch": ([b, C.c_int], C.c_int),
        "mhdb_batch_config_count": ([C.c_int], C.c_int),
        "mhdb_batch_config_info": ([C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "mhdb_batch_set_config": ([b, C.c_int, C.c_int], C.c_int),
        "mhdb_batch_debug_stall_copies": ([b, C.c_int, C.c_int], C.c_int),
        "mhdb_batch_poll": ([b, C.POINTER(C.c_int)], C.c_int),
        "mhdb_batch_status": ([b, C.c_int, C.POINTER(Result), C.POINTER(C.c_int)], C.c_int),
        "mhdb_batch_download": ([b, C.c_int, _PPD, C.c_size_t], C.c_int),
        "mhdb_batch_info": ([b, C.POINTER(C.c_size_t), C.POINTER(C.c_int),
                             C.POINTER(C.c_longlong)], C.c_int),
        "mhdb_batch_stream": ([b], C.c_void_p),
        "mhdb_batch_add_generated": ([b, C.POINTER(Grid), C.POINTER(Params), C.c_int, C.c_int,
                                      C.POINTER(Init), C.c_int, C.POINTER(C.c_int)], C.c_int),
        "mhdb_generate": ([h, C.POINTER(Init), C.POINTER(Params)], C.c_int),
        "mhdb_set_cell_size": ([h, C.c_double, C.c_double], C.c_int),
        "mhdb_set_reduce_rows": ([h, C.c_int, C.c_int], C.c_int),
        "mhdb_strip_view": ([h, C.POINTER(StripState)], C.c_int),
        "mhdb_strip_begin": ([h, C.POINTER(Params), C.c_int], C.c_int),
        "mhdb_strip_step": ([h], C.c_int),
        "mhdb_strip_finish": ([h], C.c_int),
        "mhdb_strip_poll": ([h, C.POINTER(C.c_int), C.POINTER(C.c_int), _PD], C.c_int),
        "mhdb_strip_end": ([h, C.POINTER(Result)], C.c_int),
    })
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


class MhdbError(RuntimeError):
    """Failure reported through the C ABI; ``code`` is the mhdb_status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class MhdbValueError(ValueError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def raise_for(code: int, handle) -> None:
    if code == OK:
        return
    msg = lib.mhdb_last_error(handle)
    text = msg.decode() if msg else f"mhdb status {code}"
    if code in (INVALID_ARGUMENT, BAD_TIMESTEP):
        raise MhdbValueError(code, text)
    raise MhdbError(code, text)


def cuda_available() -> bool:
    return bool(lib.mhdb_cuda_available())


def plane_pointers(state: np.ndarray):
    """Array of 9 double* into the planes of a C-contiguous (9, ny_tot, nx_tot) float64 array."""
    if state.dtype != np.float64 or not state.flags.c_contiguous or state.shape[0] != 9:
        raise ValueError("state must be a C-contiguous float64 array of shape (9, ny_tot, nx_tot)")
    base = state.ctypes.data
    stride = state.strides[0]
    arr = (_PD * 9)(*[C.cast(C.c_void_p(base + c * stride), _PD) for c in range(9)])
    return arr


class DeviceSolver:
    """Owning wrapper of one mhdb_solver handle (the reference DeviceSolver interface)."""

    def __init__(self, nx: int, ny: int, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, ng=2,
                 precision: int = FP64):
        self._h = C.c_void_p()
        g = Grid(int(nx), int(ny), int(ng), float(x_min), float(x_max), float(y_min),
                 float(y_max))
        raise_for(lib.mhdb_create(C.byref(g), int(precision), C.byref(self._h)), None)
        self.nx, self.ny, self.ng = int(nx), int(ny), int(ng)
        self.shape = (9, self.ny + 2 * self.ng, self.nx + 2 * self.ng)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.mhdb_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def device_name(self) -> str:
        buf = C.create_string_buffer(256)
        raise_for(lib.mhdb_device_name(self._h, buf, 256), self._h)
        return buf.value.decode()

    def precision(self) -> int:
        return lib.mhdb_precision(self._h)

    def configure(self, bc_x: int, bc_y: int, mask=None, reflective_walls: bool = True) -> None:
        if mask is None:
            rc = lib.mhdb_configure(self._h, int(bc_x), int(bc_y), None, 0, int(reflective_walls))
        else:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            rc = lib.mhdb_configure(self._h, int(bc_x), int(bc_y),
                                    m.ctypes.data_as(C.POINTER(C.c_uint8)), m.size,
                                    int(reflective_walls))
        raise_for(rc, self._h)

    def configure_shapes(self, bc_x: int, bc_y: int, shapes, reflective_walls: bool = True) -> None:
        """configure() with a mask rasterised on the device from (kind, solid, a, b, c, d)
        shapes (workloads.circles_and_rectangles_shapes), painted in order."""
        arr = (Shape * max(1, len(shapes)))(*[Shape(int(k), int(sd), float(a), float(b),
                                                    float(c), float(d))
                                              for k, sd, a, b, c, d in shapes])
        raise_for(lib.mhdb_configure_shapes(self._h, int(bc_x), int(bc_y), arr, len(shapes),
                                            int(reflective_walls)), self._h)

    def get_mask(self) -> np.ndarray:
        """The interior fluid mask in use, (ny, nx) uint8, 1 = fluid."""
        ny, nx = self.shape[1] - 2 * self.ng, self.shape[2] - 2 * self.ng
        out = np.empty((ny, nx), dtype=np.uint8)
        raise_for(lib.mhdb_get_mask(self._h, out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size),
                  self._h)
        return out

    def upload(self, state: np.ndarray) -> None:
        ptrs = plane_pointers(state)
        raise_for(lib.mhdb_upload(self._h, ptrs, state.shape[1] * state.shape[2]), self._h)

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        ptrs = plane_pointers(out)
        raise_for(lib.mhdb_download(self._h, ptrs, out.shape[1] * out.shape[2]), self._h)
        return out

    def solve(self, params: Params) -> Result:
        r = Result()
        raise_for(lib.mhdb_solve(self._h, C.byref(params), C.byref(r)), self._h)
        return r

    def solve_steps(self, params: Params, nsteps: int) -> Result:
        r = Result()
        raise_for(lib.mhdb_solve_steps(self._h, C.byref(params), int(nsteps), C.byref(r)),
                  self._h)
        return r

    def diagnostics(self, params: Params) -> dict:
        d = Diag()
        raise_for(lib.mhdb_diagnostics(self._h, C.byref(params), C.byref(d)), self._h)
        return {"mass": d.mass, "energy": d.energy, "div_b_max": d.div_b_max,
                "div_b_l2": d.div_b_l2, "rho_min": d.rho_min, "p_min": d.p_min,
                "finite": bool(d.finite)}

    def stream(self) -> int:
        return lib.mhdb_stream(self._h) or 0

    def set_profiling(self, enabled: bool) -> None:
        raise_for(lib.mhdb_set_profiling(self._h, int(enabled)), self._h)

    def profile_read(self, reset: bool = True) -> dict:
        m1, m2 = C.c_double(), C.c_double()
        n1, n2 = C.c_int(), C.c_int()
        raise_for(lib.mhdb_profile_read(self._h, C.byref(m1), C.byref(n1), C.byref(m2),
                                        C.byref(n2), int(reset)), self._h)
        return {"stage1_ms": m1.value, "stage1_launches": n1.value, "stage2_ms": m2.value,
                "stage2_launches": n2.value}

    def launch_count(self) -> int:
        return int(lib.mhdb_launch_count(self._h))

    def generate(self, init: "InitSpec", params: Params) -> None:
        """Replace the device state by a seeded initial state generated on the device."""
        c = init.c()
        raise_for(lib.mhdb_generate(self._h, C.byref(c), C.byref(params)), self._h)

    def set_tile_config(self, config: int) -> None:
        raise_for(lib.mhdb_set_tile_config(self._h, int(config)), self._h)

    def debug_stall_copies(self, extra_bytes: int) -> None:
        """Test hook: make one bulk-copy wait of the TMA strip marches run out
        (mhdb_debug_stall_copies); 0 turns it off."""
        raise_for(lib.mhdb_debug_stall_copies(self._h, int(extra_bytes)), self._h)

    # Deferred solves of one strip of a split grid (strips.py drives them).
    def set_cell_size(self, dx: float, dy: float) -> None:
        raise_for(lib.mhdb_set_cell_size(self._h, float(dx), float(dy)), self._h)

    def set_reduce_rows(self, y0: int, y1: int) -> None:
        raise_for(lib.mhdb_set_reduce_rows(self._h, int(y0), int(y1)), self._h)

    def strip_view(self) -> StripState:
        v = StripState()
        raise_for(lib.mhdb_strip_view(self._h, C.byref(v)), self._h)
        return v

    def strip_begin(self, params: Params, nsteps: int) -> None:
        raise_for(lib.mhdb_strip_begin(self._h, C.byref(params), int(nsteps)), self._h)

    def strip_step(self) -> None:
        raise_for(lib.mhdb_strip_step(self._h), self._h)

    def strip_finish(self) -> None:
        raise_for(lib.mhdb_strip_finish(self._h), self._h)

    def strip_poll(self) -> tuple[bool, int, float]:
        f, n, t = C.c_int(), C.c_int(), C.c_double()
        raise_for(lib.mhdb_strip_poll(self._h, C.byref(f), C.byref(n), C.byref(t)), self._h)
        return bool(f.value), n.value, t.value

    def strip_end(self) -> Result:
        r = Result()
        raise_for(lib.mhdb_strip_end(self._h, C.byref(r)), self._h)
        return r


KERNEL_KINDS = {0: "tile", 1: "tile_merged", 2: "march", 3: "march_tma", 4: "march_tma_delta",
                5: "march_tma_pair"}


def tile_configs(precision: int) -> list[dict]:
    out = []
    for c in range(lib.mhdb_tile_config_count(int(precision))):
        v = [C.c_int() for _ in range(4)]
        raise_for(lib.mhdb_tile_config_info(int(precision), c, *[C.byref(x) for x in v]), None)
        out.append({"config": c, "tile_x": v[0].value, "tile_y": v[1].value,
                    "threads": v[2].value, "min_blocks": v[3].value,
                    "kind": KERNEL_KINDS[lib.mhdb_tile_config_kind(int(precision), c)]})
    return out


def make_params(t_end=0.0, cfl=0.4, gamma=5.0 / 3.0, glm_alpha=0.1, limiter=MC, ohmic=False,
                hall=False, ambipolar=False, eta_ohm=0.0, eta_hall=0.0, eta_ambipolar=0.0,
                max_steps=1_000_000) -> Params:
    return Params(float(t_end), float(cfl), float(gamma), float(glm_alpha), int(limiter),
                  int(bool(ohmic)), int(bool(hall)), int(bool(ambipolar)), float(eta_ohm),
                  float(eta_hall), float(eta_ambipolar), int(max_steps))


class InitSpec:
    """Seeded initial state for the device generator: ``fourier(seed)`` or ``quadrants(seed)``
    (the same draws as workloads.fourier_state / workloads.four_quadrant)."""

    def __init__(self, kind: int, kmax: int = 8, coef=None, quad=None):
        self.kind = kind
        self.kmax = kmax
        self._coef = None
        if coef is not None:
            self._coef = np.ascontiguousarray(
                np.stack([coef.real, coef.imag], axis=-1), dtype=np.float64)
        self.quad = np.zeros((4, 5)) if quad is None else np.asarray(quad, dtype=np.float64)

    @staticmethod
    def fourier(seed: int, kmax: int = 8) -> "InitSpec":
        from .workloads import fourier_coefficients
        return InitSpec(INIT_FOURIER, kmax, coef=fourier_coefficients(seed, kmax))

    @staticmethod
    def quadrants(seed: int) -> "InitSpec":
        from .workloads import quadrant_values
        return InitSpec(INIT_QUADRANTS, quad=quadrant_values(seed))

    def c(self) -> Init:
        out = Init()
        out.kind = self.kind
        out.kmax = self.kmax
        out.coef = (self._coef.ctypes.data_as(C.POINTER(C.c_double))
                    if self._coef is not None else None)
        for q in range(4):
            for v in range(5):
                out.quad[q][v] = float(self.quad[q, v])
        return out
