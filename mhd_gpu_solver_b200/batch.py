"""Batched form: many independent solves advanced together (C ABI ``mhdb_batch_*``).

Every RK2 step of the batch is one persistent launch per stage (per limiter and non-ideal
combination present) over a tile work-list of all unfinished solves; chunks of steps are CUDA
graphs. Each solve keeps its own grid, parameters, boundary rule, time target, HBM-resident state
and FP64 clock, so its result does not depend on the other solves in the batch.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _capi


def batch_configs(precision: int) -> list[dict]:
    """The batch configurations of a precision form: kernel kind, work-item tile, threads."""
    out = []
    for c in range(_capi.lib.mhdb_batch_config_count(int(precision))):
        tx, ty, nt, kind = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _capi.lib.mhdb_batch_config_info(int(precision), c, C.byref(tx), C.byref(ty),
                                         C.byref(nt), C.byref(kind))
        out.append({"config": c, "tile_x": tx.value, "tile_y": ty.value, "threads": nt.value,
                    "kind": _capi.KERNEL_KINDS[kind.value]})
    return out


class BatchSolver:
    """tune=True: each added solve runs the batch configuration the batch autotuner picked for
    its size class (tuned on first use, cached per process); otherwise the library's default."""

    def __init__(self, precision: int = _capi.FP32, tune: bool = False):
        self._b = C.c_void_p()
        rc = _capi.lib.mhdb_batch_create(int(precision), C.byref(self._b))
        if rc != _capi.OK:
            raise _capi.MhdbError(rc, _capi.lib.mhdb_batch_last_error(None).decode())
        self.precision = int(precision)
        self.tune = bool(tune)
        self._shapes: dict[int, tuple[int, int, int]] = {}

    def _raise(self, rc: int) -> None:
        if rc == _capi.OK:
            return
        msg = _capi.lib.mhdb_batch_last_error(self._b).decode()
        if rc in (_capi.INVALID_ARGUMENT, _capi.BAD_TIMESTEP):
            raise _capi.MhdbValueError(rc, msg)
        raise _capi.MhdbError(rc, msg)

    def close(self) -> None:
        if getattr(self, "_b", None) is not None and self._b.value:
            _capi.lib.mhdb_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, state: np.ndarray, params: _capi.Params, bc=(0, 0), fixed_steps: bool = False,
            x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, ng: int = 2) -> int:
        """Add a solve from a ghosted (9, ny + 2 ng, nx + 2 ng) float64 host state."""
        state = np.ascontiguousarray(state, dtype=np.float64)
        ny, nx = state.shape[1] - 2 * ng, state.shape[2] - 2 * ng
        g = _capi.Grid(nx, ny, ng, float(x_min), float(x_max), float(y_min), float(y_max))
        sid = C.c_int()
        self._raise(_capi.lib.mhdb_batch_add(
            self._b, C.byref(g), C.byref(params), int(bc[0]), int(bc[1]),
            _capi.plane_pointers(state), state.shape[1] * state.shape[2], int(bool(fixed_steps)),
            C.byref(sid)))
        self._shapes[sid.value] = state.shape
        self._tuned(sid.value, nx, ny, params)
        return sid.value

    def add_generated(self, nx: int, ny: int, init: "_capi.InitSpec", params: _capi.Params,
                      bc=(0, 0), fixed_steps: bool = False, x_min=0.0, x_max=1.0, y_min=0.0,
                      y_max=1.0, ng: int = 2) -> int:
        """Add a solve whose seeded initial state is generated on the device (no upload)."""
        g = _capi.Grid(int(nx), int(ny), ng, float(x_min), float(x_max), float(y_min),
                       float(y_max))
        c = init.c()
        sid = C.c_int()
        self._raise(_capi.lib.mhdb_batch_add_generated(
            self._b, C.byref(g), C.byref(params), int(bc[0]), int(bc[1]), C.byref(c),
            int(bool(fixed_steps)), C.byref(sid)))
        self._shapes[sid.value] = (9, int(ny) + 2 * ng, int(nx) + 2 * ng)
        self._tuned(sid.value, int(nx), int(ny), params)
        return sid.value

    def _tuned(self, sid: int, nx: int, ny: int, params: _capi.Params) -> None:
        if not self.tune:
            return
        from . import autotune

        ni = _capi.nonideal_any(params)
        self.set_config(sid, autotune.tune_batch(self.precision, params.limiter, nx, ny, ni))

    def set_config(self, sid: int, config: int) -> None:
        """Run this solve with batch configuration `config` (-1: chosen by its size)."""
        self._raise(_capi.lib.mhdb_batch_set_config(self._b, int(sid), int(config)))

    def debug_stall_copies(self, sid: int, extra_bytes: int) -> None:
        """Test hook: make one bulk-copy wait of this solve's TMA strip march run out
        (mhdb_batch_debug_stall_copies); 0 turns it off."""
        self._raise(_capi.lib.mhdb_batch_debug_stall_copies(self._b, int(sid), int(extra_bytes)))

    def remove(self, sid: int) -> None:
        self._raise(_capi.lib.mhdb_batch_remove(self._b, int(sid)))
        self._shapes.pop(sid, None)

    def step(self, nsteps: int) -> int:
        """Advance all unfinished solves by up to nsteps steps; returns how many are unfinished."""
        active = C.c_int()
        self._raise(_capi.lib.mhdb_batch_step(self._b, int(nsteps), C.byref(active)))
        return active.value

    def launch(self, nsteps: int) -> None:
        """Issue up to nsteps steps of every unfinished solve without waiting for them."""
        self._raise(_capi.lib.mhdb_batch_launch(self._b, int(nsteps)))

    def poll(self) -> int:
        """Wait for the issued steps and refresh every status; returns the unfinished count."""
        active = C.c_int()
        self._raise(_capi.lib.mhdb_batch_poll(self._b, C.byref(active)))
        return active.value

    def status(self, sid: int):
        """(Result, finished); raises for a solve that hit max_steps or a bad dt."""
        r = _capi.Result()
        fin = C.c_int()
        self._raise(_capi.lib.mhdb_batch_status(self._b, int(sid), C.byref(r), C.byref(fin)))
        return r, bool(fin.value)

    def download(self, sid: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self._shapes[sid], dtype=np.float64)
        self._raise(_capi.lib.mhdb_batch_download(self._b, int(sid), _capi.plane_pointers(out),
                                                  out.shape[1] * out.shape[2]))
        return out

    def info(self) -> dict:
        nbytes = C.c_size_t()
        live = C.c_int()
        launches = C.c_longlong()
        _capi.lib.mhdb_batch_info(self._b, C.byref(nbytes), C.byref(live), C.byref(launches))
        return {"bytes_in_use": nbytes.value, "live": live.value, "launches": launches.value}

    def stream(self) -> int:
        return _capi.lib.mhdb_batch_stream(self._b) or 0


def state_bytes(nx: int, ny: int) -> int:
    """HBM bytes a solve of nx x ny interior cells holds in a batch (two padded states)."""
    pitch = (nx + 31) // 32 * 32
    return 2 * 9 * pitch * ny * 8


def fixed_params(nsteps: int, **kw) -> _capi.Params:
    """Parameters of a fixed-step solve (t_end ignored, exactly nsteps steps)."""
    return _capi.make_params(t_end=math.inf, max_steps=int(nsteps), **kw)
