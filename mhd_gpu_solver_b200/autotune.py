"""Per-size-class tile autotuner for the stage kernels.

The stage kernels are compiled for a few tile configurations (tile width x height, threads per
CTA, minimum CTAs per SM; ``_capi.tile_configs``). For a grid size class (interior cells rounded
to a power of two, per precision form and limiter) the tuner times each configuration on a
synthetic smooth state for a few RK2 steps, with CUDA events on the solver's stream, and
remembers the fastest. Results are cached in memory for the process and can be saved to / loaded
from a JSON file. Configurations other than 0 serve unmasked solves (the strip-march ones ideal
and non-ideal solves, the other tile ones ideal solves only; FP32-mixed configurations 11, 13
and 17 and FP64 configuration 7 also masked solves); a solve that the chosen configuration does
not serve runs the library's default for its size.

``tune_batch`` does the same for the batched form: per (precision, limiter, ideal or non-ideal,
size class) it times every batch configuration (``batch.batch_configs``: strip march with or
without TMA staging of the rows, work-item shapes) on a batch of same-class solves that fills the
GPU, and remembers the fastest; ``BatchSolver(tune=True)`` applies the choice to each solve.
"""

from __future__ import annotations

import json
import math
import threading

import numpy as np

from . import _capi
from . import workloads as wl

_lock = threading.Lock()
_cache: dict[str, int] = {}


def size_class(nx: int, ny: int) -> int:
    """log2 of the interior cell count, rounded to the nearest integer."""
    return int(round(math.log2(max(1, nx * ny))))


def _key(precision: int, limiter: int, nx: int, ny: int) -> str:
    return f"p{precision}-l{limiter}-s{size_class(nx, ny)}"


def _time_config(precision: int, limiter: int, nx: int, ny: int, config: int, state: np.ndarray,
                 steps: int) -> float:
    dev = _capi.DeviceSolver(nx, ny, precision=precision)
    try:
        dev.set_tile_config(config)
        dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
        dev.upload(state)
        params = _capi.make_params(limiter=limiter)
        dev.solve_steps(params, 2)  # warm-up: graphs, attributes, caches
        dev.set_profiling(True)
        dev.profile_read(reset=True)
        dev.solve_steps(params, steps)
        prof = dev.profile_read(reset=True)
        return prof["stage1_ms"] + prof["stage2_ms"]
    finally:
        dev.close()


def tune(precision: int, limiter: int, nx: int, ny: int, steps: int = 6,
         force: bool = False) -> int:
    """Best tile configuration for this precision, limiter and size class (timed once)."""
    key = _key(precision, limiter, nx, ny)
    with _lock:
        if not force and key in _cache:
            return _cache[key]
    configs = _capi.tile_configs(precision)
    if len(configs) == 1:
        best = 0
    else:
        # The class representative: a square grid with the class's cell count.
        n = max(16, int(round(math.sqrt(2.0 ** size_class(nx, ny)))))
        prim = wl.fourier_state(n, n, 0)
        state = wl.embed(wl.to_conservative(prim, 5.0 / 3.0))
        from .mhd_solver import apply_boundary_conditions

        apply_boundary_conditions(state, n, n, 2, 0, 0)
        times = {c["config"]: _time_config(precision, limiter, n, n, c["config"], state, steps)
                 for c in configs}
        best = min(times, key=times.get)
    with _lock:
        _cache[key] = best
    return best


def _time_batch_config(precision: int, limiter: int, n: int, ni: bool, config: int,
                       steps: int) -> float:
    import torch

    from .batch import BatchSolver, fixed_params

    kw = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2,
              eta_ambipolar=1e-3) if ni else {}
    copies = max(1, min(64, (1 << 22) // (n * n)))
    b = BatchSolver(precision)
    try:
        for i in range(copies):
            sid = b.add_generated(n, n, _capi.InitSpec.fourier(i), fixed_params(
                steps + 2, limiter=limiter, **kw), (0, 0), fixed_steps=True)
            b.set_config(sid, config)
        b.step(2)  # warm-up: work lists, graph capture
        stream = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)
    finally:
        b.close()


def tune_batch(precision: int, limiter: int, nx: int, ny: int, ni: bool = False,
               steps: int = 4, force: bool = False) -> int:
    """Best batch configuration for this precision, limiter, ideal/non-ideal and size class."""
    key = "b" + _key(precision, limiter, nx, ny) + f"-n{int(bool(ni))}"
    with _lock:
        if not force and key in _cache:
            return _cache[key]
    from .batch import batch_configs

    configs = batch_configs(precision)
    if len(configs) == 1:
        best = 0
    else:
        n = max(16, int(round(math.sqrt(2.0 ** size_class(nx, ny)))))
        times = {c["config"]: _time_batch_config(precision, limiter, n, ni, c["config"], steps)
                 for c in configs}
        best = min(times, key=times.get)
    with _lock:
        _cache[key] = best
    return best


def choice(precision: int, limiter: int, nx: int, ny: int) -> int | None:
    """Cached choice, or None when this class has not been tuned."""
    with _lock:
        return _cache.get(_key(precision, limiter, nx, ny))


def save(path: str) -> None:
    with _lock:
        data = dict(_cache)
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def load(path: str) -> None:
    with open(path) as f:
        data = json.load(f)
    with _lock:
        _cache.update({str(k): int(v) for k, v in data.items()})
