"""Throughput benchmark of the B200 GLM-MHD backend (one JSON line on rank 0).

Workload: the smooth periodic Fourier state at 4096^2 (gamma 5/3, CFL 0.4, van Leer, ideal
GLM-MHD), seeded synthetic input. A step is one SSP-RK2 step of the whole grid; the metric is
zone-updates/s (interior cells x steps / device seconds).

* ``value``: FP32-mixed form, state resident in HBM, K timed steps bracketed by CUDA events on
  the solver's stream after W warm-up steps. The state (1.2 GB) is far larger than L2 (126 MB),
  so no flush is needed between steps. ``fp64`` reports the plain FP64 form the same way.
* ``e2e``: the same metric through the C ABI the way a caller uses it: per call, upload from
  pinned host memory, 500 RK2 steps, download to pinned host memory (bytes per step = the
  state's bytes / 500). ``e2e_dropin``: through the reference's own route, its Python module's
  MHDSolver.run with set_backend("cuda", "fp32") (MC: the module has no van Leer).
* ``fp64_mc``: the plain FP64 form with the MC limiter on the same state, the like-for-like pair
  of the reference CPU solver. ``l1_fp32_mixed_vs_fp64``: the FP32-mixed result against the FP64
  result after 500 steps of the headline state, every component.
* ``roofline``: the dominant stage kernel's algorithmic bytes per launch (9 fields x 8 B:
  stage 1 reads U and writes U*, 144 B/cell; stage 2 reads U* and U and writes U, 216 B/cell;
  360 B per zone-update) over its average event-timed duration, against the measured HBM copy
  bandwidth; ``traffic`` = that kernel's DRAM bytes per launch from the committed ncu capture of
  the same kernel kind (profiles/stage_traffic.json, bytes per cell x cells). The FP32-mixed
  increment form moves fewer bytes (72 and 180 B/cell, ``form_bytes_per_launch``); the fraction
  is still taken on the canonical bytes.
* ``cpu_baseline``: the reference CPU solver (SIMD + threads), compiled from the reference's
  own headers into oracle/_ref, on all host cores, on a bounded number of steps of the same
  4096^2 state (MC limiter: the reference has no van Leer).

* ``batched``, ``masked_nonideal``, ``served``: the batched, masked non-ideal and served
  workloads (rank 0). ``strips``: the 4096^2 grid split into 2 y strips on this GPU (strips.py)
  against the same grid as one solver.

``--impl reference`` times that reference CPU solver alone as the reference arm; it builds the
state in numpy and loads only the reference library (oracle/_ref), not this backend.
Multi-GPU: the measured operator runs replicas; each rank runs the same workload on its own GPU
and the value is the sum over ranks divided by the slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 4096
SEED = 0
GAMMA = 5.0 / 3.0
E2E_STEPS = 500
BYTES_STAGE = {1: 144.0, 2: 216.0}  # algorithmic bytes per interior cell per launch
# bytes per interior cell a stage of the FP32-mixed increment form moves (it stores the FP32
# increment instead of U*); the roofline still divides the canonical BYTES_STAGE by the time
BYTES_FORM = {"march_tma_delta": {1: 72.0, 2: 180.0}}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--e2e-calls", type=int, default=2)
    ap.add_argument("--cpu-steps", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default="fp64,fp32_mixed",
                    help="comma-separated subset of fp64,fp32_mixed (profiling runs)")
    ap.add_argument("--tile-config", default="-1",
                    help="stage-kernel tile configuration, one value for both forms or "
                         "'fp64,fp32_mixed' (-1: autotune)")
    ap.add_argument("--ref-seconds", type=float, default=60.0,
                    help="CPU time bound of the reference arm's timed sample")
    ap.add_argument("--batch-solves", type=int, default=256,
                    help="solves of the batched workload (0 skips it)")
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--masked-steps", type=int, default=300,
                    help="RK2 steps of the masked non-ideal 2048^2 leg (0 skips it)")
    ap.add_argument("--strip-steps", type=int, default=100,
                    help="RK2 steps of the 2-strip split of the 4096^2 grid (0 skips it)")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="requests of the served stream (0 skips it)")
    ap.add_argument("--serve-side", default="128,1024")
    ap.add_argument("--serve-tend", default="0.01,0.05")
    ap.add_argument("--serve-rate", type=float, default=200.0,
                    help="Poisson arrival rate of the served stream (requests/s)")
    ap.add_argument("--serve-plain-sample", type=int, default=0,
                    help="time the one-at-a-time FP64 path on this many seeded requests of the "
                         "stream and estimate the whole stream from them (0: run it all)")
    ap.add_argument("--serve-log", default=None,
                    help="file that receives one JSON line per finished served request")
    ap.add_argument("--accuracy-steps", type=int, default=500,
                    help="steps of the FP32-mixed vs FP64 L1 check at the headline size (0 skips)")
    return ap.parse_args()


def initial_state(n: int) -> np.ndarray:
    """The ghosted n^2 periodic Fourier state in the reference's StateField layout: conservative
    interior, periodic ghosts (numpy's wrap padding is the reference's x-then-y periodic fill).
    Pure numpy, so the reference arm builds it without loading the CUDA library."""
    from mhd_gpu_solver_b200 import workloads as wl

    cons = wl.to_conservative(wl.fourier_state(n, n, SEED), GAMMA)
    return np.pad(cons, ((0, 0), (2, 2), (2, 2)), mode="wrap")


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
             "clocks.mem")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        sm, mem, power, mx, reasons = [], [], [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
            try:
                power.append(float(f[3]))
                if len(f) > 9:
                    mem.append(float(f[9]))
            except ValueError:
                pass
        loaded = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": mx,
                "mem_mhz": statistics.median(mem) if mem else None,
                "power_w": statistics.median(power) if power else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def rank_device(world: int, local: int, visible: str | None):
    """(physical GPU index for nvidia-smi, CUDA_VISIBLE_DEVICES to set or None, device index to
    use). One GPU per process: with several ranks each process sees only its own GPU, so the CUDA
    runtime linked into libmhd_b200.so and torch's runtime both address it as device 0."""
    if world <= 1:
        return local, None, local
    ids = visible.split(",") if visible else [str(i) for i in range(local + 1)]
    mine = ids[local].strip()
    return (int(mine) if mine.isdigit() else local), mine, 0


def max_over_ranks(ms: float, dist=None) -> float:
    """Slowest rank's device time (ms): the whole-job time of a replicas run."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return ms
    import torch

    backend = dist.get_backend()
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(units_per_rank: float, ms_max: float, world: int) -> float:
    """Whole-job throughput of N replicas: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / (ms_max * 1e-3)


def measured_hbm_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def measured_traffic(kind: str, stage: int, cells: float):
    """DRAM bytes (read + write) of one stage launch, scaled by cells from the per-cell figure of
    the committed ncu capture of that kernel kind (traffic grows in proportion to the cells), or
    None when no capture of this kind is committed."""
    path = os.path.join(ROOT, "profiles", "stage_traffic.json")
    try:
        with open(path) as f:
            prof = json.load(f)["kinds"].get(kind)
    except (OSError, ValueError, KeyError):
        return None, None
    if prof is None:
        return None, None
    return prof["dram_bytes_per_cell"][f"stage{stage}"] * cells, prof.get("source")


def time_form(dev, params, steps: int, warmup: int, n: int) -> dict:
    """Warm-up, then K steps with per-launch events on the solver's stream."""
    import torch

    dev.solve_steps(params, warmup)
    dev.set_profiling(True)
    dev.profile_read(reset=True)
    stream = torch.cuda.ExternalStream(dev.stream())
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    launches0 = dev.launch_count()
    start.record(stream)
    dev.solve_steps(params, steps)
    end.record(stream)
    torch.cuda.synchronize()
    launches = dev.launch_count() - launches0
    ms = start.elapsed_time(end)
    prof = dev.profile_read(reset=True)
    dev.set_profiling(False)
    cells = float(n) * n
    out = {"ms": ms, "zone_updates_per_s": cells * steps / (ms * 1e-3), "launches": launches,
           "prof": prof}
    for stg in (1, 2):
        k = prof[f"stage{stg}_launches"]
        avg = prof[f"stage{stg}_ms"] / k if k else float("nan")
        out[f"stage{stg}_avg_ms"] = avg
        out[f"stage{stg}_gbs"] = BYTES_STAGE[stg] * cells / (avg * 1e-3) / 1e9 if k else None
    return out


def e2e_form(dev, params, host: np.ndarray, calls: int, n: int) -> dict:
    """upload (pinned host) -> 500 steps -> download (pinned host), timed on the stream."""
    import torch

    stream = torch.cuda.ExternalStream(dev.stream())
    dev.upload(host)
    dev.solve_steps(params, 40)  # warm-up: captures the 32-step graph batch
    dev.download(host)
    total = 0.0
    for _ in range(calls):
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        dev.upload(host)
        dev.solve_steps(params, E2E_STEPS)
        dev.download(host)
        end.record(stream)
        torch.cuda.synchronize()
        total += start.elapsed_time(end)
    nbytes = int(host.nbytes)
    return {"value": float(n) * n * E2E_STEPS * calls / (total * 1e-3), "unit": "zone-updates/s",
            "h2d_bytes_per_step": nbytes / E2E_STEPS, "d2h_bytes_per_step": nbytes / E2E_STEPS,
            "bytes_per_call": nbytes, "steps_per_call": E2E_STEPS, "calls": calls}


def e2e_dropin(n: int, calls: int, steps_per_call: int = E2E_STEPS) -> dict:
    """The same metric through the reference's own drop-in route: its Python module
    (python/mhd_pybind.cpp compiled with this backend in its CUDA seam, oracle/_ref) with
    MHDSolver.set_backend("cuda", "fp32") and MHDSolver.run(dt), which per call configures,
    uploads the host StateField, solves to the time and downloads (include/mhd/solver_api.hpp:
    294-321). The module offers minmod and MC only, so MC. The call is synchronous (it returns
    after the download), so it is timed by the host clock between device synchronisations."""
    import glob
    import importlib

    import torch

    from mhd_gpu_solver_b200 import workloads as wl

    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not glob.glob(os.path.join(ref_dir, "mhd_solver*.so")):
        return {"unavailable": "reference module with this backend not built (oracle/_ref)"}
    sys.path.insert(0, ref_dir)
    try:
        ms = importlib.import_module("mhd_solver")
    finally:
        sys.path.remove(ref_dir)
    prim = wl.fourier_state(n, n, SEED)
    s = ms.MHDSolver(n, n)
    s.set_periodic_bc()
    s.set_gamma(GAMMA)
    s.set_cfl(0.4)
    s.set_glm_alpha(0.1)
    s.set_limiter_mc()
    s.set_primitives(prim["rho"], prim["vx"], prim["vy"], prim["vz"], prim["p"], prim["bx"],
                     prim["by"], prim["bz"], prim["psi"])
    s.set_backend("cuda", "fp32")
    r0 = s.run(1e-6)  # warm-up: device object, kernel attributes
    # about steps_per_call steps per run() at the CFL step of the current signal speed
    t_call = steps_per_call * 0.4 / (r0.c_h * n + r0.c_h * n)
    s.run(t_call)  # warm-up at full length: graph capture
    total, steps = 0.0, 0
    for _ in range(calls):
        k0 = s.steps
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.run(t_call)
        torch.cuda.synchronize()
        total += time.perf_counter() - t0
        steps += s.steps - k0
    nbytes = 9 * (n + 4) * (n + 4) * 8
    return {"value": float(n) * n * steps / total, "unit": "zone-updates/s",
            "route": "reference mhd_solver module, MHDSolver.run, backend cuda/fp32, MC",
            "steps_per_call": steps / calls, "calls": calls,
            "h2d_bytes_per_step": nbytes * calls / steps, "d2h_bytes_per_step": nbytes * calls / steps,
            "device": s.backend_device()}


def accuracy_leg(host: np.ndarray, n: int, params, steps: int = 500) -> dict:
    """The FP32-mixed result against the FP64 result after `steps` steps of the same n^2 state
    (the headline workload), per component (mhd_gpu_solver_b200.accuracy.component_l1)."""
    from mhd_gpu_solver_b200 import _capi
    from mhd_gpu_solver_b200.accuracy import COMPONENTS, component_l1

    outs = {}
    for name, prec in (("fp64", _capi.FP64), ("fp32_mixed", _capi.FP32)):
        dev = _capi.DeviceSolver(n, n, precision=prec)
        try:
            dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
            dev.upload(host)
            r = dev.solve_steps(params, steps)
            outs[name] = (dev.download(), r)
        finally:
            dev.close()
    (u64, r64), (u32, r32) = outs["fp64"], outs["fp32_mixed"]
    err = component_l1(u32, u64, r64.c_h)
    return {"steps": steps, "same_step_count": r64.steps == r32.steps == steps,
            "t_rel_diff": abs(r32.t - r64.t) / r64.t, "max": float(np.max(err)),
            "per_component": {c: float(e) for c, e in zip(COMPONENTS, err)},
            "rule": "relative L1 per component (absolute where FP64 is identically zero), "
                    "psi on max(sum|psi|, c_h sum|B|)"}


def bench_batched(nsolves: int, steps: int, seed: int = 1) -> dict:
    """256 independent ideal solves, nx and ny each log-uniform in [64, 1024], own seeded Fourier
    state (generated on the device) and own gamma ~ U[1.4, 5/3], periodic, van Leer, fixed step
    count, FP32-mixed batch. Also runs the same solves as an FP64 batch (the per-solve L1
    reference) and one at a time through the single-solve FP32-mixed path."""
    import math

    import torch

    from mhd_gpu_solver_b200 import _capi
    from mhd_gpu_solver_b200.batch import BatchSolver, fixed_params

    rng = np.random.Generator(np.random.PCG64(seed))
    solves = []
    for i in range(nsolves):
        nx = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        ny = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        solves.append((nx, ny, float(rng.uniform(1.4, 5.0 / 3.0)), int(rng.integers(0, 2**31 - 1))))
    cells = sum(nx * ny for nx, ny, _, _ in solves)

    def run(precision):
        b = BatchSolver(precision, tune=True)  # the warm-up build tunes every size class
        ids = [b.add_generated(nx, ny, _capi.InitSpec.fourier(sd),
                               fixed_params(steps, gamma=g, limiter=_capi.VANLEER), (0, 0),
                               fixed_steps=True) for nx, ny, g, sd in solves]
        b.step(2)  # warm-up: kernel attributes, first graph capture
        # rebuild the same batch and time it from the start
        b.close()
        b = BatchSolver(precision, tune=True)
        ids = [b.add_generated(nx, ny, _capi.InitSpec.fourier(sd),
                               fixed_params(steps, gamma=g, limiter=_capi.VANLEER), (0, 0),
                               fixed_steps=True) for nx, ny, g, sd in solves]
        stream = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        while b.step(steps) > 0:
            pass
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        launches = b.info()["launches"]
        return b, ids, ms, launches

    bm, idm, ms_m, launches = run(_capi.FP32)
    b64, id64, ms_64, _ = run(_capi.FP64)
    from mhd_gpu_solver_b200.accuracy import component_l1

    errs = []
    for (nx, ny, g, sd), a, c in zip(solves, idm, id64):
        um, u64 = bm.download(a), b64.download(c)
        errs.append(float(np.max(component_l1(um, u64, b64.status(c)[0].c_h,
                                              vector_scale=True))))
    bm.close()
    b64.close()
    # one at a time through the single-solve FP32-mixed path
    t0 = time.perf_counter()
    for nx, ny, g, sd in solves:
        dev = _capi.DeviceSolver(nx, ny, precision=_capi.FP32)
        dev.configure(0, 0)
        p = _capi.make_params(gamma=g, limiter=_capi.VANLEER)
        dev.generate(_capi.InitSpec.fourier(sd), p)
        dev.solve_steps(p, steps)
        dev.close()
    one_s = time.perf_counter() - t0
    return {"workload": f"{nsolves} ideal solves, nx, ny log-uniform in [64,1024], {steps} steps",
            "cells": cells, "solves_per_s": nsolves / (ms_m * 1e-3),
            "zone_updates_per_s": cells * steps / (ms_m * 1e-3), "ms": ms_m,
            "fp64_batch_solves_per_s": nsolves / (ms_64 * 1e-3),
            "one_at_a_time_fp32_mixed_solves_per_s": nsolves / one_s,
            "l1_fp32_mixed_vs_fp64": {"max": max(errs), "median": float(np.median(errs))},
            "gpu_launches": launches}


def bench_strips(U: np.ndarray, n: int, steps: int, count: int = 2) -> dict:
    """The n^2 periodic Fourier grid split into `count` y strips on this GPU (strips.py: one
    solver and stream per strip, 6 overlap rows, combined CFL maximum and overlap-row copies on
    the device, stepped by the host), FP32-mixed, against the same grid as one solver. Device
    time on the host stream that waits for every strip; the strips' host loop is inside it."""
    import torch

    from mhd_gpu_solver_b200 import _capi
    from mhd_gpu_solver_b200.strips import OVERLAP, StripSolver

    params = _capi.make_params(cfl=0.4, gamma=GAMMA, glm_alpha=0.1, limiter=_capi.VANLEER)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    with StripSolver(n, n, _capi.FP32, strips=count, distributed=False) as ss:
        ss.upload(U)
        ss.solve_steps(params, 3)  # warm-up: kernel attributes, stream waits
        ss.upload(U)
        main = torch.cuda.current_stream()
        e0, e1 = ev(), ev()
        torch.cuda.synchronize()
        e0.record(main)
        r = ss.solve_steps(params, steps)
        for e in ss.engines:
            main.wait_stream(e.stream)
        e1.record(main)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        split = ss.gather()
    dev = _capi.DeviceSolver(n, n, precision=_capi.FP32)
    try:
        dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
        dev.upload(U)
        dev.solve_steps(params, 40)  # warm-up: captures the 32-step graph batch
        dev.upload(U)
        stream = torch.cuda.ExternalStream(dev.stream())
        w0, w1 = ev(), ev()
        torch.cuda.synchronize()
        w0.record(stream)
        dev.solve_steps(params, steps)
        w1.record(stream)
        torch.cuda.synchronize()
        ms_whole = w0.elapsed_time(w1)
        whole = dev.download()[:, 2:-2, 2:-2]
    finally:
        dev.close()
    from mhd_gpu_solver_b200.accuracy import component_l1

    l1 = component_l1(split, whole, r[2], ng=0)
    cells = float(n) * n * steps
    return {"workload": f"{n}^2 periodic Fourier, FP32-mixed, van Leer, {count} y strips of "
                        f"{n // count} rows + {OVERLAP} overlap rows per side on one GPU, "
                        f"{steps} steps",
            "zone_updates_per_s": cells / (ms * 1e-3), "ms": ms, "steps": r[1],
            "whole_grid_zone_updates_per_s": cells / (ms_whole * 1e-3),
            "ratio_to_whole_grid": ms_whole / ms,
            "exchange_bytes_per_step": 2 * count * OVERLAP * n * 18 * 4,
            "l1_vs_whole_grid_max": float(np.max(l1))}


def bench_masked_nonideal(n: int, steps: int, seed: int = 3) -> dict:
    """The non-ideal, masked workload: n^2, the seeded Fourier state and mask (both generated on
    the device), Ohmic 1e-3, Hall 1e-2, ambipolar 1e-3, 12 circles and 6 rectangles of reflective
    walls, outflow in x and periodic in y, van Leer, `steps` RK2 steps, FP64 plain vs FP32-mixed
    (both on their masked default kernels, the masked TMA strip marches). Reports each form's
    zone-updates/s, the FP32-mixed L1 error against the FP64 result (every component), and the
    FP64 div-B norms and mass/energy drift."""
    import torch

    from mhd_gpu_solver_b200 import _capi
    from mhd_gpu_solver_b200 import workloads as wl

    shapes = wl.circles_and_rectangles_shapes(seed)  # rasterised on the device
    params = _capi.make_params(limiter=_capi.VANLEER, ohmic=True, hall=True, ambipolar=True,
                               eta_ohm=1e-3, eta_hall=1e-2, eta_ambipolar=1e-3)
    out, states = {}, {}
    for name, prec in (("fp64", _capi.FP64), ("fp32_mixed", _capi.FP32)):
        dev = _capi.DeviceSolver(n, n, precision=prec)
        try:
            dev.configure_shapes(_capi.BC_OUTFLOW, _capi.BC_PERIODIC, shapes, True)
            dev.generate(_capi.InitSpec.fourier(seed), params)
            d0 = dev.diagnostics(params)
            dev.solve_steps(params, 40)  # warm-up: kernel attributes, the 32-step graph batch
            dev.generate(_capi.InitSpec.fourier(seed), params)
            stream = torch.cuda.ExternalStream(dev.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            r = dev.solve_steps(params, steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            d1 = dev.diagnostics(params)
            states[name] = dev.download()
            if name == "fp64":
                c_h64 = r.c_h
        finally:
            dev.close()
        out[name] = {"zone_updates_per_s": float(n) * n * steps / (ms * 1e-3), "ms": ms,
                     "steps": r.steps, "t": r.t,
                     "div_b_l2": d1["div_b_l2"], "div_b_max": d1["div_b_max"],
                     "mass_drift": (d1["mass"] - d0["mass"]) / d0["mass"],
                     "energy_drift": (d1["energy"] - d0["energy"]) / d0["energy"]}
    from mhd_gpu_solver_b200.accuracy import COMPONENTS, component_l1

    l1 = component_l1(states["fp32_mixed"], states["fp64"], c_h64)
    l1v = component_l1(states["fp32_mixed"], states["fp64"], c_h64, vector_scale=True)
    out["workload"] = (f"{n}^2 masked (12 circles, 6 rectangles, reflective walls), Ohmic/Hall/"
                       f"ambipolar 1e-3/1e-2/1e-3, outflow x, periodic y, van Leer, {steps} steps")
    out["speedup_fp32_mixed_over_fp64"] = out["fp64"]["ms"] / out["fp32_mixed"]["ms"]
    out["l1_fp32_mixed_vs_fp64_max"] = float(np.max(l1v))
    out["l1_fp32_mixed_vs_fp64"] = {
        "relative": {c: float(e) for c, e in zip(COMPONENTS, l1)},
        "vector_scale": {c: float(e) for c, e in zip(COMPONENTS, l1v)},
        "rule": "max: every component, m and B components on their vector's scale"}
    return out


def bench_served(nreq: int, side, tend, rate: float, plain_sample: int = 0,
                 log_path: str | None = None) -> dict:
    """The served stream: seeded Poisson arrivals at `rate`, FP32-mixed continuous batching
    under the 150 GB cap, against the plain FP64 path one request at a time. With plain_sample >
    0 the plain path runs a seeded random subsample of that many requests (first, back to back)
    and its time for the whole stream is estimated by a least-squares fit of per-request seconds
    = a + b x zone-updates over the sample, summed over every request (the plain path's requests
    run back to back at a saturating rate, so its makespan is that sum). log_path: one JSON line
    per finished request (and the plain estimate), written as the run goes."""
    from mhd_gpu_solver_b200.serve import make_stream, prepare, serve, serve_one_at_a_time

    log = open(log_path, "a", buffering=1) if log_path else None

    def note(obj):
        if log is not None:
            log.write(json.dumps(obj) + "\n")

    stream = make_stream(nreq, rate=rate, seed=2, side=side, t_end=tend, nonideal_frac=0.3)
    out = {"workload": f"{nreq} requests, Poisson arrivals at {rate:g}/s, side "
                       f"log-uniform in [{side[0]},{side[1]}], t_end ~ U[{tend[0]},{tend[1]}], "
                       "Fourier or four-quadrant 50/50, 30% non-ideal, FP32-mixed, 150 GB cap"}
    sample = None
    if 0 < plain_sample < nreq:
        import copy

        rng = np.random.Generator(np.random.PCG64(11))
        pick = sorted(rng.choice(nreq, size=plain_sample, replace=False).tolist())
        sample = [copy.copy(stream[i]) for i in pick]
        for r in sample:
            r.arrival = 0.0  # back to back: the plain path is the bottleneck at a saturating rate
        ps = serve_one_at_a_time(sample)
        note({"plain_sample_done": plain_sample, "seconds": ps.makespan})
    prepare(stream)  # batch autotuning of the stream's size classes, outside the timed run
    stats = serve(stream, on_complete=lambda c, st: note(
        {"rid": c.rid, "n": int(round(c.cells ** 0.5)), "steps": c.steps, "arrival": c.arrival,
         "finished": c.finished, "latency_s": c.latency, "done": len(st.completions)}))
    served = stats.summary()
    out["served"] = served
    note({"served": served})
    if sample is None:
        plain = serve_one_at_a_time(stream).summary()
        out["one_at_a_time_fp64"] = plain
        out["solves_per_s_ratio"] = served["solves_per_s"] / plain["solves_per_s"]
        return out
    work = {c.rid: c.cells * c.steps for c in stats.completions}
    secs = np.array([c.finished - c.admitted for c in ps.completions])
    zu = np.array([float(work[c.rid]) for c in ps.completions])
    A = np.stack([np.ones_like(zu), zu], axis=1)
    (a, b), *_ = np.linalg.lstsq(A, secs, rcond=None)
    est = float(sum(a + b * w for w in work.values()))
    out["one_at_a_time_fp64"] = {
        "method": f"{plain_sample} seeded random requests of the stream run back to back; "
                  "per-request seconds fitted as a + b x zone-updates (least squares) and summed "
                  "over all requests",
        "sample_requests": plain_sample, "sample_seconds": float(secs.sum()),
        "sample_zone_updates": float(zu.sum()), "fit_a_s": float(a), "fit_b_s": float(b),
        "estimated_makespan_s": est, "solves_per_s": nreq / est}
    out["solves_per_s_ratio"] = served["solves_per_s"] / (nreq / est)
    note({"result": out})
    return out


def cpu_reference_rate(U: np.ndarray, n: int, steps: int) -> dict:
    from oracle import oracle as orc

    threads = os.cpu_count() or 1
    orc.ref_set_threads(threads)
    p = orc.Params(cfl=0.4, gamma=GAMMA, glm_alpha=0.1, limiter=orc.MC, max_steps=1,
                   fixed_steps=True)
    orc.solve(U, orc.Grid(n, n), p, impl="ref")  # warm-up (thread pool, page faults)
    p.max_steps = steps
    orc.solve(U, orc.Grid(n, n), p, impl="ref")
    dt = orc.ref_last_loop_seconds()
    return {"value": float(n) * n * steps / dt, "unit": "zone-updates/s", "cores": threads,
            "kind": "reference", "simd": orc.ref_simd_backend(), "seconds": dt,
            "sample": f"{steps} SSP-RK2 steps of the {n}^2 periodic Fourier state, MC limiter "
                      f"(the reference has no van Leer), reference CPU solver with "
                      f"{orc.ref_simd_backend()} and {threads} threads"}


def run_reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    from oracle import oracle as orc

    n = args.n
    if orc.ref_library_path() is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU library not built"}))
        return
    U = initial_state(n)
    threads = os.cpu_count() or 1
    orc.ref_set_threads(threads)
    p = orc.Params(cfl=0.4, gamma=GAMMA, glm_alpha=0.1, limiter=orc.MC, max_steps=1,
                   fixed_steps=True)
    p.max_steps = max(1, args.warmup)
    state, *_ = orc.solve(U, orc.Grid(n, n), p, impl="ref")
    # Bound the timed sample: as many of the K steps as fit in --ref-seconds at the warm-up rate.
    per_step = orc.ref_last_loop_seconds() / p.max_steps
    timed = max(1, min(args.steps, int(args.ref_seconds / max(per_step, 1e-9))))
    p.max_steps = timed
    orc.solve(state, orc.Grid(n, n), p, impl="ref")
    dt = orc.ref_last_loop_seconds()
    value = float(n) * n * timed / dt
    sample = (f"{timed} of the {args.steps} requested SSP-RK2 steps (bounded to about "
              f"{args.ref_seconds:.0f} s of CPU work) of the {n}^2 periodic Fourier state after "
              f"{args.warmup} warm-up steps, step loop timed alone, MC limiter (no van Leer in "
              f"the reference), {orc.ref_simd_backend()}, {threads} threads")
    line = {"metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "steps_timed": timed, "ms_per_step": dt * 1e3 / timed,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"fourier_periodic_{n}x{n}", "grid": [n, n],
                       "limiter": "MC", "parallelism": "cpu-threads"},
            "cpu_baseline": {"value": value, "unit": "zone-updates/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch

    phys, visible, index = rank_device(world, local, os.environ.get("CUDA_VISIBLE_DEVICES"))
    if visible is not None:
        os.environ["CUDA_VISIBLE_DEVICES"] = visible
    torch.cuda.set_device(index)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from mhd_gpu_solver_b200 import _capi

    n = args.n
    U = initial_state(n)
    host = torch.empty(U.shape, dtype=torch.float64, pin_memory=True).numpy()
    host[...] = U
    params = _capi.make_params(cfl=0.4, gamma=GAMMA, glm_alpha=0.1, limiter=_capi.VANLEER)
    params_mc = _capi.make_params(cfl=0.4, gamma=GAMMA, glm_alpha=0.1, limiter=_capi.MC)

    results = {}
    # the headline form first, on a GPU that has not yet run the FP64 form
    forms = [f for f in (("fp32_mixed", _capi.FP32), ("fp64", _capi.FP64))
             if f[0] in args.forms.split(",")]
    from mhd_gpu_solver_b200 import autotune

    chosen = {}
    cfgs = [int(v) for v in args.tile_config.split(",")]
    cfg_of = {"fp64": cfgs[0], "fp32_mixed": cfgs[-1]}
    for name, prec in forms:
        cfg = cfg_of[name]
        if cfg < 0:
            cfg = autotune.tune(prec, _capi.VANLEER, n, n)
        chosen[name] = cfg
        dev = _capi.DeviceSolver(n, n, precision=prec)
        dev.set_tile_config(cfg)
        dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
        dev.upload(host)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        if name == "fp32_mixed":
            with ClockSampler(phys) as clk:
                r = time_form(dev, params, args.steps, args.warmup, n)
            r["clocks"] = clk.summary()
        else:
            r = time_form(dev, params, args.steps, args.warmup, n)
        r["ms_max"] = max_over_ranks(r["ms"], dist)
        if name == "fp32_mixed" and args.e2e_calls > 0:
            r["e2e"] = e2e_form(dev, params, host, args.e2e_calls, n)
        dev.close()
        results[name] = r
    if "fp64" in results and "fp64" in args.forms.split(","):
        # like-for-like with the reference CPU solver: FP64, MC, the same state
        dev = _capi.DeviceSolver(n, n, precision=_capi.FP64)
        dev.configure(_capi.BC_PERIODIC, _capi.BC_PERIODIC)
        dev.upload(host)
        r = time_form(dev, params_mc, args.steps, args.warmup, n)
        r["ms_max"] = max_over_ranks(r["ms"], dist)
        dev.close()
        results["fp64_mc"] = r
    if "fp32_mixed" not in results or "fp64" not in results:
        if rank == 0:  # profiling run: no JSON line
            print(json.dumps({k: {kk: vv for kk, vv in v.items() if kk != "prof"}
                              for k, v in results.items()}))
        if dist is not None:
            dist.destroy_process_group()
        return

    mixed = results["fp32_mixed"]
    ms = mixed["ms_max"]
    value = replicas_value(float(n) * n * args.steps, ms, world)
    peak, peak_kind = measured_hbm_peak()
    dom = 2 if mixed["prof"]["stage2_ms"] >= mixed["prof"]["stage1_ms"] else 1
    achieved = mixed[f"stage{dom}_gbs"]
    mixed_cfg = next(c for c in _capi.tile_configs(_capi.FP32) if c["config"] == chosen["fp32_mixed"])
    traffic, traffic_src = measured_traffic(mixed_cfg["kind"], dom, float(n) * n)
    line = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"fourier_periodic_{n}x{n}", "grid": [n, n], "form": "fp32_mixed",
                   "limiter": "van Leer", "gamma": GAMMA, "cfl": 0.4, "seed": SEED,
                   "parallelism": f"replicas{world}",
                   "l2": "state 1.21 GB per buffer >> 126 MB L2, no flush"},
        "tile_configs": {k: next(c for c in _capi.tile_configs(p) if c["config"] == chosen[k])
                         for k, p in (("fp64", _capi.FP64), ("fp32_mixed", _capi.FP32))},
        "fp64": {"value": replicas_value(float(n) * n * args.steps, results["fp64"]["ms_max"], world),
                 "ms_per_step": results["fp64"]["ms_max"] / args.steps,
                 "stage1_avg_ms": results["fp64"]["stage1_avg_ms"],
                 "stage2_avg_ms": results["fp64"]["stage2_avg_ms"],
                 "stage2_gbs": results["fp64"]["stage2_gbs"]},
        "fp64_mc": {"value": replicas_value(float(n) * n * args.steps,
                                            results["fp64_mc"]["ms_max"], world),
                    "ms_per_step": results["fp64_mc"]["ms_max"] / args.steps,
                    "stage1_avg_ms": results["fp64_mc"]["stage1_avg_ms"],
                    "stage2_avg_ms": results["fp64_mc"]["stage2_avg_ms"],
                    "note": "FP64, MC limiter, same state: the like-for-like pair of the "
                            "reference CPU solver (cpu_baseline, the reference arm)"},
        "speedup_fp32_mixed_over_fp64": results["fp64"]["ms_max"] / ms,
        "roofline": {"bound": "hbm", "kernel": f"stage{dom} (fp32_mixed)", "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "algorithmic_bytes_per_launch": BYTES_STAGE[dom] * n * n,
                     "form_bytes_per_launch": (BYTES_FORM[mixed_cfg["kind"]][dom] * n * n
                                               if mixed_cfg["kind"] in BYTES_FORM else None),
                     "stage1_avg_ms": mixed["stage1_avg_ms"],
                     "stage2_avg_ms": mixed["stage2_avg_ms"]},
        "clocks": mixed["clocks"],
        "e2e": mixed.get("e2e"),
        "gpu_launches": mixed["launches"],
    }
    if rank == 0 and args.accuracy_steps > 0:
        line["l1_fp32_mixed_vs_fp64"] = accuracy_leg(host, n, params, args.accuracy_steps)
    if rank == 0 and args.e2e_calls > 0:
        line["e2e_dropin"] = e2e_dropin(n, args.e2e_calls)
    if rank == 0 and args.batch_solves > 0:
        line["batched"] = bench_batched(args.batch_solves, args.batch_steps)
    if rank == 0 and args.masked_steps > 0:
        line["masked_nonideal"] = bench_masked_nonideal(2048, args.masked_steps)
    if rank == 0 and args.strip_steps > 0:
        line["strips"] = bench_strips(U, n, args.strip_steps)
    if rank == 0 and args.serve_requests > 0:
        side = tuple(int(v) for v in args.serve_side.split(","))
        tend = tuple(float(v) for v in args.serve_tend.split(","))
        line["served"] = bench_served(args.serve_requests, side, tend, args.serve_rate,
                                      args.serve_plain_sample, args.serve_log)
    if rank == 0 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_reference_rate(U, n, args.cpu_steps)
        except (FileNotFoundError, OSError) as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
