"""Serving form: a request loop with continuous batching over the batched solver.

Requests (grid side, initial-state seed and kind, physics parameters, t_end) arrive over time.
The loop

* admits arrived requests while their HBM footprint (two padded FP32-mixed states) fits under
  the memory cap, by default the ones of least estimated work first and only while the running
  requests hold at most a cap of interior cells that still fills the GPU (short requests do not
  wait for the long ones they would otherwise advance beside), generating each initial state
  directly in HBM (no host state, no upload);
* advances every admitted, unfinished request together: each chunk of RK2 steps is one
  persistent launch per stage over all of them, so requests that arrive while others are on the
  GPU join the next chunk (continuous batching);
* when a request finishes, downloads its result while the next chunk runs, frees its memory and
  records its latency (completion minus arrival).

``serve_one_at_a_time`` runs the same requests through the plain FP64 single-solve path, one after
the other, as the comparison. ``make_stream`` draws a seeded request stream: Poisson arrivals,
side log-uniform, t_end uniform, Fourier or four-quadrant states 50/50, and a fraction with
Ohmic, Hall and ambipolar terms.
"""

from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from .batch import BatchSolver, state_bytes

# Non-ideal coefficients of the masked 2048^2 workload, reused for non-ideal requests.
NONIDEAL = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2,
                eta_ambipolar=1e-3)


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the stream starts
    n: int                  # square grid side
    t_end: float
    kind: str               # "fourier" or "quadrants"
    seed: int
    nonideal: bool
    gamma: float = 5.0 / 3.0
    limiter: int = _capi.VANLEER

    def params(self) -> _capi.Params:
        kw = dict(NONIDEAL) if self.nonideal else {}
        return _capi.make_params(t_end=self.t_end, gamma=self.gamma, limiter=self.limiter, **kw)

    def init(self) -> _capi.InitSpec:
        return (_capi.InitSpec.fourier(self.seed) if self.kind == "fourier"
                else _capi.InitSpec.quadrants(self.seed))

    @property
    def bc(self):
        return (0, 0) if self.kind == "fourier" else (2, 2)

    def work_estimate(self) -> float:
        """Zone-updates the request will take, estimated before it runs: cells x t_end / dt with
        dt the CFL step at a typical signal speed of its state kind (4 for the smooth Fourier
        states, 7 for the four-quadrant ones), or the non-ideal diffusion limit
        cfl h^2 / (4 eta_max) where that is smaller (the reference's dt rule, which makes the
        estimate exact for non-ideal requests)."""
        h = 1.0 / self.n
        c_h = 4.0 if self.kind == "fourier" else 7.0
        dt = 0.4 / (2.0 * c_h * self.n)
        if self.nonideal:
            eta = max(NONIDEAL["eta_ohm"], NONIDEAL["eta_hall"], NONIDEAL["eta_ambipolar"])
            dt = min(dt, 0.4 * h * h / (4.0 * eta))
        return float(self.n) * self.n * self.t_end / dt


@dataclass
class Completion:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    t: float
    cells: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def make_stream(n_requests: int, rate: float, seed: int = 0, side=(128, 2048),
                t_end=(0.1, 0.5), nonideal_frac: float = 0.3) -> list[Request]:
    """Seeded request stream: exponential inter-arrival times of mean 1/rate, side log-uniform
    in [side[0], side[1]], t_end uniform, Fourier or quadrant state with probability 1/2 each,
    non-ideal terms with probability nonideal_frac."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(side[0]), math.log(side[1])))))
        out.append(Request(rid=i, arrival=t, n=n, t_end=float(rng.uniform(*t_end)),
                           kind="fourier" if rng.uniform() < 0.5 else "quadrants",
                           seed=int(rng.integers(0, 2**31 - 1)),
                           nonideal=bool(rng.uniform() < nonideal_frac)))
    return out


class ResultBuffer:
    """One page-locked host buffer, grown to the largest result seen, that results are copied
    into before they are handed on (a fresh array per result would fault its pages in during
    every copy). Both serving paths use it, so they pay the same host-side cost."""

    def __init__(self):
        self._flat = np.empty(0, dtype=np.float64)
        self._pinned = None

    def view(self, shape) -> np.ndarray:
        n = int(np.prod(shape))
        if n > self._flat.size:
            try:
                import torch

                self._pinned = torch.empty(n, dtype=torch.float64, pin_memory=True)
                self._flat = self._pinned.numpy()
            except (ImportError, RuntimeError):
                self._pinned = None
                self._flat = np.empty(n, dtype=np.float64)
        return self._flat[:n].reshape(shape)


def _result_shape(n: int, ng: int = 2):
    return (9, n + 2 * ng, n + 2 * ng)


@dataclass
class ServeStats:
    completions: list = field(default_factory=list)
    makespan: float = 0.0
    peak_bytes: int = 0
    max_active: int = 0
    peak_cells: int = 0  # most interior cells admitted and unfinished at once
    chunks: int = 0
    joins: int = 0      # requests admitted while others were on the GPU (continuous batching)
    cap_waits: int = 0  # admission rounds in which the next request waited for memory
    cell_waits: int = 0  # admission rounds in which the next request waited for the cells cap
    states: dict = field(default_factory=dict)  # rid -> final state when kept

    def summary(self) -> dict:
        lat = np.array([c.latency for c in self.completions]) if self.completions else np.zeros(1)
        zu = float(sum(c.cells * c.steps for c in self.completions))
        return {"requests": len(self.completions), "makespan_s": self.makespan,
                "solves_per_s": len(self.completions) / self.makespan if self.makespan else 0.0,
                "zone_updates_per_s": zu / self.makespan if self.makespan else 0.0,
                "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "peak_hbm_bytes": self.peak_bytes, "max_active": self.max_active,
                "peak_active_cells": self.peak_cells,
                "chunks": self.chunks, "joined_mid_flight": self.joins,
                "admission_waits_for_memory": self.cap_waits,
                "admission_waits_for_cells": self.cell_waits}


def prepare(requests: list[Request], precision: int = _capi.FP32) -> None:
    """Tune the batch configuration of every size class the requests fall into (the batch
    autotuner caches its choices per process), so that serving does not tune on admission."""
    from . import autotune

    seen = set()
    for req in requests:
        ni = _capi.nonideal_any(req.params())
        key = (req.limiter, ni, autotune.size_class(req.n, req.n))
        if key not in seen:
            seen.add(key)
            autotune.tune_batch(precision, req.limiter, req.n, req.n, ni)


def serve(requests: list[Request], precision: int = _capi.FP32, memory_cap: float = 150e9,
          chunk: int = 16, download: bool = True, keep_states: bool = False,
          tune: bool = True, on_complete=None, order: str = "shortest",
          cells_cap: float = 64e6) -> ServeStats:
    """Serve a request stream in real time with continuous batching. tune: each request runs
    the batch configuration tuned for its size class (see prepare). on_complete(completion,
    stats) is called after each request finishes (progress records of long streams).

    Admission: a request is admitted only while the batch's HBM footprint stays under
    memory_cap. With order="shortest" the arrived requests are admitted by their estimated work
    (Request.work_estimate, smallest first) and, beyond the memory cap, only while the admitted
    unfinished requests hold at most cells_cap interior cells (at least one request always runs):
    64M cells keep the persistent batch kernels as busy as one 8k x 8k grid, and short requests no
    longer wait for the long ones they would otherwise advance beside step for step. The results
    do not depend on the order (a solve's values are the same alone and in any mix).
    order="arrival" admits in arrival order under the memory cap alone."""
    batch = BatchSolver(precision, tune=tune)
    stats = ServeStats()
    results = ResultBuffer()
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    queue: deque[Request] = deque()
    active: dict[int, tuple[Request, float]] = {}  # admitted, not finished at the last poll
    done: list = []  # (sid, request, admitted, result, poll time) finished at the last poll
    in_use = 0
    active_cells = 0
    start = time.perf_counter()
    try:
        while pending or queue or active or done:
            now = time.perf_counter() - start
            arrived = False
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
                arrived = True
            if arrived and order == "shortest":
                queue = deque(sorted(queue, key=lambda r: (r.work_estimate(), r.arrival)))
            # admission while the footprint fits under the caps
            while queue:
                req = queue[0]
                need = state_bytes(req.n, req.n)
                if in_use + need > memory_cap and (active or done):
                    stats.cap_waits += 1
                    break
                if (order == "shortest" and active
                        and active_cells + req.n * req.n > cells_cap):
                    stats.cell_waits += 1
                    break
                queue.popleft()
                if active:
                    stats.joins += 1
                sid = batch.add_generated(req.n, req.n, req.init(), req.params(), req.bc)
                in_use += need
                active_cells += req.n * req.n
                active[sid] = (req, time.perf_counter() - start)
            stats.peak_bytes = max(stats.peak_bytes, in_use)
            stats.max_active = max(stats.max_active, len(active))
            stats.peak_cells = max(stats.peak_cells, active_cells)
            if not active and not done:
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - start)))
                continue
            if active:
                batch.launch(chunk)  # the next chunk runs while finished requests leave
                stats.chunks += 1
            for sid, req, admitted, r, polled in done:
                if download or keep_states:
                    out = batch.download(sid, out=results.view(_result_shape(req.n)))
                    if keep_states:
                        stats.states[req.rid] = out.copy()
                stats.completions.append(Completion(req.rid, req.arrival, admitted,
                                                    time.perf_counter() - start if download
                                                    else polled, r.steps, r.t, req.n * req.n))
                if on_complete is not None:
                    on_complete(stats.completions[-1], stats)
                batch.remove(sid)
                in_use -= state_bytes(req.n, req.n)
            done = []
            if active:
                batch.poll()
                polled = time.perf_counter() - start
                for sid in list(active):
                    r, fin = batch.status(sid)
                    if fin:
                        req, admitted = active.pop(sid)
                        active_cells -= req.n * req.n
                        done.append((sid, req, admitted, r, polled))
        stats.makespan = time.perf_counter() - start
    finally:
        batch.close()
    return stats


def serve_one_at_a_time(requests: list[Request], precision: int = _capi.FP64,
                        download: bool = True, keep_states: bool = False) -> ServeStats:
    """The same stream through the plain single-solve path, one request at a time, in arrival
    order (a request waits until it has arrived and the previous one has finished)."""
    stats = ServeStats()
    results = ResultBuffer()
    start = time.perf_counter()
    for req in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter() - start
        if req.arrival > now:
            time.sleep(req.arrival - now)
        admitted = time.perf_counter() - start
        dev = _capi.DeviceSolver(req.n, req.n, precision=precision)
        try:
            dev.configure(*req.bc)
            params = req.params()
            dev.generate(req.init(), params)
            r = dev.solve(params)
            if download or keep_states:
                out = dev.download(out=results.view(_result_shape(req.n)))
                if keep_states:
                    stats.states[req.rid] = out.copy()
        finally:
            dev.close()
        stats.completions.append(Completion(req.rid, req.arrival, admitted,
                                            time.perf_counter() - start, r.steps, r.t,
                                            req.n * req.n))
        stats.max_active = 1
    stats.makespan = time.perf_counter() - start
    return stats
