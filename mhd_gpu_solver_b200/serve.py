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

``serve`` replays a request stream with given arrival times; ``Server`` is the online form (a
worker thread runs the same engine while requests are submitted from any thread, with
submit/poll/result/summary). ``serve_one_at_a_time`` runs the same requests through the plain
FP64 single-solve path, one after the other, as the comparison. ``make_stream`` draws a seeded request stream: Poisson arrivals,
side log-uniform, t_end uniform, Fourier or four-quadrant states 50/50, and a fraction with
Ohmic, Hall and ambipolar terms.
"""

from __future__ import annotations

import math
import threading
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


class _Engine:
    """The continuous-batching core shared by serve() and Server: admission under the memory
    and cells caps, chunked advance of every admitted request, completion of finished ones. All
    of its calls come from one thread."""

    def __init__(self, precision: int, memory_cap: float, chunk: int, download: bool,
                 keep_states: bool, tune: bool, order: str, cells_cap: float, stats: ServeStats,
                 on_complete=None, start: float | None = None, batch=None):
        if order not in ("shortest", "arrival"):
            raise ValueError(f"unknown admission order {order!r}")
        # batch: the BatchSolver to drive (default: a new one; host tests pass a stand-in)
        self.batch = BatchSolver(precision, tune=tune) if batch is None else batch
        self.results = ResultBuffer()
        self.memory_cap, self.chunk, self.download = memory_cap, chunk, download
        self.keep_states, self.order, self.cells_cap = keep_states, order, cells_cap
        self.stats = stats
        self.on_complete = on_complete
        self.active: dict[int, tuple[Request, float]] = {}  # admitted, not finished at last poll
        self.done: list = []  # (sid, request, admitted, result, poll time) finished at last poll
        self.in_use = 0
        self.active_cells = 0
        self.start = time.perf_counter() if start is None else start  # the clock's origin

    def clock(self) -> float:
        return time.perf_counter() - self.start

    @property
    def busy(self) -> bool:
        return bool(self.active or self.done)

    def order_queue(self, queue: deque) -> deque:
        if self.order == "shortest":
            return deque(sorted(queue, key=lambda r: (r.work_estimate(), r.arrival)))
        return queue

    def admit(self, queue: deque) -> None:
        """Admit queued requests, in queue order, while the footprint fits under the caps (one
        request always runs)."""
        stats = self.stats
        while queue:
            req = queue[0]
            need = state_bytes(req.n, req.n)
            if self.in_use + need > self.memory_cap and self.busy:
                stats.cap_waits += 1
                break
            if (self.order == "shortest" and self.active
                    and self.active_cells + req.n * req.n > self.cells_cap):
                stats.cell_waits += 1
                break
            queue.popleft()
            if self.active:
                stats.joins += 1
            sid = self.batch.add_generated(req.n, req.n, req.init(), req.params(), req.bc)
            self.in_use += need
            self.active_cells += req.n * req.n
            self.active[sid] = (req, self.clock())
        stats.peak_bytes = max(stats.peak_bytes, self.in_use)
        stats.max_active = max(stats.max_active, len(self.active))
        stats.peak_cells = max(stats.peak_cells, self.active_cells)

    def advance(self) -> list[Completion]:
        """One round: issue the next chunk of steps, hand on the requests that had finished at
        the previous poll while it runs, then wait for the chunk and note the newly finished.
        Returns the completions handed on."""
        stats, batch = self.stats, self.batch
        if self.active:
            batch.launch(self.chunk)  # the next chunk runs while finished requests leave
            stats.chunks += 1
        out = []
        for sid, req, admitted, r, polled in self.done:
            if self.download or self.keep_states:
                state = batch.download(sid, out=self.results.view(_result_shape(req.n)))
                if self.keep_states:
                    stats.states[req.rid] = state.copy()
            c = Completion(req.rid, req.arrival, admitted,
                           self.clock() if self.download else polled, r.steps, r.t,
                           req.n * req.n)
            stats.completions.append(c)
            out.append(c)
            if self.on_complete is not None:
                self.on_complete(c, stats)
            batch.remove(sid)
            self.in_use -= state_bytes(req.n, req.n)
        self.done = []
        if self.active:
            batch.poll()
            polled = self.clock()
            for sid in list(self.active):
                r, fin = batch.status(sid)
                if fin:
                    req, admitted = self.active.pop(sid)
                    self.active_cells -= req.n * req.n
                    self.done.append((sid, req, admitted, r, polled))
        return out

    def close(self) -> None:
        self.batch.close()


def serve(requests: list[Request], precision: int = _capi.FP32, memory_cap: float = 150e9,
          chunk: int = 16, download: bool = True, keep_states: bool = False,
          tune: bool = True, on_complete=None, order: str = "shortest",
          cells_cap: float = 64e6, engine_factory=None) -> ServeStats:
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
    order="arrival" admits in arrival order under the memory cap alone. engine_factory(stats)
    replaces the GPU engine (host tests, as for Server)."""
    stats = ServeStats()
    if engine_factory is None:
        eng = _Engine(precision, memory_cap, chunk, download, keep_states, tune, order,
                      cells_cap, stats, on_complete)
    else:
        eng = engine_factory(stats)
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    queue: deque[Request] = deque()
    eng.start = time.perf_counter()
    try:
        while pending or queue or eng.busy:
            now = eng.clock()
            arrived = False
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
                arrived = True
            if arrived:
                queue = eng.order_queue(queue)
            eng.admit(queue)
            if not eng.busy:
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - eng.clock()))
                continue
            eng.advance()
        stats.makespan = eng.clock()
    finally:
        eng.close()
    return stats


class Server:
    """Online serving: requests are submitted from any thread while a worker thread runs the
    continuous-batching engine of serve() (same admission policy, chunked advance, download of
    finished requests while the next chunk runs).

    ``submit`` returns a request id; ``poll(timeout)`` returns the completions since the last
    poll, waiting up to ``timeout`` seconds for one; ``result(rid)`` hands over the final
    ghosted state (9, n + 4, n + 4) of a completed request (``keep_states``); ``summary()`` gives
    latency percentiles and throughput so far (latency counts from submission); ``close()``
    stops taking requests, lets the submitted ones finish and stops the worker. A failed solve
    (max_steps, a bad dt, a CUDA error) stops the worker; later calls raise its error.

    ``engine_factory`` replaces the GPU engine (a callable of the ServeStats returning an object
    with admit, advance, order_queue, busy and close; for testing the threading on a host)."""

    def __init__(self, precision: int = _capi.FP32, memory_cap: float = 150e9, chunk: int = 16,
                 order: str = "shortest", cells_cap: float = 64e6, tune: bool = True,
                 keep_states: bool = True, engine_factory=None):
        self.stats = ServeStats()
        self._cond = threading.Condition()
        self._incoming: deque[Request] = deque()
        self._completed: list[Completion] = []
        self._closing = False
        self._stopped = False
        self._error: BaseException | None = None
        self._next_rid = 0
        self._start = time.perf_counter()
        if engine_factory is None:
            def engine_factory(stats):
                return _Engine(precision, memory_cap, chunk, True, keep_states, tune, order,
                               cells_cap, stats, start=self._start)
        self._factory = engine_factory
        self._ready = threading.Event()
        self._thread = threading.Thread(target=self._run, name="mhdb-server", daemon=True)
        self._thread.start()
        self._ready.wait()
        if self._error is not None:
            raise RuntimeError(f"server start failed: {self._error}") from self._error

    def _clock(self) -> float:
        return time.perf_counter() - self._start

    def _raise_if_failed(self) -> None:
        if self._error is not None:
            raise RuntimeError(f"serving stopped: {self._error}") from self._error

    def submit(self, n: int, t_end: float, kind: str = "fourier", seed: int = 0,
               nonideal: bool = False, limiter: int = _capi.VANLEER,
               gamma: float = 5.0 / 3.0) -> int:
        """Queue a request (square grid of side n, seeded Fourier or four-quadrant state, solved
        to t_end); returns its id."""
        if kind not in ("fourier", "quadrants"):
            raise ValueError(f"unknown initial state {kind!r}")
        if int(n) < 1 or not t_end > 0.0:
            raise ValueError("n must be positive and t_end > 0")
        with self._cond:
            if self._closing:
                raise RuntimeError("server is closed")
            self._raise_if_failed()
            rid = self._next_rid
            self._next_rid += 1
            self._incoming.append(Request(rid, self._clock(), int(n), float(t_end), kind,
                                          int(seed), bool(nonideal), float(gamma), int(limiter)))
            self._cond.notify_all()
        return rid

    def poll(self, timeout: float = 0.0) -> list[Completion]:
        """Completions since the last poll (waits up to timeout seconds for the first one)."""
        with self._cond:
            if not self._completed and timeout > 0.0:
                self._cond.wait_for(lambda: self._completed or self._stopped, timeout)
            out, self._completed = self._completed, []
            if not out:
                self._raise_if_failed()
        return out

    def result(self, rid: int) -> np.ndarray:
        """The final state of a completed request (kept until it is taken)."""
        with self._cond:
            if rid not in self.stats.states:
                raise KeyError(f"no kept result for request {rid}")
            return self.stats.states.pop(rid)

    def summary(self) -> dict:
        with self._cond:
            snap = ServeStats(completions=list(self.stats.completions),
                              makespan=self._clock(), peak_bytes=self.stats.peak_bytes,
                              max_active=self.stats.max_active, peak_cells=self.stats.peak_cells,
                              chunks=self.stats.chunks, joins=self.stats.joins,
                              cap_waits=self.stats.cap_waits, cell_waits=self.stats.cell_waits)
        out = snap.summary()
        out["submitted"] = self._next_rid
        return out

    def close(self) -> None:
        with self._cond:
            self._closing = True
            self._cond.notify_all()
        self._thread.join()
        self._raise_if_failed()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _run(self) -> None:
        try:
            eng = self._factory(self.stats)
        except BaseException as e:  # reported by the constructor
            self._error = e
            self._stopped = True
            self._ready.set()
            return
        self._ready.set()
        queue: deque[Request] = deque()
        try:
            while True:
                with self._cond:
                    self._cond.wait_for(lambda: self._incoming or queue or eng.busy
                                        or self._closing)
                    arrived = bool(self._incoming)
                    while self._incoming:
                        queue.append(self._incoming.popleft())
                    if self._closing and not queue and not eng.busy:
                        break
                if arrived:
                    queue = eng.order_queue(queue)
                eng.admit(queue)
                if not eng.busy:
                    continue
                done = eng.advance()
                if done:
                    with self._cond:
                        self._completed.extend(done)
                        self._cond.notify_all()
        except BaseException as e:
            with self._cond:
                self._error = e
        finally:
            try:
                eng.close()
            finally:
                with self._cond:
                    self._stopped = True
                    self._cond.notify_all()


def shard_requests(requests: list[Request], world: int) -> list[list[Request]]:
    """Split a request stream over `world` GPUs by estimated work: longest first, each onto the
    GPU with the least estimated work so far (ties to the lower rank). Every process computes
    the same split from the same stream; each share keeps arrival order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    loads = [0.0] * world
    parts: list[list[Request]] = [[] for _ in range(world)]
    for r in sorted(requests, key=lambda r: (-r.work_estimate(), r.rid)):
        k = min(range(world), key=lambda i: (loads[i], i))
        parts[k].append(r)
        loads[k] += r.work_estimate()
    return [sorted(p, key=lambda r: (r.arrival, r.rid)) for p in parts]


def serve_sharded(requests: list[Request], group=None, **kw) -> ServeStats:
    """Serving sharded by request over the processes of a torch.distributed group, one GPU
    each: every process serves its share of the stream (shard_requests) with serve(kw), with no
    collective on the data path. The processes start together (a barrier) and afterwards
    exchange their statistics once (all_gather_object), so every process returns the combined
    statistics: all completions, the slowest process's makespan, the per-GPU peaks at their
    maximum and the counters summed; kept states stay with the process that computed them.
    Without an initialized process group this is serve()."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return serve(requests, **kw)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    mine = shard_requests(requests, world)[rank]
    dist.barrier(group=group)
    local = serve(mine, **kw) if mine else ServeStats()
    parts = [None] * world
    dist.all_gather_object(parts, (local.completions, local.makespan, local.peak_bytes,
                                   local.max_active, local.peak_cells, local.chunks, local.joins,
                                   local.cap_waits, local.cell_waits), group=group)
    out = ServeStats(states=local.states)
    for comps, makespan, peak, active, cells, chunks, joins, cap, cell in parts:
        out.completions += comps
        out.makespan = max(out.makespan, makespan)
        out.peak_bytes = max(out.peak_bytes, peak)
        out.max_active = max(out.max_active, active)
        out.peak_cells = max(out.peak_cells, cells)
        out.chunks += chunks
        out.joins += joins
        out.cap_waits += cap
        out.cell_waits += cell
    out.completions.sort(key=lambda c: c.rid)
    return out


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
