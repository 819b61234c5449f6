"""One grid split into y strips: several GPUs (one process each) or several solvers on one GPU.

The reference runs a grid on one device (include/mhd/time_integrator.hpp:62-106,
src/cuda/cuda_solver.cu:504-776); this module splits a grid too large for one GPU's HBM into
strips of rows. Each strip is an ordinary solver (``_capi.DeviceSolver``) over its owned rows
plus ``OVERLAP`` rows copied from each neighbour, with the outflow y rule at its own ends, so
every RK2 step runs the same stage kernels as a whole grid:

* A step corrupts at most 3 rows per stage next to a strip end (2 rows of MUSCL stencil plus 1
  row of wall fill from a neighbour), 6 per step, so 6 overlap rows keep every owned row exact.
* The CFL reduction covers only the owned rows (``set_reduce_rows``); the strips' maxima are
  combined (max of the IEEE bits of non-negative doubles: an integer max) before dt, c_h and the
  clock are set (``strip_finish``), so all strips take the reference's global dt and finish at
  the same step.
* After every step each strip sends its first and last ``OVERLAP`` owned rows to its neighbours'
  overlap rows: NCCL send/recv between processes (torch.distributed), a device copy within one.

One step costs two stage launches, one 8-byte all-reduce, one finish launch and two row-block
exchanges of 6 rows x 9 planes. Results match the whole-grid solve: owned cells see the same
stencil values and the same dt.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

OVERLAP = 6
# With reflective walls the reference's wall fill stops at the grid's y boundary: a cell next to
# the periodic seam never takes a fill value from across it, and the ghosts across it hold
# unfilled copies. A strip whose overlap rows wrap around the seam reproduces that exactly when
# no cell within SEAM_ROWS rows of the seam is solid.
SEAM_ROWS = 2


@dataclass(frozen=True)
class Strip:
    """Strip ``index`` owns interior rows [y0, y0 + ny) of the grid and holds ``lo`` overlap rows
    below and ``hi`` above them (0 at an outflow end of the grid)."""

    index: int
    y0: int
    ny: int
    lo: int
    hi: int

    @property
    def rows(self) -> int:
        return self.lo + self.ny + self.hi


def plan_strips(ny: int, count: int, periodic_y: bool, overlap: int = OVERLAP) -> list[Strip]:
    """Even split of ny rows into ``count`` strips (the first ny % count strips one row more);
    each strip owns at least ``overlap`` rows, so a neighbour's overlap rows come from it alone."""
    if count < 1:
        raise ValueError("strip count must be at least 1")
    if count == 1:
        return [Strip(0, 0, ny, 0, 0)]
    if ny < count * overlap:
        raise ValueError(f"{ny} rows cannot be split into {count} strips of at least {overlap} rows")
    base, extra = divmod(ny, count)
    out, y = [], 0
    for i in range(count):
        n = base + (1 if i < extra else 0)
        lo = overlap if (i > 0 or periodic_y) else 0
        hi = overlap if (i < count - 1 or periodic_y) else 0
        out.append(Strip(i, y, n, lo, hi))
        y += n
    return out


def neighbours(plan: list[Strip], i: int, periodic_y: bool) -> tuple[int | None, int | None]:
    """Indices of the strips below and above strip i (None at an outflow end)."""
    n = len(plan)
    if n == 1:
        return None, None
    lo = i - 1 if i > 0 else (n - 1 if periodic_y else None)
    hi = i + 1 if i < n - 1 else (0 if periodic_y else None)
    return lo, hi


def strip_y_extent(y_min: float, dy: float, first_row: int, rows: int) -> tuple[float, float]:
    """y range of a strip's rows. Its (y_max - y_min) / rows may differ from dy in the last bit,
    so a strip solver is also given the whole grid's cell size (``set_cell_size``)."""
    a = y_min + first_row * dy
    return a, a + rows * dy


def global_rows(strip: Strip, ny: int, periodic_y: bool) -> np.ndarray:
    """Global interior row of each of the strip's rows (overlap rows wrap when periodic)."""
    r = np.arange(strip.y0 - strip.lo, strip.y0 + strip.ny + strip.hi)
    return np.mod(r, ny) if periodic_y else r


# ---------------------------------------------------------------- communication


class _Comm:
    """Who holds which strip, and the collectives between the processes that hold them. Every
    process holds a contiguous block of ``count / world`` strips."""

    def __init__(self, count: int, group=None, distributed: bool | None = None):
        import torch.distributed as dist

        up = dist.is_available() and dist.is_initialized()
        self.dist = dist if (up if distributed is None else distributed) else None
        self.group = group
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.world = self.dist.get_world_size(group) if self.dist else 1
        if count % self.world != 0:
            raise ValueError(f"{count} strips do not divide among {self.world} processes")
        self.per = count // self.world

    def owner(self, i: int) -> int:
        return i // self.per

    def global_rank(self, r: int) -> int:
        if self.group is None:
            return r
        return self.dist.get_global_rank(self.group, r)

    def all_reduce_max(self, t) -> None:
        if self.world > 1:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)

    def exchange(self, sends: list, recvs: list) -> None:
        """sends: (peer, key, tensor); recvs: (peer, key, tensor). Both sides of a pair of
        processes issue their messages ordered by key, so that the n-th send from A to B meets
        the n-th receive at B from A (NCCL point-to-point has no tags)."""
        if not sends and not recvs:
            return
        d = self.dist
        sends = sorted(sends, key=lambda m: (m[0], m[1]))
        recvs = sorted(recvs, key=lambda m: (m[0], m[1]))
        # One batch for every backend (NCCL runs it as one group, so sends and receives to the
        # same peer cannot wait on each other; gloo matches the tags): the CPU tests run the code
        # path the GPUs run.
        ops = [d.P2POp(d.isend, t, self.global_rank(p), self.group, tag) for p, tag, t in sends]
        ops += [d.P2POp(d.irecv, t, self.global_rank(p), self.group, tag) for p, tag, t in recvs]
        for w in d.batch_isend_irecv(ops):
            w.wait()

    def gather_objects(self, obj) -> list:
        if self.world == 1:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj, group=self.group)
        return out


# ---------------------------------------------------------------- strip engines


class DeviceStrip:
    """One strip on the current CUDA device: a DeviceSolver and torch views of its state and of
    its reduction word (zero-copy, on the solver's memory)."""

    def __init__(self, strip: Strip, nx: int, ny: int, precision: int, domain, ng: int,
                 bc_x: int, bc_y: int, mask_rows, walls: bool, tile_config: int = -1):
        import torch

        from . import _capi

        x_min, x_max, y_min, y_max = domain
        dy = (y_max - y_min) / ny
        ys0, ys1 = strip_y_extent(y_min, dy, strip.y0 - strip.lo, strip.rows)
        self.strip = strip
        self.nx = nx
        self.dev = _capi.DeviceSolver(nx, strip.rows, x_min, x_max, ys0, ys1, ng,
                                      precision=precision)
        self.dev.set_tile_config(tile_config)
        self.dev.set_cell_size((x_max - x_min) / nx, dy)
        self.dev.configure(bc_x, bc_y, mask_rows, walls)
        self.dev.set_reduce_rows(strip.lo, strip.lo + strip.ny)
        self.device = torch.device("cuda", torch.cuda.current_device())
        v = self.dev.strip_view()
        self.ch = _device_tensor(v.ch_bits, (1,), (1,), torch.int64, self.device)
        self.stream = torch.cuda.ExternalStream(self.dev.stream(), device=self.device)
        self._ptr = None
        self._refresh()

    def _refresh(self) -> None:
        """View of the current state buffer (the FP32-mixed increment form alternates between
        two buffers step by step)."""
        import torch

        v = self.dev.strip_view()
        if v.state != self._ptr:
            dtype = torch.float64 if v.elem_bytes == 8 else torch.float32
            self.state = _device_tensor(v.state, (v.planes, self.strip.rows, v.pitch),
                                        (v.plane, v.pitch, 1), dtype, self.device)
            self._ptr = v.state

    def rows(self, a: int, b: int):
        """All planes of strip rows [a, b), interior columns (a writable view)."""
        return self.state[:, a:b, :self.nx]

    def begin(self, params, nsteps: int) -> None:
        self.dev.strip_begin(params, nsteps)
        self._refresh()

    def step(self) -> None:
        self.dev.strip_step()
        self._refresh()

    def finish(self) -> None:
        self.dev.strip_finish()

    def poll(self) -> tuple[bool, int, float]:
        return self.dev.strip_poll()

    def end(self):
        r = self.dev.strip_end()
        return r.t, r.steps, r.c_h

    def upload(self, state: np.ndarray) -> None:
        self.dev.upload(state)

    def download(self) -> np.ndarray:
        return self.dev.download()

    def diagnostics(self, params) -> dict:
        return self.dev.diagnostics(params)

    def close(self) -> None:
        self.dev.close()


class _CudaArray:
    def __init__(self, ptr: int, shape, strides, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "strides": tuple(strides),
                                         "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "stream": None}


def _device_tensor(ptr, shape, strides_elems, dtype, device):
    import torch

    size = torch.tensor([], dtype=dtype).element_size()
    typestr = {torch.float64: "<f8", torch.float32: "<f4", torch.int64: "<i8"}[dtype]
    arr = _CudaArray(ptr, shape, [s * size for s in strides_elems], typestr)
    t = torch.as_tensor(arr, device=device)
    if t.data_ptr() != int(ptr):
        raise RuntimeError("strip view is not zero-copy")
    return t


# ---------------------------------------------------------------- the split solver


class StripSolver:
    """A grid of nx x ny interior cells split into ``strips`` y strips over the processes of a
    torch.distributed group (one block of strips each) or within one process.

    ``engine`` builds the solver of one strip (default: ``DeviceStrip`` on the current CUDA
    device); it gets (strip, nx, ny, precision, domain, ng, bc_x, bc_y, mask_rows, walls).
    ``distributed``: None spreads the strips over the processes of ``group`` when
    torch.distributed is initialized; False keeps every strip in this process.
    """

    def __init__(self, nx: int, ny: int, precision: int, *, strips: int | None = None,
                 domain=(0.0, 1.0, 0.0, 1.0), ng: int = 2, bc=(0, 0), mask=None,
                 walls: bool = True, group=None, engine=None, overlap: int = OVERLAP,
                 tile_config: int = -1, distributed: bool | None = None):
        from . import _capi

        if bc[0] == _capi.BC_REFLECTIVE or bc[1] == _capi.BC_REFLECTIVE:
            raise ValueError("Reflective boundaries are not supported by the CUDA backend")
        self.nx, self.ny, self.ng = nx, ny, ng
        self.precision = precision
        self.domain = tuple(float(v) for v in domain)
        self.bc = (int(bc[0]), int(bc[1]))
        self.periodic_y = self.bc[1] == _capi.BC_PERIODIC
        if strips is None and distributed is False:
            raise ValueError("in-process strips need an explicit strip count")
        self.comm = _Comm(strips if strips is not None else _world(group), group, distributed)
        count = self.comm.per * self.comm.world
        self.plan = plan_strips(ny, count, self.periodic_y, overlap)
        self.mask = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        if self.mask is not None and self.mask.shape != (ny, nx):
            raise ValueError(f"mask shape {self.mask.shape} != {(ny, nx)}")
        if (count > 1 and self.periodic_y and walls and self.mask is not None
                and not (self.mask[:SEAM_ROWS].all() and self.mask[-SEAM_ROWS:].all())):
            raise ValueError(
                "a masked grid with periodic y splits into strips only when its first and last "
                f"{SEAM_ROWS} rows are all fluid: the wall fill treats the periodic seam as a "
                "boundary, which a strip holding rows on both sides of it does not")
        strip_bc_y = self.bc[1] if count == 1 else _capi.BC_OUTFLOW
        first = self.comm.rank * self.comm.per
        self.local = self.plan[first:first + self.comm.per]
        make = engine or (lambda *a: DeviceStrip(*a, tile_config=tile_config))
        self.engines = []
        for s in self.local:
            rows = global_rows(s, ny, self.periodic_y)
            m = None if self.mask is None else np.ascontiguousarray(self.mask[rows])
            self.engines.append(make(s, nx, ny, precision, self.domain, ng, self.bc[0],
                                     strip_bc_y, m, walls))
        self._gpu = isinstance(self.engines[0], DeviceStrip)

    # -- state in and out

    def upload(self, state: np.ndarray) -> None:
        """state: the whole grid in the StateField layout, (9, ny + 2 ng, nx + 2 ng); every
        process passes it (each takes its strips' rows)."""
        g = self.ng
        if state.shape != (9, self.ny + 2 * g, self.nx + 2 * g):
            raise ValueError(f"state shape {state.shape} does not match the grid")
        for s, e in zip(self.local, self.engines):
            rows = global_rows(s, self.ny, self.periodic_y) + g
            # the strip's own y ghost rows repeat its end rows (outflow rule of the strip)
            rows = np.concatenate([[rows[0]] * g, rows, [rows[-1]] * g])
            e.upload(np.ascontiguousarray(state[:, rows, :]))

    def owned(self) -> list[tuple[int, np.ndarray]]:
        """(y0, owned interior rows (9, ny_s, nx)) of this process's strips, wall-filled as the
        reference leaves a solved state."""
        g = self.ng
        out = []
        for s, e in zip(self.local, self.engines):
            a = e.download()
            out.append((s.y0, a[:, g + s.lo:g + s.lo + s.ny, g:g + self.nx].copy()))
        return out

    def gather(self) -> np.ndarray:
        """The whole interior (9, ny, nx), on every process."""
        full = np.empty((9, self.ny, self.nx))
        for part in self.comm.gather_objects(self.owned()):
            for y0, a in part:
                full[:, y0:y0 + a.shape[1], :] = a
        return full

    def diagnostics(self, params) -> dict:
        """Whole-grid diagnostics (mhdb_diagnostics) combined over the strips' owned rows."""
        mine = [(s.ny, e.diagnostics(params)) for s, e in zip(self.local, self.engines)]
        parts = [p for r in self.comm.gather_objects(mine) for p in r]
        n = sum(ny for ny, _ in parts) * self.nx
        return {
            "mass": sum(d["mass"] for _, d in parts),
            "energy": sum(d["energy"] for _, d in parts),
            "div_b_max": max(d["div_b_max"] for _, d in parts),
            "div_b_l2": math.sqrt(sum(d["div_b_l2"] ** 2 * ny * self.nx for ny, d in parts) / n),
            "rho_min": min(d["rho_min"] for _, d in parts),
            "p_min": min(d["p_min"] for _, d in parts),
            "finite": all(d["finite"] for _, d in parts),
        }

    # -- stepping

    def solve(self, params):
        """Advance to params.t_end (the reference's solve()); returns (t, steps, c_h)."""
        return self._run(params, -1)

    def solve_steps(self, params, nsteps: int):
        """Advance exactly nsteps steps; returns (t, steps, c_h)."""
        if nsteps < 0:
            raise ValueError("nsteps must be non-negative")
        return self._run(params, nsteps)

    def _run(self, params, nsteps: int):
        for e in self.engines:
            e.begin(params, nsteps)
        self._combine_and_finish()
        if nsteps >= 0:
            for _ in range(nsteps):
                self._step()
        else:
            # Rounds of steps between polls: one step first (to measure dt), then the steps that
            # remain at the mean dt of the steps taken so far. The strips' common clock ends the
            # solve on the device (steps issued past the end do nothing), and a dt that shrinks
            # as the flow steepens costs one more round.
            while True:
                done, n, t = self._poll()
                if done:
                    break
                queue = 1 if n == 0 or t <= 0.0 else math.ceil((params.t_end - t) * n / t)
                for _ in range(max(1, min(queue, params.max_steps - n))):
                    self._step()
        results = [e.end() for e in self.engines]
        return results[0]

    def _poll(self) -> tuple[bool, int, float]:
        states = [e.poll() for e in self.engines]
        if len({s for s in states}) != 1:
            raise RuntimeError(f"strips disagree on the clock: {states}")
        return states[0]

    def _step(self) -> None:
        for e in self.engines:
            e.step()
        self._combine_and_finish()
        self._exchange()

    def _sync_in(self):
        """A stream on which the combine and the exchange run after the engines' launches."""
        if not self._gpu:
            return None
        import torch

        main = torch.cuda.current_stream(self.engines[0].device)
        for e in self.engines:
            main.wait_stream(e.stream)
        return main

    def _sync_out(self, main) -> None:
        if main is not None:
            for e in self.engines:
                e.stream.wait_stream(main)

    def _combine_and_finish(self) -> None:
        import torch

        main = self._sync_in()
        m = self.engines[0].ch.clone()
        for e in self.engines[1:]:
            m = torch.maximum(m, e.ch)
        self.comm.all_reduce_max(m)
        for e in self.engines:
            e.ch.copy_(m)
        self._sync_out(main)
        for e in self.engines:
            e.finish()

    def _exchange(self) -> None:
        """Owned edge rows into the neighbours' overlap rows. Message key (receiving strip,
        side): side 0 fills the receiver's lower overlap rows, side 1 its upper ones."""
        import torch

        main = self._sync_in()
        by_index = {s.index: (s, e) for s, e in zip(self.local, self.engines)}
        sends, recvs, local_copies = [], [], []
        for s, e in zip(self.local, self.engines):
            lo, hi = neighbours(self.plan, s.index, self.periodic_y)
            if hi is not None:  # my top owned rows -> the lower overlap rows of the strip above
                t = self.plan[hi]
                src = e.rows(s.lo + s.ny - t.lo, s.lo + s.ny)
                if hi in by_index:
                    local_copies.append((by_index[hi][1].rows(0, t.lo), src))
                else:
                    sends.append((self.comm.owner(hi), 2 * hi, src.contiguous()))
            if lo is not None:  # my bottom owned rows -> the upper overlap rows of the strip below
                b = self.plan[lo]
                src = e.rows(s.lo, s.lo + b.hi)
                if lo in by_index:
                    local_copies.append((by_index[lo][1].rows(b.lo + b.ny, b.rows), src))
                else:
                    sends.append((self.comm.owner(lo), 2 * lo + 1, src.contiguous()))
            if lo is not None and lo not in by_index:
                buf = torch.empty_like(e.rows(0, s.lo).contiguous())
                recvs.append((self.comm.owner(lo), 2 * s.index, buf, e.rows(0, s.lo)))
            if hi is not None and hi not in by_index:
                buf = torch.empty_like(e.rows(s.lo + s.ny, s.rows).contiguous())
                recvs.append((self.comm.owner(hi), 2 * s.index + 1, buf,
                              e.rows(s.lo + s.ny, s.rows)))
        # every source is owned rows and every destination overlap rows: the copies commute
        for dst, src in local_copies:
            dst.copy_(src)
        self.comm.exchange(sends, [(p, k, buf) for p, k, buf, _ in recvs])
        for _, _, buf, dst in recvs:
            dst.copy_(buf)
        self._sync_out(main)

    def close(self) -> None:
        for e in self.engines:
            e.close()
        self.engines = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _world(group) -> int:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group)
    return 1
