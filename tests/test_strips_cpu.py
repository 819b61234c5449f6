"""Strip decomposition of one grid (mhd_gpu_solver_b200/strips.py) on CPU: the orchestration
(overlap rows, combined CFL reduction, exchange order over torch.distributed) drives strips
whose solver is the FP64 oracle, one RK2 step of the reference at a time
(include/mhd/time_integrator.hpp:36-106 restated from the oracle's BC, wall-fill and RHS
entry points). The split result must equal the whole-grid oracle solve bit for bit: owned cells
see the same stencil values and every strip takes the global dt."""

import math
import os
import socket
import struct

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from mhd_gpu_solver_b200 import strips
from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc

from helpers import initial_state, interior


def _bits(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", x))[0]


def _value(b: int) -> float:
    return struct.unpack("<d", struct.pack("<q", b))[0]


def _max_diffusivity(p: orc.Params) -> float:
    eta = 0.0
    if p.ohmic:
        eta = max(eta, abs(p.eta_ohm))
    if p.hall:
        eta = max(eta, abs(p.eta_hall))
    if p.ambipolar:
        eta = max(eta, abs(p.eta_ambipolar))
    return eta


class OracleStrip:
    """The solver of one strip on the oracle, with the deferred-step protocol of DeviceStrip:
    begin / step reduce the owned rows' signal speed into ``ch``, finish sets dt from the
    combined value (the step control of the oracle's solve loop)."""

    def __init__(self, strip, nx, ny, precision, domain, ng, bc_x, bc_y, mask_rows, walls):
        x_min, x_max, y_min, y_max = domain
        dy = (y_max - y_min) / ny
        ys0, ys1 = strips.strip_y_extent(y_min, dy, strip.y0 - strip.lo, strip.rows)
        # the oracle takes the spacing from the extent: the test grids keep it exact
        assert (ys1 - ys0) / strip.rows == dy
        self.s, self.nx, self.ng = strip, nx, ng
        self.grid = orc.Grid(nx, strip.rows, ng, x_min, x_max, ys0, ys1)
        os0, os1 = strips.strip_y_extent(y_min, dy, strip.y0, strip.ny)
        self.own = orc.Grid(nx, strip.ny, ng, x_min, x_max, os0, os1)
        self.bc = (bc_x, bc_y)
        self.mask = mask_rows
        self.own_mask = None if mask_rows is None else np.ascontiguousarray(
            mask_rows[strip.lo:strip.lo + strip.ny])
        self.walls = walls
        self.inv_dx = 1.0 / ((x_max - x_min) / nx)
        self.inv_dy = 1.0 / dy
        self.h = min((x_max - x_min) / nx, dy)
        self.ch_np = np.zeros(1, dtype=np.int64)
        self.ch = torch.from_numpy(self.ch_np)
        self.U = None

    def rows(self, a, b):
        g = self.ng
        return torch.from_numpy(self.U)[:, g + a:g + b, g:g + self.nx]

    def upload(self, state):
        self.U = np.ascontiguousarray(state, dtype=np.float64).copy()

    def download(self):
        return self.U.copy()

    def _bc_fill(self, U):
        U = orc.apply_bc(U, self.grid, self.bc)
        if self.mask is not None and self.walls:
            U = orc.wall_fill(U, self.grid, self.mask, self.p.gamma)
        return U

    def _reduce(self):
        g, s = self.ng, self.s
        sub = np.ascontiguousarray(self.U[:, s.lo:s.lo + s.ny + 2 * g, :])
        _, c_h = orc.cfl(sub, self.own, self.p, self.own_mask)
        self.ch_np[0] = _bits(c_h)

    def begin(self, p, nsteps):
        self.p = p
        self.t, self.steps, self.c_h, self.dt = 0.0, 0, 0.0, 0.0
        self.t_end = math.inf if nsteps >= 0 else p.t_end
        self.max_steps = nsteps if nsteps >= 0 else p.max_steps
        self.finished, self.advance = False, False
        self._reduce()

    def finish(self):
        if self.finished:
            return
        c_h = _value(int(self.ch_np[0]))
        self.ch_np[0] = 0
        if self.advance:
            self.t += self.dt
            self.steps += 1
        if not (self.t < self.t_end) or self.steps >= self.max_steps:
            self.finished = True
            return
        dt = math.inf if c_h <= 0.0 else self.p.cfl / (c_h * self.inv_dx + c_h * self.inv_dy)
        eta = _max_diffusivity(self.p)
        if eta > 0.0:
            dt = min(dt, self.p.cfl * self.h * self.h / (2.0 * 2.0 * eta))
        dt = min(dt, self.t_end - self.t)
        assert dt > 0.0
        self.dt, self.c_h = dt, c_h

    def step(self):
        self.advance = True
        if self.finished:
            return
        p, dt, m = self.p, self.dt, self.mask
        U = self._bc_fill(self.U)
        Us = U + dt * orc.rhs(U, self.grid, p, self.c_h, m)
        Us = self._bc_fill(Us)
        self.U = 0.5 * (U + Us) + (0.5 * dt) * orc.rhs(Us, self.grid, p, self.c_h, m)
        self._reduce()

    def poll(self):
        return self.finished, self.steps, self.t

    def end(self):
        self.U = self._bc_fill(self.U)
        return self.t, self.steps, self.c_h

    def diagnostics(self, params):
        raise NotImplementedError

    def close(self):
        pass


CASES = {
    "periodic_quadrants": dict(nx=24, ny=40, bc=(orc.PERIODIC, orc.PERIODIC), mask=False,
                               ni=False, steps=10, limiter=orc.MC),
    "outflow_masked_nonideal": dict(nx=28, ny=36, bc=(orc.OUTFLOW, orc.PERIODIC), mask=True,
                                    ni=True, steps=8, limiter=orc.MINMOD),
    "outflow_time_based": dict(nx=20, ny=30, bc=(orc.OUTFLOW, orc.OUTFLOW), mask=True, ni=False,
                               steps=-1, limiter=orc.VANLEER),
}


def _problem(case):
    c = CASES[case]
    nx, ny = c["nx"], c["ny"]
    prim = wl.four_quadrant(nx, ny, seed=3)
    mask = None
    if c["mask"]:
        mask = wl.circles_and_rectangles(nx, ny, seed=5, n_circles=3, n_rects=2).copy()
        if c["bc"][1] == orc.PERIODIC:
            mask[:strips.SEAM_ROWS] = 1
            mask[-strips.SEAM_ROWS:] = 1
        assert not mask.all()
    kw = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2,
              eta_ambipolar=1e-3) if c["ni"] else {}
    if c["steps"] >= 0:
        p = orc.Params(limiter=c["limiter"], max_steps=c["steps"], fixed_steps=True, **kw)
    else:
        p = orc.Params(t_end=0.02, limiter=c["limiter"], **kw)
    # cell size 1/32: every strip's extent / rows is the grid's spacing exactly
    grid = orc.Grid(nx, ny, 2, 0.0, nx / 32, 0.0, ny / 32)
    U0 = initial_state(prim, p.gamma, c["bc"], mask)
    return grid, p, U0, mask, c


def _split_solve(case, strips_count, group=None):
    grid, p, U0, mask, c = _problem(case)
    domain = (grid.x_min, grid.x_max, grid.y_min, grid.y_max)
    with strips.StripSolver(grid.nx, grid.ny, 0, strips=strips_count, bc=c["bc"], mask=mask,
                            domain=domain, group=group, engine=OracleStrip) as ss:
        ss.upload(U0)
        res = ss.solve_steps(p, c["steps"]) if c["steps"] >= 0 else ss.solve(p)
        return ss.gather(), res


def _whole_solve(case):
    grid, p, U0, mask, c = _problem(case)
    out, t, steps, c_h = orc.solve(U0, grid, p, c["bc"], mask)
    return interior(out), (t, steps, c_h)


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("count", [2, 3])
def test_in_process_strips_equal_whole_grid(case, count):
    got, res = _split_solve(case, count)
    want, wres = _whole_solve(case)
    assert res == wres
    assert np.array_equal(got, want)


def test_single_strip_is_the_whole_grid():
    got, res = _split_solve("periodic_quadrants", 1)
    want, wres = _whole_solve("periodic_quadrants")
    assert res == wres
    assert np.array_equal(got, want)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, case, per_rank, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got, res = _split_solve(case, per_rank * world)
        # the same split kept inside this process while the process group is up
        grid, p, U0, mask, c = _problem(case)
        with strips.StripSolver(grid.nx, grid.ny, 0, strips=2, bc=c["bc"], mask=mask,
                                domain=(grid.x_min, grid.x_max, grid.y_min, grid.y_max),
                                engine=OracleStrip, distributed=False) as ss:
            ss.upload(U0)
            local_res = (ss.solve_steps(p, c["steps"]) if c["steps"] >= 0 else ss.solve(p))
            local = ss.gather()
        assert local_res == res and np.array_equal(local, got)
        q.put((rank, got, res))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("case,world,per_rank", [("periodic_quadrants", 2, 1),
                                                 ("outflow_masked_nonideal", 2, 2),
                                                 ("outflow_time_based", 3, 1),
                                                 ("periodic_quadrants", 4, 1)])
def test_gloo_ranks_equal_whole_grid(case, world, per_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, case, per_rank, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    out = [q.get(timeout=200) for _ in procs]
    for pr in procs:
        pr.join(timeout=30)
        assert pr.exitcode == 0
    want, wres = _whole_solve(case)
    for rank, got, res in out:
        assert res == wres, rank
        assert np.array_equal(got, want), rank


def test_masked_periodic_seam_must_be_fluid():
    nx, ny = 16, 32
    mask = np.ones((ny, nx), dtype=np.uint8)
    mask[1, 5] = 0
    with pytest.raises(ValueError, match="periodic seam"):
        strips.StripSolver(nx, ny, 0, strips=2, bc=(orc.PERIODIC, orc.PERIODIC), mask=mask,
                           engine=OracleStrip)
    # the same mask splits with outflow y, and without walls
    strips.StripSolver(nx, ny, 0, strips=2, bc=(orc.PERIODIC, orc.OUTFLOW), mask=mask,
                       engine=OracleStrip).close()
    strips.StripSolver(nx, ny, 0, strips=2, bc=(orc.PERIODIC, orc.PERIODIC), mask=mask,
                       walls=False, engine=OracleStrip).close()


def test_plan_strips_rules():
    p = strips.plan_strips(40, 3, periodic_y=True)
    assert [(s.y0, s.ny, s.lo, s.hi) for s in p] == [(0, 14, 6, 6), (14, 13, 6, 6),
                                                      (27, 13, 6, 6)]
    p = strips.plan_strips(40, 2, periodic_y=False)
    assert [(s.y0, s.ny, s.lo, s.hi) for s in p] == [(0, 20, 0, 6), (20, 20, 6, 0)]
    assert strips.neighbours(p, 0, False) == (None, 1)
    assert strips.neighbours(strips.plan_strips(40, 2, True), 0, True) == (1, 1)
    with pytest.raises(ValueError):
        strips.plan_strips(11, 2, periodic_y=False)
    assert strips.global_rows(strips.plan_strips(20, 2, True)[0], 20, True)[:6].tolist() == \
        [14, 15, 16, 17, 18, 19]


def test_strip_extent():
    a, b = strips.strip_y_extent(0.25, 1.0 / 64, -6, 20)
    assert (a, b) == (0.25 - 6.0 / 64, 0.25 + 14.0 / 64)
