"""Batched form: every solve of a batch gives the result it gives alone, through the batch and
through the single-solve path, for fixed-step and time-based solves of uneven sizes, mixed
limiters, ideal and non-ideal, and when solves join and leave while others run."""

import math

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200 import workloads as wl
from mhd_gpu_solver_b200.batch import BatchSolver, fixed_params
from mhd_gpu_solver_b200.mhd_solver import apply_boundary_conditions
from oracle import oracle as orc
from tests.helpers import assert_components

pytestmark = pytest.mark.gpu


def state(nx, ny, seed, gamma, bc, quadrant=False):
    prim = wl.four_quadrant(nx, ny, seed) if quadrant else wl.fourier_state(nx, ny, seed)
    U = wl.embed(wl.to_conservative(prim, gamma))
    apply_boundary_conditions(U, nx, ny, 2, bc[0], bc[1])
    return U


CASES = [
    # nx, ny, gamma, bc, limiter, nonideal, quadrant
    (64, 96, 5.0 / 3.0, (0, 0), _capi.VANLEER, False, False),
    (131, 47, 1.4, (2, 0), _capi.VANLEER, False, False),
    (33, 200, 1.55, (0, 2), _capi.MC, False, True),
    (100, 100, 5.0 / 3.0, (2, 2), _capi.MINMOD, True, True),
    (257, 65, 1.6, (0, 0), _capi.VANLEER, True, False),
    (7, 5, 1.5, (0, 0), _capi.VANLEER, False, False),
]


def params_of(case, **kw):
    nx, ny, gamma, bc, lim, ni, _ = case
    extra = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2,
                 eta_ambipolar=1e-3) if ni else {}
    return dict(gamma=gamma, limiter=lim, **extra, **kw)


def single(U, case, precision, nsteps=None, t_end=None):
    nx, ny, _, bc, *_ = case
    dev = _capi.DeviceSolver(nx, ny, precision=precision)
    try:
        dev.configure(bc[0], bc[1])
        dev.upload(U)
        if nsteps is not None:
            r = dev.solve_steps(_capi.make_params(**params_of(case)), nsteps)
        else:
            r = dev.solve(_capi.make_params(**params_of(case, t_end=t_end)))
        return dev.download(), r
    finally:
        dev.close()


@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
def test_fixed_step_batch_equals_single_solves(precision):
    b = BatchSolver(precision)
    states, ids = [], []
    for i, case in enumerate(CASES):
        U = state(case[0], case[1], i, case[2], case[3], case[6])
        states.append(U)
        ids.append(b.add(U, fixed_params(30, **params_of(case)), case[3], fixed_steps=True))
    assert b.step(25) == len(CASES)
    assert b.step(10) == 0  # every solve stops at exactly 30 steps
    for i, case in enumerate(CASES):
        r, fin = b.status(ids[i])
        assert fin and r.steps == 30
        got = b.download(ids[i])
        ref, rr = single(states[i], case, precision, nsteps=30)
        # The batch kernels use their own tile shape; per-cell arithmetic is the same source,
        # held to the parity tolerance of each form.
        tol = 1e-12 if precision == _capi.FP64 else 1e-6
        assert abs(r.t - rr.t) <= tol * rr.t and abs(r.c_h - rr.c_h) <= tol * rr.c_h
        assert_components(got, ref, tol, rr.c_h, what=i)
    b.close()


def test_time_based_batch_and_fp64_oracle():
    b = BatchSolver(_capi.FP64)
    t_ends = [0.01, 0.02, 0.005, 0.015]
    items = []
    for i, (case, t_end) in enumerate(zip(CASES[:4], t_ends)):
        U = state(case[0], case[1], 10 + i, case[2], case[3], case[6])
        sid = b.add(U, _capi.make_params(**params_of(case, t_end=t_end)), case[3])
        items.append((sid, U, case, t_end))
    while b.step(8) > 0:
        pass
    for sid, U, case, t_end in items:
        r, fin = b.status(sid)
        ref, rr = single(U, case, _capi.FP64, t_end=t_end)
        assert fin and r.steps == rr.steps and r.t == rr.t == t_end
        got = b.download(sid)
        assert_components(got, ref, 1e-12, rr.c_h)
        nx, ny, gamma, bc, lim, ni, _ = case
        op = orc.Params(t_end=t_end, gamma=gamma, limiter=lim)
        if ni:
            op.ohmic = op.hall = op.ambipolar = True
            op.eta_ohm, op.eta_hall, op.eta_ambipolar = 1e-3, 1e-2, 1e-3
        oref, ot, osteps, _ = orc.solve(U, orc.Grid(nx, ny), op, bc)
        assert osteps == r.steps
        assert_components(got, oref, 1e-12, r.c_h)
    b.close()


def test_result_is_the_same_alone_and_in_the_mix_with_joins_and_leaves():
    case = CASES[1]
    U = state(case[0], case[1], 3, case[2], case[3])
    alone = BatchSolver(_capi.FP32)
    sid = alone.add(U, fixed_params(40, **params_of(case)), case[3], fixed_steps=True)
    alone.step(40)
    ref = alone.download(sid)
    alone.close()

    mix = BatchSolver(_capi.FP32)
    others = [mix.add(state(c[0], c[1], 20 + j, c[2], c[3], c[6]),
                      fixed_params(60, **params_of(c)), c[3], fixed_steps=True)
              for j, c in enumerate(CASES[2:5])]
    mix.step(7)                       # the others run ahead
    sid = mix.add(U, fixed_params(40, **params_of(case)), case[3], fixed_steps=True)
    mix.step(11)
    mix.remove(others[0])             # one leaves mid-run
    late = mix.add(state(64, 64, 99, 5.0 / 3.0, (0, 0)),
                   fixed_params(10, limiter=_capi.VANLEER), (0, 0), fixed_steps=True)
    while mix.step(9) > 0:
        pass
    r, fin = mix.status(sid)
    assert fin and r.steps == 40
    assert np.array_equal(mix.download(sid), ref)
    assert mix.status(late)[0].steps == 10
    mix.close()


def test_batch_errors():
    b = BatchSolver(_capi.FP32)
    U = state(16, 16, 0, 5.0 / 3.0, (0, 0))
    with pytest.raises(ValueError, match="Reflective"):
        b.add(U, _capi.make_params(t_end=0.1), (1, 0))
    with pytest.raises(ValueError, match="t_end must be non-negative"):
        b.add(U, _capi.make_params(t_end=-1.0), (0, 0))
    sid = b.add(U, _capi.make_params(t_end=1.0, max_steps=3), (0, 0))
    while b.step(4) > 0:
        pass
    with pytest.raises(RuntimeError, match="max_steps"):
        b.status(sid)
    with pytest.raises(ValueError, match="unknown solve id"):
        b.status(12345)
    with pytest.raises(ValueError, match="unknown batch configuration"):
        b.set_config(sid, -2)
    with pytest.raises(ValueError, match="unknown batch configuration"):
        b.set_config(sid, _capi.lib.mhdb_batch_config_count(_capi.FP32))
    b.set_config(sid, -1)  # back to the choice by size
    b.close()
    assert math.isinf(fixed_params(3).t_end)


@pytest.mark.parametrize("kind", ["fourier", "quadrants"])
@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
def test_device_generator_matches_host_generator(kind, precision):
    nx, ny, gamma = 97, 64, 1.5
    if kind == "fourier":
        spec, prim = _capi.InitSpec.fourier(7), wl.fourier_state(nx, ny, 7)
    else:
        spec, prim = _capi.InitSpec.quadrants(7), wl.four_quadrant(nx, ny, 7)
    host = wl.embed(wl.to_conservative(prim, gamma))
    apply_boundary_conditions(host, nx, ny, 2, 0, 0)
    tol = 1e-12 if precision == _capi.FP64 else 1e-12
    dev = _capi.DeviceSolver(nx, ny, precision=precision)
    dev.configure(0, 0)
    dev.generate(spec, _capi.make_params(gamma=gamma))
    got = dev.download()
    dev.close()
    assert np.max(np.abs(got - host)) <= tol * max(1.0, float(np.max(np.abs(host))))
    b = BatchSolver(precision)
    sid = b.add_generated(nx, ny, spec, fixed_params(0, gamma=gamma), (0, 0), fixed_steps=True)
    assert np.array_equal(b.download(sid), got)
    b.close()


def test_launch_poll_and_downloads_beside_running_steps():
    """mhdb_batch_launch / mhdb_batch_poll give the results of mhdb_batch_step, and a solve that
    a poll reported finished downloads unchanged while the next steps of the others run."""
    steps = [12, 30, 45]
    cases = [CASES[0], CASES[1], CASES[4]]
    states = [state(c[0], c[1], 40 + i, c[2], c[3], c[6]) for i, c in enumerate(cases)]

    ref_b = BatchSolver(_capi.FP32)
    ref_ids = [ref_b.add(U, fixed_params(n, **params_of(c)), c[3], fixed_steps=True)
               for U, n, c in zip(states, steps, cases)]
    while ref_b.step(8) > 0:
        pass
    refs = [ref_b.download(i) for i in ref_ids]
    ref_b.close()

    b = BatchSolver(_capi.FP32)
    ids = [b.add(U, fixed_params(n, **params_of(c)), c[3], fixed_steps=True)
           for U, n, c in zip(states, steps, cases)]
    got, done = {}, []
    active = len(ids)
    while active > 0 or done:
        if active > 0:
            b.launch(8)
        for sid in done:  # finished at the previous poll; the next chunk is in flight
            got[sid] = b.download(sid)
            b.remove(sid)
        done = []
        if active > 0:
            active = b.poll()
            done = [sid for sid in ids if sid not in got and b.status(sid)[1]]
    b.close()
    for sid, ref in zip(ids, refs):
        assert np.array_equal(got[sid], ref)


def test_increment_form_batch_with_odd_step_counts():
    """Batch configuration 3 (increment form: each solve's state alternates between its two
    buffers, the parity taken from its own step counter) with odd and even step counts, finished
    solves downloaded while the others still step: the same values as the stored form
    (configuration 0) within the FP32-mixed tolerance. A stepped solve cannot switch between the
    two forms; other changes stay open."""
    steps = [13, 20, 27]
    cases = [CASES[0], CASES[1], CASES[4]]
    states = [state(c[0], c[1], 70 + i, c[2], c[3], c[6]) for i, c in enumerate(cases)]
    outs = {}
    for cfg in (0, 3):
        b = BatchSolver(_capi.FP32)
        ids = []
        for U, n, c in zip(states, steps, cases):
            sid = b.add(U, fixed_params(n, **params_of(c)), c[3], fixed_steps=True)
            b.set_config(sid, cfg)
            ids.append(sid)
        got, active = {}, len(ids)
        while active > 0:
            b.launch(5)
            active = b.poll()
            for sid in ids:
                if sid not in got and b.status(sid)[1]:
                    got[sid] = b.download(sid)
        for sid, n in zip(ids, steps):
            assert b.status(sid)[0].steps == n
        outs[cfg] = [got[i] for i in ids]
        if cfg == 3:
            live = b.add(states[0], fixed_params(9, **params_of(cases[0])), cases[0][3],
                         fixed_steps=True)
            b.set_config(live, 3)
            b.step(1)
            with pytest.raises(_capi.MhdbValueError):
                b.set_config(live, 0)
            b.set_config(live, 3)
        b.close()
    for a, c, case in zip(outs[0], outs[3], cases):
        assert_components(c, a, 1e-6, gamma=case[2])


def test_every_batch_configuration_gives_the_same_values():
    """The FP32-mixed batch configurations (TMA strip march with 32- or 64-row items, register
    strip march) run the same arithmetic and agree to FP32 rounding (the compiler may contract
    the non-ideal products differently in the segment prologue and the row loop), and match the
    FP64 batch within the FP32-mixed tolerance, ideal and non-ideal."""
    from mhd_gpu_solver_b200 import autotune
    from mhd_gpu_solver_b200.batch import batch_configs

    cases = [CASES[0], CASES[1], CASES[3], CASES[4], CASES[5]]
    states = [state(c[0], c[1], 60 + i, c[2], c[3], c[6]) for i, c in enumerate(cases)]
    configs = batch_configs(_capi.FP32)
    assert {c["kind"] for c in configs} >= {"march", "march_tma"}
    outs = []
    for cfg in configs:
        b = BatchSolver(_capi.FP32)
        ids = []
        for U, c in zip(states, cases):
            sid = b.add(U, fixed_params(20, **params_of(c)), c[3], fixed_steps=True)
            b.set_config(sid, cfg["config"])
            ids.append(sid)
        assert b.step(20) == 0
        outs.append([b.download(i) for i in ids])
        b.close()
    for cfg, other in zip(configs[1:], outs[1:]):
        for a, c, case in zip(outs[0], other, cases):
            assert_components(c, a, 1e-6, gamma=case[2], what=cfg)
    b64 = BatchSolver(_capi.FP64)
    ids = [b64.add(U, fixed_params(20, **params_of(c)), c[3], fixed_steps=True)
           for U, c in zip(states, cases)]
    b64.step(20)
    for sid, got, case in zip(ids, outs[0], cases):
        assert_components(got, b64.download(sid), 1e-6, gamma=case[2])
    b64.close()
    best = autotune.tune_batch(_capi.FP32, _capi.VANLEER, 100, 100, False, steps=2)
    assert 0 <= best < len(configs)
    with pytest.raises(ValueError):
        BatchSolver(_capi.FP32).set_config(0, 0)  # unknown solve id
