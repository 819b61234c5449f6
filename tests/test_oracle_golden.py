"""Pins the C oracle to the reference's own regression goldens and to fixtures produced by the
reference CPU solver (tests/golden/make_goldens.py)."""

import json
import os

import numpy as np
import pytest

from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import initial_state, interior

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return json.loads(str(d["meta"])), d


def rel_l2(a, b):
    return np.sqrt(np.sum((a - b) ** 2) / np.sum(b * b))


_NAMES = {"rho": 0, "energy": 4, "bx": 5, "by": 6, "bz": 7}


def test_orszag_tang_32_matches_reference_golden():
    # tests/test_regression_golden.cpp:51-80,144-156 of the reference: 36 steps,
    # rel L2 <= 1e-8 and Linf <= max(1e-10, 1e-7).
    meta, g = load("orszag_tang_32")
    U0 = initial_state(wl.orszag_tang(32, 32), 5.0 / 3.0)
    p = orc.Params(t_end=0.05, cfl=0.4, gamma=5.0 / 3.0, glm_alpha=0.1, limiter=orc.MC)
    out, t, steps, _ = orc.solve(U0, orc.Grid(32, 32), p)
    assert steps == int(meta["steps"]) == 36
    for name in ("rho", "bx", "by", "energy"):
        got = interior(out)[_NAMES[name]]
        assert rel_l2(got, g[name]) <= 1e-8, name
        assert np.max(np.abs(got - g[name])) <= 1e-7, name


def test_ohmic_sine_bz_32_matches_reference_golden():
    # tests/test_regression_golden.cpp:82-126,158-171: 137 steps, rel L2 <= 5e-8.
    meta, g = load("ohmic_sine_bz_32")
    U0 = initial_state(wl.ohmic_sine_bz(32, 32), 5.0 / 3.0)
    p = orc.Params(t_end=0.1, cfl=0.3, gamma=5.0 / 3.0, glm_alpha=0.1, limiter=orc.MINMOD,
                   ohmic=True, eta_ohm=0.1)
    out, t, steps, _ = orc.solve(U0, orc.Grid(32, 32), p)
    assert steps == int(meta["steps"]) == 137
    for name in ("bz", "energy"):
        got = interior(out)[_NAMES[name]]
        assert rel_l2(got, g[name]) <= 5e-8, name
        assert np.max(np.abs(got - g[name])) <= 5e-7, name


@pytest.mark.parametrize("seed", range(5))
def test_quadrant128_matches_reference_fixture(seed):
    d = np.load(os.path.join(GOLDEN, f"quadrant128_seed{seed}.npz"))
    n = 128
    U0 = initial_state(wl.four_quadrant(n, n, seed), 5.0 / 3.0, bc=(orc.OUTFLOW, orc.OUTFLOW))
    p = orc.Params(cfl=0.4, gamma=5.0 / 3.0, glm_alpha=0.1, limiter=orc.MINMOD, max_steps=200,
                   fixed_steps=True)
    out, t, steps, c_h = orc.solve(U0, orc.Grid(n, n), p, (orc.OUTFLOW, orc.OUTFLOW))
    assert steps == int(d["steps"]) == 200
    assert abs(t - float(d["t"])) <= 1e-12 * float(d["t"])
    inner = interior(out).reshape(9, -1)
    abs_sum = np.abs(inner).sum(axis=1)
    ref_abs = d["abs_sum"]
    rel = np.abs(abs_sum - ref_abs) / np.where(ref_abs > 0, ref_abs, 1.0)
    assert np.all(rel <= 1e-12), rel
    sample = inner[:, ::37]
    scale = np.maximum(np.abs(d["sample"]).max(axis=1, keepdims=True), 1e-300)
    assert np.all(np.abs(sample - d["sample"]) / scale <= 1e-10)
