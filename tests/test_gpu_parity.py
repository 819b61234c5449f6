"""CUDA backend (through the C ABI) against the CPU oracle and the reference fixtures.

Tolerances: the plain FP64 form must match the oracle to relative L1 <= 1e-12 per conserved
component after the stated step count, with the same step count (the FP64 parity bar), and the
mask must be handled the same way. The FP32-mixed form is held to relative L1 <= 1e-6. Every one
of the nine components is held (tests.helpers.assert_components): components whose reference value
is identically zero in absolute L1, psi on the scale max(sum|psi|, c_h sum|B|), and under the
FP32-mixed bar the components of m and B on their vector's scale.
"""

import json
import os

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import assert_components, initial_state, interior, rel_l1

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FP64_L1 = 1e-12
MIXED_L1 = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _need_device():
    if not _capi.cuda_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")


def _gpu(*a, **k):
    from tests.gpu_util import gpu_solve
    return gpu_solve(*a, **k)


def check_fp64(U0, grid, p, bc=(orc.PERIODIC, orc.PERIODIC), mask=None, walls=True,
               tol=FP64_L1):
    ref, tr, sr, cr = orc.solve(U0, grid, p, bc, mask, walls)
    got, tg, sg, cg = _gpu(U0, grid, p, bc, mask, walls)
    assert sg == sr, (sg, sr)
    assert abs(tg - tr) <= 1e-12 * max(1.0, abs(tr)), (tg, tr)
    assert abs(cg - cr) <= 1e-12 * max(1.0, abs(cr)), (cg, cr)
    assert_components(got, ref, tol, cr)
    # ghosts and wall-filled solids of the downloaded state (final BC + fill)
    scale = max(1.0, float(np.max(np.abs(ref))))
    assert float(np.max(np.abs(got - ref))) <= 1e-9 * scale
    return got, ref


@pytest.mark.parametrize("seed", range(5))
def test_quadrant128_fp64_matches_oracle_and_reference_fixture(seed):
    # 128^2, outflow x outflow, ideal, gamma 5/3, CFL 0.4, minmod, 200 SSP-RK2 steps.
    n = 128
    bc = (orc.OUTFLOW, orc.OUTFLOW)
    U0 = initial_state(wl.four_quadrant(n, n, seed), 5.0 / 3.0, bc)
    p = orc.Params(cfl=0.4, gamma=5.0 / 3.0, glm_alpha=0.1, limiter=orc.MINMOD, max_steps=200,
                   fixed_steps=True)
    got, _ = check_fp64(U0, orc.Grid(n, n), p, bc)
    d = np.load(os.path.join(GOLDEN, f"quadrant128_seed{seed}.npz"))
    inner = interior(got).reshape(9, -1)
    ref_abs = d["abs_sum"]
    rel = np.abs(np.abs(inner).sum(axis=1) - ref_abs) / np.where(ref_abs > 0, ref_abs, 1.0)
    assert np.all(rel <= 1e-11), rel


def test_orszag_tang_48x40_mc_time_based():
    # tests/test_gpu_backends.cpp:85-91 of the reference.
    U0 = initial_state(wl.orszag_tang(48, 40), 5.0 / 3.0)
    check_fp64(U0, orc.Grid(48, 40), orc.Params(t_end=0.05, limiter=orc.MC))


def test_sod_64x1_minmod_outflow_periodic():
    # tests/test_gpu_backends.cpp:93-100: ny = 1 strip, y extent 1/nx, gamma 1.4.
    grid = orc.Grid(64, 1, 2, 0.0, 1.0, 0.0, 1.0 / 64)
    bc = (orc.OUTFLOW, orc.PERIODIC)
    U0 = initial_state(wl.sod(64, 1, 0.0, 1.0, 0.0, 1.0 / 64), 1.4, bc)
    check_fp64(U0, grid, orc.Params(t_end=0.05, gamma=1.4, limiter=orc.MINMOD), bc)


def test_nonideal_all_terms_32():
    # tests/test_gpu_backends.cpp:102-110.
    U0 = initial_state(wl.orszag_tang(32, 32), 5.0 / 3.0)
    p = orc.Params(t_end=0.03, limiter=orc.MC, ohmic=True, hall=True, ambipolar=True,
                   eta_ohm=2e-3, eta_hall=1e-3, eta_ambipolar=5e-4)
    check_fp64(U0, orc.Grid(32, 32), p)


def _block_mask(nx, ny):
    m = np.ones((ny, nx), dtype=np.uint8)
    m[15:25, 12:20] = 0
    return m


def test_solid_block_mask_40():
    # tests/test_gpu_backends.cpp:112-124.
    mask = _block_mask(40, 40)
    U0 = initial_state(wl.orszag_tang(40, 40), 5.0 / 3.0, mask=mask)
    check_fp64(U0, orc.Grid(40, 40), orc.Params(t_end=0.03, limiter=orc.MC), mask=mask)


def _edge_mask(nx, ny, seed=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    m = (rng.uniform(size=(ny, nx)) > 0.12).astype(np.uint8)
    m[0, :4] = 0       # solids on every domain edge and in the corners
    m[-1, -3:] = 0
    m[:, 0][::5] = 0
    m[:, -1][2::4] = 0
    m[ny // 2, :] = 0  # a full wall row
    m[ny // 2, nx // 2] = 1
    return m


@pytest.mark.parametrize("bc", [(orc.OUTFLOW, orc.PERIODIC), (orc.PERIODIC, orc.OUTFLOW),
                                (orc.PERIODIC, orc.PERIODIC)])
@pytest.mark.parametrize("walls", [True, False])
def test_mask_touching_edges_nonideal(bc, walls):
    nx, ny = 37, 29
    mask = _edge_mask(nx, ny)
    U0 = initial_state(wl.fourier_state(nx, ny, 3), 5.0 / 3.0, bc, mask, walls)
    p = orc.Params(cfl=0.4, limiter=orc.MC, ohmic=True, hall=True, ambipolar=True,
                   eta_ohm=1e-3, eta_hall=1e-2, eta_ambipolar=1e-3, max_steps=30,
                   fixed_steps=True)
    check_fp64(U0, orc.Grid(nx, ny), p, bc, mask, walls)


@pytest.mark.parametrize("lim", [orc.MINMOD, orc.MC, orc.VANLEER])
def test_fourier_64_periodic_limiters(lim):
    U0 = initial_state(wl.fourier_state(64, 64, 0), 5.0 / 3.0)
    p = orc.Params(limiter=lim, max_steps=100, fixed_steps=True)
    check_fp64(U0, orc.Grid(64, 64), p)


def test_masked_nonideal_fourier_96_circles_rectangles():
    # The 2048^2 masked non-ideal case at 96^2: periodic y, outflow x.
    n = 96
    bc = (orc.OUTFLOW, orc.PERIODIC)
    mask = wl.circles_and_rectangles(n, n, 0)
    U0 = initial_state(wl.fourier_state(n, n, 0), 5.0 / 3.0, bc, mask)
    p = orc.Params(limiter=orc.VANLEER, ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3,
                   eta_hall=1e-2, eta_ambipolar=1e-3, max_steps=60, fixed_steps=True)
    check_fp64(U0, orc.Grid(n, n), p, bc, mask)


@pytest.mark.parametrize("nx,ny", [(1, 1), (1, 5), (5, 1), (7, 7), (31, 9), (33, 17), (65, 3),
                                   (32, 8), (64, 16)])
def test_odd_and_tile_edge_sizes(nx, ny):
    bc = (orc.PERIODIC, orc.OUTFLOW)
    U0 = initial_state(wl.four_quadrant(nx, ny, 11), 5.0 / 3.0, bc)
    p = orc.Params(limiter=orc.MC, max_steps=12, fixed_steps=True)
    check_fp64(U0, orc.Grid(nx, ny), p, bc)


def test_goldens_through_gpu():
    d = np.load(os.path.join(GOLDEN, "orszag_tang_32.npz"))
    U0 = initial_state(wl.orszag_tang(32, 32), 5.0 / 3.0)
    got, t, steps, _ = _gpu(U0, orc.Grid(32, 32), orc.Params(t_end=0.05, limiter=orc.MC))
    assert steps == int(json.loads(str(d["meta"]))["steps"]) == 36
    for name, c in (("rho", 0), ("bx", 5), ("by", 6), ("energy", 4)):
        g = interior(got)[c]
        assert np.sqrt(np.sum((g - d[name]) ** 2) / np.sum(d[name] ** 2)) <= 1e-8
    d = np.load(os.path.join(GOLDEN, "ohmic_sine_bz_32.npz"))
    U0 = initial_state(wl.ohmic_sine_bz(32, 32), 5.0 / 3.0)
    p = orc.Params(t_end=0.1, cfl=0.3, limiter=orc.MINMOD, ohmic=True, eta_ohm=0.1)
    got, t, steps, _ = _gpu(U0, orc.Grid(32, 32), p)
    assert steps == 137
    for name, c in (("bz", 7), ("energy", 4)):
        g = interior(got)[c]
        assert np.sqrt(np.sum((g - d[name]) ** 2) / np.sum(d[name] ** 2)) <= 5e-8


def test_contract_errors_and_round_trip():
    dev = _capi.DeviceSolver(16, 12)
    try:
        with pytest.raises(ValueError, match="Reflective boundary conditions"):
            dev.configure(_capi.BC_REFLECTIVE, _capi.BC_PERIODIC)
        with pytest.raises(ValueError, match="FluidMask size"):
            dev.configure(0, 0, np.zeros((3, 3), np.uint8))
        dev.configure(0, 0)
        U0 = initial_state(wl.orszag_tang(16, 12), 5.0 / 3.0)
        U0[:, 0, 0] = 123.0  # ghost values survive an upload/download round trip
        dev.upload(U0)
        assert np.array_equal(dev.download(), U0)
        with pytest.raises(ValueError, match="t_end must be non-negative"):
            dev.solve(_capi.make_params(t_end=-1.0))
        with pytest.raises(ValueError, match="CFL number must be positive"):
            dev.solve(_capi.make_params(t_end=1.0, cfl=0.0))
        r = dev.solve(_capi.make_params(t_end=0.0))
        assert (r.t, r.steps) == (0.0, 0)
        with pytest.raises(RuntimeError, match="reached max_steps before t_end") as e:
            dev.solve(_capi.make_params(t_end=1.0, max_steps=3))
        assert e.value.code == _capi.MAX_STEPS
        with pytest.raises(ValueError):
            dev.upload(np.zeros((9, 3, 3)))
        assert dev.device_name().startswith("CUDA: ")
    finally:
        dev.close()
    g = _capi.Grid(8, 8, 1, 0.0, 1.0, 0.0, 1.0)
    h = _capi.C.c_void_p()
    assert _capi.lib.mhdb_create(_capi.C.byref(g), 0, _capi.C.byref(h)) == _capi.INVALID_ARGUMENT
    assert b"ng >= 2" in _capi.lib.mhdb_last_error(None)


def test_resident_continuation_equals_round_trip():
    """Two solves on resident state == solve, download, upload, solve (the reference's two
    run() calls), bit for bit, with a mask touching the edges."""
    nx, ny = 37, 29
    bc = (orc.OUTFLOW, orc.PERIODIC)
    mask = _edge_mask(nx, ny, 3)
    U0 = initial_state(wl.fourier_state(nx, ny, 5), 5.0 / 3.0, bc, mask)
    cp = _capi.make_params(limiter=_capi.MC)
    outs = []
    for round_trip in (False, True):
        dev = _capi.DeviceSolver(nx, ny)
        dev.configure(bc[0], bc[1], mask, True)
        dev.upload(U0)
        dev.solve_steps(cp, 7)
        if round_trip:
            dev.upload(dev.download())
        dev.solve_steps(cp, 9)
        outs.append(dev.download())
        dev.close()
    assert np.array_equal(outs[0], outs[1])
    p = orc.Params(limiter=orc.MC, max_steps=7, fixed_steps=True)
    mid, *_ = orc.solve(U0, orc.Grid(nx, ny), p, bc, mask)
    p.max_steps = 9
    ref, *_ = orc.solve(mid, orc.Grid(nx, ny), p, bc, mask)
    assert_components(outs[0], ref, FP64_L1)


@pytest.mark.parametrize("config", [13, 17])
@pytest.mark.parametrize("masked", [False, True])
def test_increment_form_state_buffers_alternate_correctly(masked, config):
    """The increment form writes U^{n+1} to the other state buffer: solves of odd and even step
    counts in sequence (7, then 40 through a captured 32-step batch and 8 direct steps, then 3)
    equal a download/upload round trip between them and, without a mask, one 50-step solve (with
    a mask every solve ends with the reference's wall fill, which the next one starts from), and
    download, diagnostics and the next solve all see the current buffer."""
    nx, ny = 150, 96
    bc = (orc.PERIODIC, orc.OUTFLOW)
    mask = _edge_mask(nx, ny, 4) if masked else None
    U0 = initial_state(wl.fourier_state(nx, ny, 8), 5.0 / 3.0, bc, mask)
    cp = _capi.make_params(limiter=_capi.VANLEER)
    outs, diags = [], []
    for plan in ((7, 40, 3), (7, 40, 3, "rt"), (50,)):
        dev = _capi.DeviceSolver(nx, ny, precision=_capi.FP32)
        dev.set_tile_config(config)
        dev.configure(bc[0], bc[1], mask, True)
        dev.upload(U0)
        for n in plan:
            if n == "rt":
                continue
            dev.solve_steps(cp, n)
            if "rt" in plan and n == 7:
                dev.upload(dev.download())
        outs.append(dev.download())
        diags.append(dev.diagnostics(cp))
        dev.close()
    assert np.array_equal(outs[0], outs[1])
    if not masked:
        assert np.array_equal(outs[0], outs[2])
        assert diags[0] == diags[2]
    ref = U0
    for n in (7, 40, 3):
        p = orc.Params(limiter=orc.VANLEER, max_steps=n, fixed_steps=True)
        ref, *_ = orc.solve(ref, orc.Grid(nx, ny), p, bc, mask)
    assert_components(outs[0], ref, MIXED_L1)


@pytest.mark.parametrize("config", [13, 17])
def test_increment_form_time_based_solves(config):
    """Time-based solves (batches of steps between polls, graph batches and odd remainders) on
    the increment form, twice in a row on resident state: the oracle's step counts and clock,
    values within the FP32-mixed tolerance."""
    nx, ny = 150, 96
    bc = (orc.PERIODIC, orc.PERIODIC)
    U0 = initial_state(wl.fourier_state(nx, ny, 3), 5.0 / 3.0, bc)
    dev = _capi.DeviceSolver(nx, ny, precision=_capi.FP32)
    ref = U0
    try:
        dev.set_tile_config(config)
        dev.configure(bc[0], bc[1])
        dev.upload(U0)
        for t_end in (0.021, 0.0137):
            r = dev.solve(_capi.make_params(t_end=t_end, limiter=_capi.VANLEER))
            p = orc.Params(t_end=t_end, limiter=orc.VANLEER)
            ref, tr, sr, _ = orc.solve(ref, orc.Grid(nx, ny), p, bc)
            assert r.steps == sr and abs(r.t - tr) <= 1e-6 * tr
        got = dev.download()
    finally:
        dev.close()
    assert_components(got, ref, MIXED_L1)


def test_diagnostics_match_oracle():
    n = 64
    bc = (orc.OUTFLOW, orc.PERIODIC)
    mask = wl.circles_and_rectangles(n, n, 1)
    U0 = initial_state(wl.fourier_state(n, n, 2), 5.0 / 3.0, bc, mask)
    p = orc.Params(limiter=orc.VANLEER, max_steps=20, fixed_steps=True)
    ref, *_ = orc.solve(U0, orc.Grid(n, n), p, bc, mask)
    dref = orc.diagnostics(ref, orc.Grid(n, n), p.gamma)
    dev = _capi.DeviceSolver(n, n)
    dev.configure(bc[0], bc[1], mask, True)
    dev.upload(U0)
    cp = _capi.make_params(limiter=_capi.VANLEER)
    dev.solve_steps(cp, 20)
    d = dev.diagnostics(cp)
    dev.close()
    for k in ("mass", "energy", "div_b_max", "div_b_l2", "rho_min", "p_min"):
        assert abs(d[k] - dref[k]) <= 1e-11 * max(1.0, abs(dref[k])), (k, d[k], dref[k])
    assert d["finite"] and dref["finite"]


@pytest.mark.parametrize("case", ["quadrant128", "fourier256", "masked_nonideal128"])
def test_fp32_mixed_within_1e6_of_fp64_oracle(case):
    if case == "quadrant128":
        n, bc, mask = 128, (orc.OUTFLOW, orc.OUTFLOW), None
        U0 = initial_state(wl.four_quadrant(n, n, 0), 5.0 / 3.0, bc)
        p = orc.Params(limiter=orc.MINMOD, max_steps=200, fixed_steps=True)
    elif case == "fourier256":
        n, bc, mask = 256, (orc.PERIODIC, orc.PERIODIC), None
        U0 = initial_state(wl.fourier_state(n, n, 0), 5.0 / 3.0, bc)
        p = orc.Params(limiter=orc.VANLEER, max_steps=200, fixed_steps=True)
    else:
        n, bc = 128, (orc.OUTFLOW, orc.PERIODIC)
        mask = wl.circles_and_rectangles(n, n, 0)
        U0 = initial_state(wl.fourier_state(n, n, 0), 5.0 / 3.0, bc, mask)
        p = orc.Params(limiter=orc.VANLEER, ohmic=True, hall=True, ambipolar=True,
                       eta_ohm=1e-3, eta_hall=1e-2, eta_ambipolar=1e-3, max_steps=100,
                       fixed_steps=True)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(n, n), p, bc, mask)
    got, tg, sg, _ = _gpu(U0, orc.Grid(n, n), p, bc, mask, precision=_capi.FP32)
    assert sg == sr
    assert abs(tg - tr) <= 1e-5 * tr
    err = assert_components(got, ref, MIXED_L1, cr, what=case)
    print(case, "L1 FP32-mixed vs FP64 oracle:", err, "plain relative:", rel_l1(got, ref))


@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
def test_every_tile_configuration_matches_oracle(precision):
    nx, ny = 70, 45
    U0 = initial_state(wl.fourier_state(nx, ny, 4), 5.0 / 3.0)
    p = orc.Params(limiter=orc.VANLEER, max_steps=20, fixed_steps=True)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p)
    tol = FP64_L1 if precision == _capi.FP64 else MIXED_L1
    for cfg in _capi.tile_configs(precision):
        dev = _capi.DeviceSolver(nx, ny, precision=precision)
        dev.set_tile_config(cfg["config"])
        dev.configure(0, 0)
        dev.upload(U0)
        r = dev.solve_steps(_capi.make_params(limiter=_capi.VANLEER), 20)
        got = dev.download()
        dev.close()
        assert r.steps == sr
        assert_components(got, ref, tol, cr, what=cfg)


MARCH_CASES = [
    # nx, ny, bc_x, bc_y, state, limiter: partial strips (28 columns per warp) and partial row
    # segments, every boundary rule combination, every limiter, smooth and shocked states
    (61, 150, orc.PERIODIC, orc.PERIODIC, "fourier", orc.VANLEER),
    (61, 150, orc.OUTFLOW, orc.OUTFLOW, "quadrants", orc.MC),
    (29, 33, orc.OUTFLOW, orc.PERIODIC, "fourier", orc.MINMOD),
    (140, 70, orc.PERIODIC, orc.OUTFLOW, "quadrants", orc.VANLEER),
    (5, 7, orc.PERIODIC, orc.PERIODIC, "fourier", orc.MC),
]


@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
@pytest.mark.parametrize("case", range(len(MARCH_CASES)))
def test_strip_march_configurations_match_oracle(precision, case):
    nx, ny, bcx, bcy, state, lim = MARCH_CASES[case]
    bc = (bcx, bcy)
    prim = (wl.fourier_state(nx, ny, 9) if state == "fourier" else wl.four_quadrant(nx, ny, 3))
    U0 = initial_state(prim, 5.0 / 3.0, bc)
    p = orc.Params(limiter=lim, max_steps=25, fixed_steps=True)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc)
    tol = FP64_L1 if precision == _capi.FP64 else MIXED_L1
    marches = [c for c in _capi.tile_configs(precision) if c["kind"].startswith("march")]
    assert marches
    for cfg in marches:
        dev = _capi.DeviceSolver(nx, ny, precision=precision)
        dev.set_tile_config(cfg["config"])
        dev.configure(bcx, bcy)
        dev.upload(U0)
        r = dev.solve_steps(_capi.make_params(limiter=lim), 25)
        got = dev.download()
        dev.close()
        assert r.steps == sr
        assert abs(r.t - tr) <= (1e-12 if precision == _capi.FP64 else 1e-6) * max(1.0, tr)
        assert_components(got, ref, tol, cr, what=cfg)


@pytest.mark.parametrize("case", range(len(MARCH_CASES)))
def test_tma_strip_march_equals_register_strip_march(case):
    """The TMA-fed strip march (rows staged in shared memory by bulk tensor copies) performs the
    same arithmetic as the register strip march that loads rows itself: same values, bit for
    bit, on partial strips, every boundary rule and every limiter."""
    nx, ny, bcx, bcy, state, lim = MARCH_CASES[case]
    prim = (wl.fourier_state(nx, ny, 9) if state == "fourier" else wl.four_quadrant(nx, ny, 3))
    U0 = initial_state(prim, 5.0 / 3.0, (bcx, bcy))
    cfgs = _capi.tile_configs(_capi.FP32)
    plain = [c for c in cfgs if c["kind"] == "march"]
    tma = [c for c in cfgs if c["kind"] == "march_tma"]
    assert plain and tma

    def run(cfg):
        dev = _capi.DeviceSolver(nx, ny, precision=_capi.FP32)
        dev.set_tile_config(cfg["config"])
        dev.configure(bcx, bcy)
        dev.upload(U0)
        r = dev.solve_steps(_capi.make_params(limiter=lim), 25)
        got = dev.download()
        dev.close()
        return r, got

    r0, ref = run(plain[0])
    for cfg in tma:
        r, got = run(cfg)
        assert r.steps == r0.steps and r.t == r0.t, cfg
        assert np.array_equal(got, ref), (cfg, float(np.max(np.abs(got - ref))))


NI_PARAMS = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2,
                 eta_ambipolar=1e-3)


@pytest.mark.parametrize("precision", [_capi.FP64, _capi.FP32])
@pytest.mark.parametrize("case", [0, 1, 2, 4])
def test_nonideal_strip_march_configurations_match_oracle(precision, case):
    """Ohmic, Hall and ambipolar terms in the strip-march kernels (current carried row to row,
    x neighbours by shuffle): FP64 to 1e-12, FP32-mixed to 1e-6 against the FP64 oracle."""
    nx, ny, bcx, bcy, state, lim = MARCH_CASES[case]
    bc = (bcx, bcy)
    prim = (wl.fourier_state(nx, ny, 9) if state == "fourier" else wl.four_quadrant(nx, ny, 3))
    U0 = initial_state(prim, 5.0 / 3.0, bc)
    p = orc.Params(limiter=lim, max_steps=20, fixed_steps=True, **NI_PARAMS)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc)
    tol = FP64_L1 if precision == _capi.FP64 else MIXED_L1
    marches = [c for c in _capi.tile_configs(precision) if c["kind"].startswith("march")]
    for cfg in marches:
        dev = _capi.DeviceSolver(nx, ny, precision=precision)
        dev.set_tile_config(cfg["config"])
        dev.configure(bcx, bcy)
        dev.upload(U0)
        r = dev.solve_steps(_capi.make_params(limiter=lim, **NI_PARAMS), 20)
        got = dev.download()
        dev.close()
        assert r.steps == sr
        assert abs(r.t - tr) <= (1e-12 if precision == _capi.FP64 else 1e-6) * max(1.0, tr)
        assert_components(got, ref, tol, cr, what=cfg)


def test_default_configuration_of_a_large_grid_matches_fp64():
    """Without a chosen configuration a 1024^2 FP32-mixed solve runs the TMA strip march (the
    drop-in's default for large unmasked grids); it stays within the FP32-mixed tolerance of the
    FP64 form, ideal and non-ideal."""
    n = 1024
    U0 = initial_state(wl.fourier_state(n, n, 2), 5.0 / 3.0)
    for kw in ({}, NI_PARAMS):
        outs = {}
        for prec in (_capi.FP64, _capi.FP32):
            dev = _capi.DeviceSolver(n, n, precision=prec)
            dev.configure(0, 0)
            dev.upload(U0)
            r = dev.solve_steps(_capi.make_params(limiter=_capi.VANLEER, **kw), 6)
            outs[prec] = (dev.download(), r)
            dev.close()
        (u64, r64), (u32, r32) = outs[_capi.FP64], outs[_capi.FP32]
        assert r32.steps == r64.steps == 6
        assert_components(u32, u64, MIXED_L1, r64.c_h, what=kw)


@pytest.mark.parametrize("case", range(len(MARCH_CASES)))
@pytest.mark.parametrize("ni", [False, True])
def test_increment_form_matches_stored_form(case, ni):
    """The FP32-mixed increment form (stage 1 stores the FP32 increment dt L, stage 2 rebuilds
    U* = U^n + increment) against the stored form of the same strip-march shape and against the
    FP64 oracle: within the FP32-mixed tolerance, same step count and clock."""
    nx, ny, bcx, bcy, state, lim = MARCH_CASES[case]
    prim = (wl.fourier_state(nx, ny, 9) if state == "fourier" else wl.four_quadrant(nx, ny, 3))
    bc = (bcx, bcy)
    U0 = initial_state(prim, 5.0 / 3.0, bc)
    kw = NI_PARAMS if ni else {}
    p = orc.Params(limiter=lim, max_steps=25, fixed_steps=True, **kw)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc)
    cfgs = _capi.tile_configs(_capi.FP32)
    delta = [c for c in cfgs if c["kind"] == "march_tma_delta"]
    assert delta
    for cfg in delta:
        twin = next(c for c in cfgs if c["kind"] == "march_tma" and c["tile_y"] == cfg["tile_y"]
                    and c["threads"] == cfg["threads"] and c["min_blocks"] == cfg["min_blocks"])
        got, tg, sg, _ = _gpu(U0, orc.Grid(nx, ny), p, bc, precision=_capi.FP32,
                              tile_config=cfg["config"])
        stored, ts, ss, _ = _gpu(U0, orc.Grid(nx, ny), p, bc, precision=_capi.FP32,
                                 tile_config=twin["config"])
        assert sg == ss == sr
        assert abs(tg - tr) <= 1e-6 * max(1.0, tr) and abs(tg - ts) <= 1e-6 * max(1.0, ts)
        for other in (ref, stored):
            assert_components(got, other, MIXED_L1, cr, what=cfg)


@pytest.mark.parametrize("bc", [(orc.OUTFLOW, orc.PERIODIC), (orc.PERIODIC, orc.OUTFLOW)])
@pytest.mark.parametrize("walls", [True, False])
@pytest.mark.parametrize("ni", [False, True])
def test_masked_tma_strip_march_matches_oracle(bc, walls, ni):
    """Masked solves on the strip-march configurations (FP32-mixed configuration 11 is the TMA
    strip march that serves masks; the others fall back to the tile kernel): solids wall-filled
    when their row is converted, solid updates through the FP64 wall-fill path, ghosts keeping
    pre-fill values; against the FP64 oracle within the FP32-mixed tolerance."""
    nx, ny = 61, 45
    mask = _edge_mask(nx, ny, seed=11)
    U0 = initial_state(wl.fourier_state(nx, ny, 6), 5.0 / 3.0, bc, mask, walls)
    kw = NI_PARAMS if ni else {}
    p = orc.Params(limiter=orc.VANLEER, max_steps=25, fixed_steps=True, **kw)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc, mask, walls)
    for cfg in _capi.tile_configs(_capi.FP32):
        if not cfg["kind"].startswith("march"):
            continue
        got, tg, sg, _ = _gpu(U0, orc.Grid(nx, ny), p, bc, mask, walls, precision=_capi.FP32,
                              tile_config=cfg["config"])
        assert sg == sr
        assert abs(tg - tr) <= 1e-6 * max(1.0, tr)
        assert_components(got, ref, MIXED_L1, cr, what=cfg)


@pytest.mark.parametrize("bc", [(orc.OUTFLOW, orc.PERIODIC), (orc.PERIODIC, orc.OUTFLOW)])
@pytest.mark.parametrize("walls", [True, False])
@pytest.mark.parametrize("ni", [False, True])
def test_masked_fp64_tma_strip_march_matches_oracle(bc, walls, ni):
    """Masked FP64 solves on the FP64 strip-march configurations (configuration 7 is the TMA
    strip march that serves masks: solid cells take the tile kernel's FP64 fill and solid update
    from global memory): every component within the FP64 bar of the oracle, same step count."""
    nx, ny = 61, 45
    mask = _edge_mask(nx, ny, seed=11)
    U0 = initial_state(wl.fourier_state(nx, ny, 6), 5.0 / 3.0, bc, mask, walls)
    kw = NI_PARAMS if ni else {}
    p = orc.Params(limiter=orc.VANLEER, max_steps=25, fixed_steps=True, **kw)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc, mask, walls)
    served = 0
    for cfg in _capi.tile_configs(_capi.FP64):
        if cfg["kind"] != "march_tma":
            continue
        got, tg, sg, cg = _gpu(U0, orc.Grid(nx, ny), p, bc, mask, walls,
                               tile_config=cfg["config"])
        assert sg == sr
        assert abs(tg - tr) <= 1e-12 * max(1.0, tr) and abs(cg - cr) <= 1e-12 * cr
        assert_components(got, ref, FP64_L1, cr, what=cfg)
        served += 1
    assert served >= 1


def test_default_configuration_of_a_large_masked_grid_matches_fp64():
    """A 1024^2 masked, non-ideal FP32-mixed solve without a chosen configuration runs the TMA
    strip march that serves masks; it stays within the FP32-mixed tolerance of the FP64 form."""
    n = 1024
    bc = (orc.OUTFLOW, orc.PERIODIC)
    mask = wl.circles_and_rectangles(n, n, 0)
    U0 = initial_state(wl.fourier_state(n, n, 1), 5.0 / 3.0, bc, mask)
    p = orc.Params(limiter=orc.VANLEER, max_steps=6, fixed_steps=True, **NI_PARAMS)
    u64, _, s64, c64 = _gpu(U0, orc.Grid(n, n), p, bc, mask)
    u32, _, s32, _ = _gpu(U0, orc.Grid(n, n), p, bc, mask, precision=_capi.FP32)
    assert s32 == s64 == 6
    assert_components(u32, u64, MIXED_L1, c64)


@pytest.mark.parametrize("case", range(len(MARCH_CASES)))
@pytest.mark.parametrize("ni", [False, True])
def test_two_column_strip_march_matches_single_column(case, ni):
    """The two-column strip march of the increment form (two columns per lane, 60 owned columns
    per warp) runs the single-column march's arithmetic operand for operand: on partial strips,
    every boundary rule and every limiter, ideal solves give its values bit for bit, with the same
    step count and clock; non-ideal ones are held to it and to the FP64 oracle at the FP32-mixed
    bar. 25 steps: an odd count, so the result ends in the other state buffer."""
    nx, ny, bcx, bcy, state, lim = MARCH_CASES[case]
    prim = (wl.fourier_state(nx, ny, 9) if state == "fourier" else wl.four_quadrant(nx, ny, 3))
    bc = (bcx, bcy)
    U0 = initial_state(prim, 5.0 / 3.0, bc)
    kw = NI_PARAMS if ni else {}
    p = orc.Params(limiter=lim, max_steps=25, fixed_steps=True, **kw)
    cfgs = _capi.tile_configs(_capi.FP32)
    pairs = [c["config"] for c in cfgs if c["kind"] == "march_tma_pair"]
    single = next(c["config"] for c in cfgs if c["kind"] == "march_tma_delta" and c["tile_y"] == 32)
    assert pairs
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc)
    want, tw, sw, _ = _gpu(U0, orc.Grid(nx, ny), p, bc, precision=_capi.FP32, tile_config=single)
    for cfg in pairs:
        got, tg, sg, _ = _gpu(U0, orc.Grid(nx, ny), p, bc, precision=_capi.FP32, tile_config=cfg)
        assert sg == sw == sr
        if not ni:
            assert tg == tw
            assert np.array_equal(got, want), (cfg, float(np.max(np.abs(got - want))))
        else:
            assert abs(tg - tw) <= 1e-6 * tw
            assert_components(got, want, MIXED_L1, cr, what=cfg)
        assert_components(got, ref, MIXED_L1, cr, what=cfg)


def _config_of(precision, kind, **shape):
    return [c["config"] for c in _capi.tile_configs(precision) if c["kind"] == kind
            and all(c[k] == v for k, v in shape.items())]


@pytest.mark.parametrize("case", range(len(MARCH_CASES)))
@pytest.mark.parametrize("ni", [False, True])
def test_increment_form_delta_ring_matches_own_stream(case, ni):
    """Stage 2 of the increment form with the own cells' delta taken from the halo stream (kept
    in a 3-row ring per lane) against the same march reading it through the own stream: the same
    operands, so ideal solves agree bit for bit (same step count and clock); non-ideal ones are
    held to it at the FP32-mixed bar, and both to the FP64 oracle. 25 steps (odd: the result ends
    in the other state buffer); partial strips and segments, every boundary rule and limiter."""
    nx, ny, bcx, bcy, state, lim = MARCH_CASES[case]
    prim = (wl.fourier_state(nx, ny, 9) if state == "fourier" else wl.four_quadrant(nx, ny, 3))
    bc = (bcx, bcy)
    U0 = initial_state(prim, 5.0 / 3.0, bc)
    kw = NI_PARAMS if ni else {}
    p = orc.Params(limiter=lim, max_steps=25, fixed_steps=True, **kw)
    delta = _config_of(_capi.FP32, "march_tma_delta", tile_y=32, min_blocks=16)
    assert len(delta) >= 2
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc)
    want, tw, sw, _ = _gpu(U0, orc.Grid(nx, ny), p, bc, precision=_capi.FP32,
                           tile_config=delta[0])
    for cfg in delta[1:]:
        got, tg, sg, _ = _gpu(U0, orc.Grid(nx, ny), p, bc, precision=_capi.FP32, tile_config=cfg)
        assert sg == sw == sr
        if not ni:
            assert tg == tw
            assert np.array_equal(got, want), (cfg, float(np.max(np.abs(got - want))))
        else:
            assert abs(tg - tw) <= 1e-6 * tw
            assert_components(got, want, MIXED_L1, cr, what=cfg)
        assert_components(got, ref, MIXED_L1, cr, what=cfg)


@pytest.mark.parametrize("walls", [True, False])
def test_masked_increment_form_delta_ring_matches_own_stream(walls):
    """The same with solid cells on every edge (their stage-2 update reads the delta ring too):
    bit for bit against the own-stream march, within the FP32-mixed bar of the FP64 oracle."""
    nx, ny = 61, 45
    bc = (orc.OUTFLOW, orc.PERIODIC)
    mask = _edge_mask(nx, ny, seed=11)
    U0 = initial_state(wl.fourier_state(nx, ny, 6), 5.0 / 3.0, bc, mask, walls)
    p = orc.Params(limiter=orc.VANLEER, max_steps=25, fixed_steps=True)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(nx, ny), p, bc, mask, walls)
    delta = _config_of(_capi.FP32, "march_tma_delta", tile_y=32, min_blocks=16)
    outs = [_gpu(U0, orc.Grid(nx, ny), p, bc, mask, walls, precision=_capi.FP32, tile_config=c)
            for c in delta]
    for got, tg, sg, _ in outs:
        assert sg == sr and tg == outs[0][1]
        assert np.array_equal(got, outs[0][0])
        assert_components(got, ref, MIXED_L1, cr)


def test_fp64_van_leer_reciprocal_fallback_matches_oracle():
    """The FP64 strip march's van Leer limiter inverts the nine slope sums of a cell with one
    division over their product; where that product leaves the normal range each sum takes its
    own Newton-refined reciprocal. v_z and B_z of about 1e-150 (they stay that small: in 2D ideal
    MHD they evolve linearly) make the product of a smooth cell's sums underflow, so this solve
    runs the fallback in most cells; every component, v_z and B_z on their own scale, stays
    within the FP64 bar of the oracle."""
    n = 96
    prim = wl.fourier_state(n, n, 12)
    ys, xs = np.meshgrid(np.arange(n) / n, np.arange(n) / n, indexing="ij")
    prim["vz"] = 1e-150 * np.sin(2 * np.pi * (xs + 2 * ys))
    prim["bz"] = 1e-150 * np.cos(2 * np.pi * (3 * xs - ys))
    U0 = initial_state(prim, 5.0 / 3.0)
    p = orc.Params(limiter=orc.VANLEER, max_steps=20, fixed_steps=True)
    ref, tr, sr, cr = orc.solve(U0, orc.Grid(n, n), p)
    slopes = np.abs(np.diff(interior(U0)[[3, 7]], axis=2))
    assert 0 < slopes[slopes > 0].max() < 1e-148
    marches = [c["config"] for c in _capi.tile_configs(_capi.FP64) if c["kind"] == "march_tma"]
    assert marches
    for cfg in marches:
        got, tg, sg, cg = _gpu(U0, orc.Grid(n, n), p, tile_config=cfg)
        assert sg == sr and abs(tg - tr) <= 1e-12 * tr
        assert_components(got, ref, FP64_L1, cr, what=cfg)
        for c in (3, 7):
            assert np.abs(interior(got)[c]).max() < 1e-145
