"""Host-side logic without a GPU: the numpy ghost fill and wall fill of the Python surface
against the oracle, the boundary index maps, and the seeded workload generators."""

import os

import numpy as np
import pytest

from mhd_gpu_solver_b200 import mhd_solver as ms
from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("nx,ny", [(1, 1), (1, 3), (3, 1), (2, 5), (7, 4), (33, 9)])
@pytest.mark.parametrize("bc", [(0, 0), (2, 2), (0, 2), (2, 0)])
@pytest.mark.parametrize("ng", [2, 3])
def test_ghost_fill_matches_reference_order(nx, ny, bc, ng):
    rng = np.random.Generator(np.random.PCG64(nx * 100 + ny))
    U = rng.standard_normal((9, ny + 2 * ng, nx + 2 * ng))
    ref = orc.apply_bc(U, orc.Grid(nx, ny, ng), bc)
    got = U.copy()
    ms.apply_boundary_conditions(got, nx, ny, ng, bc[0], bc[1])
    assert np.array_equal(got, ref)


def test_reflective_boundary_is_rejected():
    U = np.zeros((9, 8, 8))
    with pytest.raises(ValueError, match="Reflective"):
        ms.apply_boundary_conditions(U, 4, 4, 2, 1, 0)


@pytest.mark.parametrize("seed", range(4))
def test_wall_fill_bitwise_equal_to_oracle(seed):
    nx, ny = 29, 23
    rng = np.random.Generator(np.random.PCG64(seed))
    mask = (rng.uniform(size=(ny, nx)) > 0.3).astype(np.uint8)
    mask[5:9, 5:9] = 0  # an interior solid block with cells that have no fluid neighbour
    prim = wl.fourier_state(nx, ny, seed)
    U = wl.embed(wl.to_conservative(prim, 1.4))
    U = orc.apply_bc(U, orc.Grid(nx, ny), (0, 2))
    ref = orc.wall_fill(U, orc.Grid(nx, ny), mask, 1.4)
    got = U.copy()
    ms.apply_solid_wall_fill(got, mask, 2, 1.4)
    assert np.array_equal(got, ref)


def test_workloads_are_seeded_and_shaped():
    a = wl.fourier_state(64, 48, 3)
    b = wl.fourier_state(64, 48, 3)
    c = wl.fourier_state(64, 48, 4)
    for k in wl.FIELDS:
        assert a[k].shape == (48, 64)
        assert np.array_equal(a[k], b[k])
    assert not np.array_equal(a["vx"], c["vx"])
    # velocity and field normalised to rms 1, perturbations clipped to [-0.2, 0.2]
    assert abs(np.sqrt(np.mean(a["vx"] ** 2 + a["vy"] ** 2)) - 1.0) < 1e-12
    assert abs(np.sqrt(np.mean(a["bx"] ** 2 + a["by"] ** 2)) - 1.0) < 1e-12
    assert a["rho"].min() >= 0.8 - 1e-15 and a["rho"].max() <= 1.2 + 1e-15
    assert a["p"].min() >= 0.8 - 1e-15 and a["p"].max() <= 1.2 + 1e-15
    assert np.all(a["vz"] == 0) and np.all(a["bz"] == 0) and np.all(a["psi"] == 0)


def test_fourier_field_is_divergence_free_in_the_continuum():
    # Analytic curl of A_z: the spectral divergence of (bx, by) vanishes to round-off.
    n = 64
    f = wl.fourier_state(n, n, 1)
    kx = np.fft.fftfreq(n) * n
    BX, BY = np.fft.fft2(f["bx"]), np.fft.fft2(f["by"])
    div = kx[None, :] * BX + kx[:, None] * BY
    assert np.max(np.abs(div)) < 1e-9 * np.max(np.abs(BX))


def test_quadrants_and_mask_generators():
    q = wl.four_quadrant(16, 16, 0)
    assert np.all(q["bx"] == 0.75)
    assert len(np.unique(q["rho"])) == 4
    assert q["rho"].min() >= 0.1 and q["rho"].max() <= 2.0
    m = wl.circles_and_rectangles(256, 256, 0)
    assert m.dtype == np.uint8 and set(np.unique(m)) <= {0, 1}
    assert 0.01 < 1.0 - m.mean() < 0.6
    assert np.array_equal(m, wl.circles_and_rectangles(256, 256, 0))


def test_python_surface_names_match_reference_module():
    names = ["set_num_threads", "num_threads", "set_simd_enabled", "simd_enabled",
             "simd_backend", "simd_width", "metal_available", "cuda_available",
             "available_backends", "SlopeLimiter", "BoundaryConditionType", "NonIdealConfig",
             "SolveResult", "SolveParams", "MHDSolver"]
    for n in names:
        assert hasattr(ms, n), n
    methods = ["set_periodic_bc", "set_outflow_bc", "set_bc", "set_gamma", "set_cfl",
               "set_glm_alpha", "set_limiter_minmod", "set_limiter_mc", "set_ideal",
               "enable_ohmic", "enable_hall", "enable_ambipolar", "disable_ohmic",
               "disable_hall", "disable_ambipolar", "set_mask", "get_mask", "clear_mask",
               "set_walls_reflective", "walls_reflective", "set_field", "set_primitives",
               "initialize", "set_backend", "backend", "backend_device", "run", "advance_to",
               "time", "steps", "c_h", "max_div_b", "field", "nx", "ny", "ng", "size_x",
               "size_y", "x_min", "x_max", "y_min", "y_max", "params"]
    for n in methods:
        assert hasattr(ms.MHDSolver, n), n
    p = ms.SolveParams()
    assert (p.t_end, p.cfl, p.gamma, p.glm_alpha, p.limiter, p.max_steps) == (
        0.0, 0.4, 5.0 / 3.0, 0.1, ms.SlopeLimiter.MC, 1_000_000)
    ni = ms.NonIdealConfig.with_ohmic(0.0)
    assert not ni.any()
    assert ni.enable_hall(1e-2).any()


def test_host_state_preparation_without_device():
    s = ms.MHDSolver(16, 12)
    s.set_outflow_bc()
    s.initialize("orszag_tang")
    rho = s.field("rho")
    assert rho.shape == (16, 20)
    assert np.all(rho[0] == rho[2]) and np.all(rho[:, 0] == rho[:, 2])
    m = np.ones((12, 16), np.uint8)
    m[4:6, 4:8] = 0
    s.set_mask(m)
    assert np.array_equal(s.get_mask(), m)
    with pytest.raises(ValueError):
        s.set_mask(np.ones((3, 3), np.uint8))
    with pytest.raises(ValueError, match="Unknown field"):
        s.field("nope")
    with pytest.raises(ValueError, match="Unknown initial condition"):
        s.initialize("nope")
    with pytest.raises(RuntimeError, match="Backend not available: cpu"):
        s.set_backend("cpu")
    with pytest.raises(ValueError, match="Unknown backend"):
        s.set_backend("tpu")


def test_bench_traffic_lookup_covers_every_march_tma_kind():
    """The bench's roofline traffic comes from the committed ncu figure of the dominant kernel's
    kind: both TMA strip-march forms have one, scaled by cells; other kinds report none."""
    import bench

    for kind, s2 in (("march_tma", 215.1), ("march_tma_delta", 182.9)):
        traffic, src = bench.measured_traffic(kind, 2, 1000.0)
        assert traffic == pytest.approx(s2 * 1000.0) and src
    assert bench.measured_traffic("tile", 2, 1000.0) == (None, None)
    assert bench.BYTES_FORM["march_tma_delta"] == {1: 72.0, 2: 180.0}


def test_bench_state_is_the_reference_ghost_fill_and_loads_no_cuda_library():
    """The bench's 4096^2 state builder (numpy wrap padding) equals embed + the reference's
    periodic ghost fill, and the reference arm's path (bench.initial_state, the oracle front end)
    imports no module that loads libmhd_b200.so."""
    import subprocess
    import sys

    import bench
    from mhd_gpu_solver_b200 import workloads as wl
    from mhd_gpu_solver_b200.mhd_solver import apply_boundary_conditions

    n = 20
    U = wl.embed(wl.to_conservative(wl.fourier_state(n, n, bench.SEED), bench.GAMMA))
    apply_boundary_conditions(U, n, n, 2, 0, 0)
    assert np.array_equal(bench.initial_state(n), U)
    probe = ("import sys; sys.path.insert(0, %r); import bench; bench.initial_state(8); "
             "from oracle import oracle; "
             "print(sorted(m for m in sys.modules if m.startswith('mhd_gpu_solver_b200')))"
             % ROOT)
    res = subprocess.run([sys.executable, "-c", probe], capture_output=True, text=True,
                         timeout=120)
    assert res.returncode == 0, res.stderr
    loaded = eval(res.stdout.strip().splitlines()[-1])
    assert "mhd_gpu_solver_b200._capi" not in loaded, loaded


def test_host_rasterize_follows_the_reference_rule_cell_by_cell():
    """workloads.rasterize against a per-cell restatement of gui/geometry.py:22-38 (contains:
    inclusive circle and rectangle tests, rectangle corners sorted) and :130-156 (rasterize: all
    fluid, shapes in order, later ones overwrite), on shapes whose edges pass through cell
    centres."""
    nx, ny = 10, 8
    shapes = [(wl.RECTANGLE, 1, 0.45, 0.0625, 0.05, 0.5625),  # corners reversed; edges on centres
              (wl.CIRCLE, 1, 0.75, 0.5, 0.2, 0.0),
              (wl.CIRCLE, 0, 0.75, 0.5, 0.1, 0.0),           # fluid paint inside the solid disc
              (wl.RECTANGLE, 0, 0.25, 0.3125, 0.35, 0.3125)]  # a one-row fluid strip
    got = wl.rasterize(shapes, nx, ny)
    xs, ys = wl.cell_centers(nx, ny)
    want = np.ones((ny, nx), dtype=np.uint8)
    for j in range(ny):
        for i in range(nx):
            x, y = float(xs[i]), float(ys[j])
            for kind, solid, a, b, c, d in shapes:
                if kind == wl.CIRCLE:
                    hit = (x - a) ** 2 + (y - b) ** 2 <= c ** 2
                else:
                    hit = min(a, c) <= x <= max(a, c) and min(b, d) <= y <= max(b, d)
                if hit:
                    want[j, i] = 0 if solid else 1
    assert np.array_equal(got, want)
    # the strip's row is row 2 (y = 0.3125); its x range [0.25, 0.35] holds the centre 0.25 but
    # not 0.35000000000000003 (= 0.05 + 3 x 0.1 rounded), so one cell turns fluid
    assert (got == 0).any() and got[2, 2] == 1 and got[2, 3] == 0


def test_served_request_work_estimate():
    """The serving loop's admission order: a non-ideal request's estimate is exact (its dt is
    the diffusion limit cfl h^2 / (4 eta_max) with eta_max the Hall 1e-2), an ideal one's uses
    the CFL step at a typical signal speed, and the estimate grows with the grid side."""
    from mhd_gpu_solver_b200.serve import Request

    ni = Request(rid=0, arrival=0.0, n=512, t_end=0.2, kind="fourier", seed=1, nonideal=True)
    h = 1.0 / 512
    assert ni.work_estimate() == pytest.approx(512 * 512 * 0.2 / (0.4 * h * h / 0.04), rel=1e-12)
    small = Request(rid=1, arrival=0.0, n=128, t_end=0.2, kind="quadrants", seed=1, nonideal=False)
    big = Request(rid=2, arrival=0.0, n=1024, t_end=0.2, kind="quadrants", seed=1, nonideal=False)
    assert small.work_estimate() < big.work_estimate() < ni.work_estimate() * 10


def test_online_server_threading_with_a_fake_engine():
    """Server: submissions from two threads, completions through poll, results handed over once,
    summary counts, close waits for the submitted requests and stops the worker."""
    import threading

    from mhd_gpu_solver_b200.serve import Server
    from tests.serve_fakes import FakeEngine

    engines = []

    def factory(stats):
        engines.append(FakeEngine(stats, rounds=3))
        return engines[-1]

    srv = Server(engine_factory=factory)
    ids = []

    def submit_some(k):
        for i in range(k):
            ids.append(srv.submit(64 + i, 0.01, "quadrants" if i % 2 else "fourier", seed=i))

    threads = [threading.Thread(target=submit_some, args=(4,)) for _ in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    got = []
    for _ in range(200):
        got += srv.poll(timeout=0.05)
        if len(got) == 8:
            break
    assert sorted(c.rid for c in got) == sorted(ids) == list(range(8))
    for rid in ids:
        assert srv.result(rid)[0] == rid
    with pytest.raises(KeyError):
        srv.result(ids[0])  # handed over once
    s = srv.summary()
    assert s["requests"] == 8 and s["submitted"] == 8
    with pytest.raises(ValueError):
        srv.submit(64, 0.01, "vortex")
    with pytest.raises(ValueError):
        srv.submit(64, -1.0)
    srv.close()
    assert engines[0].closed
    with pytest.raises(RuntimeError, match="closed"):
        srv.submit(64, 0.01)


def test_online_server_reports_a_failed_solve():
    """A solve that fails in the worker stops it; poll and close raise the solve's error."""
    from mhd_gpu_solver_b200.serve import Server
    from tests.serve_fakes import FakeEngine

    srv = Server(engine_factory=lambda stats: FakeEngine(stats, rounds=2, fail_rid=1))
    srv.submit(64, 0.01)
    srv.submit(64, 0.01)
    with pytest.raises(RuntimeError, match="max_steps"):
        for _ in range(200):
            srv.poll(timeout=0.05)
    with pytest.raises(RuntimeError, match="max_steps"):
        srv.close()


def test_serving_engine_admission_policy_on_a_host():
    """The serving engine's admission (serve._Engine with a stand-in batch): shortest estimated
    work first, the cells cap (one request always runs), the memory cap in arrival order, joins
    while others run, every request completed and removed once."""
    from collections import deque

    from mhd_gpu_solver_b200 import _capi
    from mhd_gpu_solver_b200.serve import Request, ServeStats, _Engine, state_bytes
    from tests.serve_fakes import FakeBatch

    def stream():
        return [Request(rid=i, arrival=0.0, n=n, t_end=0.1, kind="fourier", seed=i,
                        nonideal=False) for i, n in enumerate([512, 128, 1024, 256])]

    def run(eng, q):
        while q or eng.busy:
            eng.admit(q)
            if eng.busy:
                eng.advance()

    stats, fb = ServeStats(), FakeBatch(rounds=2)
    cap = 2 * 512 * 512
    eng = _Engine(_capi.FP32, 150e9, 16, True, False, False, "shortest", cap, stats, batch=fb)
    q = eng.order_queue(deque(stream()))
    assert [r.n for r in q] == [128, 256, 512, 1024]
    eng.admit(q)
    assert [r.n for r in q] == [1024] and len(eng.active) == 3
    assert stats.cell_waits == 1 and stats.joins == 2
    run(eng, q)
    assert sorted(c.rid for c in stats.completions) == [0, 1, 2, 3]
    assert sorted(fb.removed) == [0, 1, 2, 3] and eng.in_use == 0 and eng.active_cells == 0
    assert stats.peak_cells == 1024 * 1024  # the 1024^2 request ran alone, above the cap

    stats, fb = ServeStats(), FakeBatch(rounds=3)
    mem = state_bytes(1024, 1024) + state_bytes(128, 128)
    eng = _Engine(_capi.FP32, mem, 16, True, False, False, "arrival", cap, stats, batch=fb)
    q = eng.order_queue(deque(stream()))
    assert [r.n for r in q] == [512, 128, 1024, 256]
    eng.admit(q)
    assert [r.n for r in q] == [1024, 256] and stats.cap_waits == 1
    run(eng, q)
    assert sorted(c.rid for c in stats.completions) == [0, 1, 2, 3]
    assert stats.peak_bytes <= mem
    with pytest.raises(ValueError):
        _Engine(_capi.FP32, mem, 16, True, False, False, "fifo", cap, ServeStats(), batch=fb)
