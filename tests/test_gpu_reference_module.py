"""The reference's own Python module with this backend plugged into its CUDA seam.

oracle/_ref/mhd_solver*.so is the reference's python/mhd_pybind.cpp compiled from its sources
with -DMHD_HAS_CUDA=1 and mhd_gpu_solver_b200/csrc/reference_backend.cpp. Its
MHDSolver.set_backend("cuda", ...) therefore runs the B200 kernels, and its default "cpu"
backend is the reference CPU solver. These tests restate the reference's GPU-vs-CPU tests
(tests/test_gpu_backends.cpp:22-157) through that module, with its tolerances: equal step
count, |t - t_cpu| <= 1e-6, relative Linf of rho and energy <= 1e-11 (FP64) or 2e-5 (FP32),
by within 10x that.
"""

import glob
import importlib
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


@pytest.fixture(scope="module")
def ms():
    if not glob.glob(os.path.join(REF, "mhd_solver*.so")):
        pytest.skip("reference module with the B200 backend not built (needs the reference)")
    sys.path.insert(0, REF)
    try:
        mod = importlib.import_module("mhd_solver")
    finally:
        sys.path.remove(REF)
    assert mod.cuda_available(), "the B200 backend reports no CUDA device"
    return mod


BACKENDS = [("fp64", 1e-11), ("fp32", 2e-5)]


def rel_linf(a, b):
    d = np.max(np.abs(a - b))
    s = np.max(np.abs(b))
    return d / s if s > 0 else d


def compare_with_cpu(ms, nx, ny, t_end, setup):
    y_max = 1.0 / nx if ny == 1 else 1.0
    cpu = ms.MHDSolver(nx, ny, 0.0, 1.0, 0.0, y_max)
    setup(cpu)
    rc = cpu.run(t_end)
    for prec, tol in BACKENDS:
        gpu = ms.MHDSolver(nx, ny, 0.0, 1.0, 0.0, y_max)
        setup(gpu)
        gpu.set_backend("cuda", prec)
        rg = gpu.run(t_end)
        label = gpu.backend_device() + " " + prec
        assert "B200" in label
        assert rg.steps == rc.steps, label
        assert abs(rg.t - rc.t) <= 1e-6 * max(1.0, t_end), label
        assert rel_linf(gpu.field("rho"), cpu.field("rho")) < tol, label
        assert rel_linf(gpu.field("energy"), cpu.field("energy")) < tol, label
        assert rel_linf(gpu.field("by"), cpu.field("by")) < 10 * tol, label


def test_orszag_tang_matches_cpu(ms):
    def setup(s):
        s.set_limiter_mc()
        s.initialize("orszag_tang")
    compare_with_cpu(ms, 48, 40, 0.05, setup)


def test_minmod_outflow_sod_matches_cpu(ms):
    def setup(s):
        s.set_limiter_minmod()
        s.set_bc(ms.BoundaryConditionType.Outflow, ms.BoundaryConditionType.Periodic)
        s.initialize("sod")
    compare_with_cpu(ms, 64, 1, 0.05, setup)


def test_nonideal_matches_cpu(ms):
    def setup(s):
        s.initialize("orszag_tang")
        s.enable_ohmic(2e-3)
        s.enable_hall(1e-3)
        s.enable_ambipolar(5e-4)
    compare_with_cpu(ms, 32, 32, 0.03, setup)


def test_solid_mask_matches_cpu(ms):
    def setup(s):
        s.initialize("orszag_tang")
        m = np.ones((40, 40), dtype=np.uint8)
        m[15:25, 12:20] = 0
        s.set_mask(m)
    compare_with_cpu(ms, 40, 40, 0.03, setup)


def test_repeated_runs_accumulate_time(ms):
    for prec, _ in BACKENDS:
        s = ms.MHDSolver(32, 32)
        s.initialize("orszag_tang")
        s.set_backend("cuda", prec)
        s.run(0.01)
        r = s.advance_to(0.02)
        assert abs(r.t - 0.02) <= 1e-12
        assert r.steps > 0
        with pytest.raises(ValueError):
            s.run(-1.0)


def test_max_steps_is_enforced(ms):
    for prec, _ in BACKENDS:
        s = ms.MHDSolver(32, 32)
        s.initialize("orszag_tang")
        s.params.max_steps = 3
        s.set_backend("cuda", prec)
        with pytest.raises(RuntimeError, match="max_steps"):
            s.run(1.0)
