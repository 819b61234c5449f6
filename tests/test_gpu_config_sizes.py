"""Parity at the benchmark workloads' own sizes and step counts.

* Smooth periodic Fourier state at 1024^2, 500 SSP-RK2 steps, MC limiter (the reference offers
  minmod and MC only): the plain FP64 form against the reference CPU solver, compiled from the
  reference's own sources into oracle/_ref, to relative L1 <= 1e-12 per conserved component with
  the same step count; the FP32-mixed form to <= 1e-6. Both the size's default FP64 kernel and
  the FP64 TMA strip march (the default of grids from 2048^2, the 4096^2 kernel) are held.
* Non-ideal and masked at 2048^2, 300 steps: the same Fourier state with Ohmic 1e-3, Hall 1e-2
  and ambipolar 1e-3, 12 circles and 6 rectangles of reflective walls, outflow in x and periodic
  in y, MC: FP64 <= 1e-12 and FP32-mixed <= 1e-6 against the reference CPU solver; the on-device
  FP64 diagnostics of the FP64 result (div B L2 and max, mass, energy) against the oracle's on the
  reference's result.
* Van Leer (no reference counterpart) at 1024^2, 500 steps: both forms against the C oracle.
* The reference's own GPU gate (tools/mhd_backend_compare.cpp --gate), compiled with this backend
  in its CUDA seam: Orszag-Tang ideal and Ohmic+Hall against the reference's FP64 CPU solution,
  Alfven-wave convergence order, for the FP64 and FP32 (here FP32-mixed) backends.

Every component is held (tests.helpers.component_errors): relative L1, absolute where the
reference is identically zero, psi on the scale max(sum|psi|, c_h sum|B|); under the FP32-mixed
bar the components of m and B on their vector's scale (with the Hall term, B_z and m_z are
generated by a second derivative of B that FP32 resolves to about 1e-5 of B_z itself at 2048^2;
their plain relative L1 is printed beside).
"""

import os
import subprocess
import tempfile

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc
from tests.gpu_util import gpu_solve
from tests.helpers import assert_components, component_errors, initial_state

pytestmark = pytest.mark.gpu

FP64_L1 = 1e-12
MIXED_L1 = 1e-6
NI = dict(ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3, eta_hall=1e-2,
          eta_ambipolar=1e-3)
REF_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                       "_ref")


@pytest.fixture(scope="module", autouse=True)
def _need_device_and_reference():
    if not _capi.cuda_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")
    if orc.ref_library_path() is None:
        pytest.skip("reference CPU solver not built (oracle/_ref)")
    orc.ref_set_threads(os.cpu_count() or 1)


def _fp64_march_config() -> int:
    return next(c["config"] for c in _capi.tile_configs(_capi.FP64) if c["kind"] == "march_tma")


def _check_steps(got_r, ref_r, tol):
    _, tg, sg, cg = got_r
    _, tr, sr, cr = ref_r
    assert sg == sr, (sg, sr)
    assert abs(tg - tr) <= tol * tr and abs(cg - cr) <= tol * cr, (tg, tr, cg, cr)


def test_fourier_1024_500_steps_mc_against_reference_cpu_solver():
    n, steps = 1024, 500
    U0 = initial_state(wl.fourier_state(n, n, 0), 5.0 / 3.0)
    p = orc.Params(limiter=orc.MC, max_steps=steps, fixed_steps=True)
    ref = orc.solve(U0, orc.Grid(n, n), p, impl="ref")
    for cfg in (-1, _fp64_march_config()):
        got = gpu_solve(U0, orc.Grid(n, n), p, tile_config=cfg)
        _check_steps(got, ref, 1e-12)
        err = assert_components(got[0], ref[0], FP64_L1, ref[3], what=("fp64", cfg))
        print("1024^2 MC 500 steps FP64 configuration", cfg, "L1:", err)
    got = gpu_solve(U0, orc.Grid(n, n), p, precision=_capi.FP32)
    _check_steps(got, ref, 1e-6)
    err = assert_components(got[0], ref[0], MIXED_L1, ref[3], what="fp32_mixed")
    print("1024^2 MC 500 steps FP32-mixed L1:", err)


def test_masked_nonideal_2048_300_steps_against_reference_cpu_solver():
    n, steps = 2048, 300
    bc = (orc.OUTFLOW, orc.PERIODIC)
    mask = wl.circles_and_rectangles(n, n, 0)
    U0 = initial_state(wl.fourier_state(n, n, 0), 5.0 / 3.0, bc, mask)
    p = orc.Params(limiter=orc.MC, max_steps=steps, fixed_steps=True, **NI)
    ref = orc.solve(U0, orc.Grid(n, n), p, bc, mask, impl="ref")
    # FP64 through one handle, so that its diagnostics see the device's own result: solid cells
    # keep their stored (pre-fill) values on the device, which the ghosts of the reference's final
    # state hold (BC before wall fill), and a download fills them
    dev = _capi.DeviceSolver(n, n)
    try:
        dev.configure(bc[0], bc[1], mask, True)
        dev.upload(U0)
        r = dev.solve_steps(_capi.make_params(limiter=_capi.MC, **NI), steps)
        d = dev.diagnostics(_capi.make_params(limiter=_capi.MC, **NI))
        got = (dev.download(), r.t, r.steps, r.c_h)
    finally:
        dev.close()
    _check_steps(got, ref, 1e-12)
    err = assert_components(got[0], ref[0], FP64_L1, ref[3], what="fp64")
    print("2048^2 masked non-ideal 300 steps FP64 L1:", err)
    mixed = gpu_solve(U0, orc.Grid(n, n), p, bc, mask, precision=_capi.FP32)
    _check_steps(mixed, ref, 1e-6)
    err = assert_components(mixed[0], ref[0], MIXED_L1, ref[3], what="fp32_mixed")
    print("2048^2 masked non-ideal 300 steps FP32-mixed L1:", err, "plain relative:",
          component_errors(mixed[0], ref[0], ref[3]))

    # FP64 diagnostics on the device against the oracle's on the reference's final state
    dref = orc.diagnostics(ref[0], orc.Grid(n, n), p.gamma)
    for k in ("mass", "energy", "div_b_max", "div_b_l2", "rho_min", "p_min"):
        assert abs(d[k] - dref[k]) <= 1e-11 * max(1.0, abs(dref[k])), (k, d[k], dref[k])
    assert d["finite"] and dref["finite"]


def test_fourier_1024_500_steps_van_leer_against_oracle():
    n, steps = 1024, 500
    U0 = initial_state(wl.fourier_state(n, n, 0), 5.0 / 3.0)
    p = orc.Params(limiter=orc.VANLEER, max_steps=steps, fixed_steps=True)
    ref = orc.solve(U0, orc.Grid(n, n), p)
    got = gpu_solve(U0, orc.Grid(n, n), p, tile_config=_fp64_march_config())
    _check_steps(got, ref, 1e-12)
    err = assert_components(got[0], ref[0], FP64_L1, ref[3], what="fp64")
    print("1024^2 van Leer 500 steps FP64 L1:", err)
    mixed = gpu_solve(U0, orc.Grid(n, n), p, precision=_capi.FP32)
    _check_steps(mixed, ref, 1e-6)
    err = component_errors(mixed[0], ref[0], ref[3], vector_scale=True)
    print("1024^2 van Leer 500 steps FP32-mixed L1:", err)
    assert np.all(err <= MIXED_L1), err


def test_reference_gpu_gate_passes():
    """tools/mhd_backend_compare.cpp --gate of the reference (registered there as the
    GpuGate.Accuracy test), with the speed check off: rc 0 means every accuracy check passed."""
    tool = os.path.join(REF_DIR, "mhd_backend_compare")
    if not os.path.exists(tool):
        pytest.skip("reference gate tool with the B200 backend not built (needs the reference)")
    with tempfile.TemporaryDirectory() as d:
        md = os.path.join(d, "gate.md")
        res = subprocess.run([tool, "--gate", "--no-speed", "--require-gpu", "--markdown", md],
                             capture_output=True, text=True, timeout=900)
        print(res.stderr[-4000:])
        assert res.returncode == 0, res.stdout[-4000:] + res.stderr[-4000:]
        text = open(md).read()
    assert "## GPU gate: passed" in text and "\u274c" not in text
    assert "[FAIL]" not in res.stderr
    assert "CUDA fp64" in text and "CUDA fp32" in text
