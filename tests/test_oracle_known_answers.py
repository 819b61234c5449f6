"""Known answers and invariants of the oracle that the reference's own unit tests state:
limiter values (tests/test_muscl_glm.cpp:14-39), Ohm's-law electric fields
(tests/test_nonideal.cpp:32-62), a uniform state has a zero right-hand side
(tests/test_mhd_operator.cpp:111-159) and a periodic solve conserves its totals
(tests/test_time_integrator.cpp:69-129). Van Leer, which the reference lacks, is checked against
its published formula 2ab/(a+b)."""

import numpy as np
import pytest

from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import initial_state, interior


def test_limiter_known_answers():
    assert orc.limiter(orc.MINMOD, 1.0, -1.0) == 0.0
    assert orc.limiter(orc.MINMOD, 2.0, 3.0) == 2.0
    assert orc.limiter(orc.MINMOD, -4.0, -1.0) == -1.0
    assert orc.limiter(orc.MINMOD, 1.0, 1.0) == 1.0
    assert orc.limiter(orc.MC, 1.0, 1.0) == 1.0
    assert orc.limiter(orc.MINMOD, 1.0, 10.0) == 1.0
    assert orc.limiter(orc.MC, 1.0, 10.0) == 2.0
    assert orc.limiter(orc.VANLEER, 1.0, 1.0) == 1.0
    assert orc.limiter(orc.VANLEER, 1.0, 3.0) == 1.5
    assert orc.limiter(orc.VANLEER, -2.0, -2.0) == -2.0
    assert orc.limiter(orc.VANLEER, 1.0, -1.0) == 0.0
    assert orc.limiter(orc.VANLEER, 0.0, 5.0) == 0.0


@pytest.mark.parametrize("which, J, B, expect", [
    ("ohmic", (1.0, -2.0, 0.5), (0.0, 0.0, 1.0), (0.3, -0.6, 0.15)),
    ("hall", (0.0, 0.0, 1.0), (1.0, 0.0, 0.0), (0.0, 0.2, 0.0)),
    ("ambipolar", (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), (0.0, -0.5, 0.0)),
])
def test_ohms_law_known_answers(which, J, B, expect):
    p = orc.Params()
    if which == "ohmic":
        p.ohmic, p.eta_ohm = True, 0.3
    elif which == "hall":
        p.hall, p.eta_hall = True, 0.2
    else:
        p.ambipolar, p.eta_ambipolar = True, 0.5
    assert np.allclose(orc.nonideal_e(J, B, p), expect, rtol=0.0, atol=1e-12)


@pytest.mark.parametrize("ni", [False, True])
def test_uniform_state_has_zero_rhs(ni):
    n = 12
    prim = {k: np.full((n, n), v) for k, v in dict(rho=1.3, vx=0.4, vy=-0.2, vz=0.1, p=0.8,
                                                   bx=0.7, by=-0.3, bz=0.2, psi=0.0).items()}
    U = initial_state(prim, 5.0 / 3.0)
    p = orc.Params(limiter=orc.MC)
    if ni:
        p.ohmic = p.hall = p.ambipolar = True
        p.eta_ohm, p.eta_hall, p.eta_ambipolar = 1e-3, 1e-2, 1e-3
    L = orc.rhs(U, orc.Grid(n, n), p, c_h=1.5)
    assert np.max(np.abs(L)) <= 1e-13


@pytest.mark.parametrize("lim", [orc.MINMOD, orc.MC, orc.VANLEER])
def test_periodic_solve_conserves_totals(lim):
    n = 40
    U0 = initial_state(wl.fourier_state(n, n, 5), 5.0 / 3.0)
    p = orc.Params(limiter=lim, max_steps=25, fixed_steps=True)
    out, _, steps, _ = orc.solve(U0, orc.Grid(n, n), p)
    assert steps == 25
    a = interior(U0).reshape(9, -1).sum(axis=1)
    b = interior(out).reshape(9, -1).sum(axis=1)
    scale = np.abs(interior(U0)).reshape(9, -1).sum(axis=1)
    # rho, momentum, energy and B are conserved (psi is damped)
    assert np.all(np.abs(b - a)[:8] <= 1e-12 * scale[:8])


_THREAD_PROBE = """
import hashlib, sys
import numpy as np
sys.path.insert(0, {root!r})
from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import initial_state
bc = (orc.OUTFLOW, orc.PERIODIC)
mask = wl.circles_and_rectangles(67, 45, 2)
U0 = initial_state(wl.fourier_state(67, 45, 4), 5.0 / 3.0, bc, mask)
p = orc.Params(limiter=orc.VANLEER, ohmic=True, hall=True, ambipolar=True, eta_ohm=1e-3,
               eta_hall=1e-2, eta_ambipolar=1e-3, max_steps=12, fixed_steps=True)
out, t, steps, c_h = orc.solve(U0, orc.Grid(67, 45), p, bc, mask)
print(hashlib.sha256(out.tobytes()).hexdigest(), t.hex(), steps, c_h.hex())
"""


def test_oracle_results_do_not_depend_on_the_thread_count():
    """The oracle's loops run on all host threads (OpenMP); every value they write depends only
    on inputs of the same pass and the CFL maximum is combined per row, so 1 and 3 threads give
    the same bits."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for threads in ("1", "3"):
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        res = subprocess.run([sys.executable, "-c", _THREAD_PROBE.format(root=root)], env=env,
                             capture_output=True, text=True, timeout=300)
        assert res.returncode == 0, res.stderr
        outs.append(res.stdout.strip())
    assert outs[0] == outs[1] and outs[0]
