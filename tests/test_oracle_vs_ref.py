"""The C restatement against the reference CPU solver compiled from its own headers
(oracle/_ref): full solves and single operator evaluations on odd grids with every feature."""

import numpy as np
import pytest

from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import initial_state, rel_l1

pytestmark = pytest.mark.skipif(orc.ref_library_path() is None,
                                reason="reference CPU library not built (oracle/_ref)")

TOL = 1e-13


def block_mask(nx, ny, edges=False):
    m = np.ones((ny, nx), dtype=np.uint8)
    m[ny // 3: ny // 2, nx // 4: nx // 2] = 0
    if edges:
        m[0, :5] = 0
        m[-2:, -3:] = 0
        m[ny // 2, 0] = 0
        m[3:6, -1] = 0
        m[-1, nx // 2] = 0
    return m


CASES = [
    # name, prim, bc, limiter, nonideal, mask
    ("ot_mc_periodic", lambda: wl.orszag_tang(37, 29), (orc.PERIODIC, orc.PERIODIC), orc.MC, None,
     None),
    ("ot_minmod_outflow", lambda: wl.orszag_tang(37, 29), (orc.OUTFLOW, orc.OUTFLOW), orc.MINMOD,
     None, None),
    ("quadrant_mixed_bc", lambda: wl.four_quadrant(37, 29, 3), (orc.OUTFLOW, orc.PERIODIC),
     orc.MINMOD, None, None),
    ("fourier_nonideal", lambda: wl.fourier_state(37, 29, 1), (orc.PERIODIC, orc.PERIODIC), orc.MC,
     (2e-3, 1e-3, 5e-4), None),
    ("fourier_mask_edges", lambda: wl.fourier_state(37, 29, 2), (orc.OUTFLOW, orc.PERIODIC),
     orc.MC, (1e-3, 1e-2, 1e-3), "edges"),
    ("ot_mask_block", lambda: wl.orszag_tang(40, 40), (orc.PERIODIC, orc.PERIODIC), orc.MC, None,
     "block"),
]


def setup(case):
    name, mk, bc, lim, ni, mk_mask = case
    prim = mk()
    ny, nx = prim["rho"].shape
    mask = None
    if mk_mask == "block":
        mask = block_mask(nx, ny)
    elif mk_mask == "edges":
        mask = block_mask(nx, ny, edges=True)
    p = orc.Params(cfl=0.4, gamma=5.0 / 3.0, glm_alpha=0.1, limiter=lim, max_steps=25,
                   fixed_steps=True)
    if ni:
        p.ohmic, p.hall, p.ambipolar = True, True, True
        p.eta_ohm, p.eta_hall, p.eta_ambipolar = ni
    U0 = initial_state(prim, p.gamma, bc, mask)
    return U0, orc.Grid(nx, ny), p, bc, mask


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_solve_matches_reference(case):
    U0, grid, p, bc, mask = setup(case)
    a, ta, sa, ca = orc.solve(U0, grid, p, bc, mask)
    b, tb, sb, cb = orc.solve(U0, grid, p, bc, mask, impl="ref")
    assert sa == sb
    assert abs(ta - tb) <= 1e-13 * tb
    err = rel_l1(a, b)
    assert np.all(err <= TOL), err
    # ghosts (final BC + wall fill) too
    assert np.max(np.abs(a - b)) <= 1e-11 * max(1.0, np.max(np.abs(b)))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_rhs_matches_reference(case):
    U0, grid, p, bc, mask = setup(case)
    _, c_h = orc.cfl(U0, grid, p, mask)
    ra = orc.rhs(U0, grid, p, c_h, mask)
    rb = orc.rhs(U0, grid, p, c_h, mask, impl="ref")
    # Components that vanish analytically (e.g. d rho/dt of Orszag-Tang) are round-off noise:
    # measure every component against the largest RHS magnitude.
    scale = np.max(np.abs(rb))
    assert np.max(np.abs(ra - rb)) <= 1e-12 * scale


def test_time_based_solve_matches_reference_and_max_steps():
    U0 = initial_state(wl.orszag_tang(48, 40), 5.0 / 3.0)
    p = orc.Params(t_end=0.05, limiter=orc.MC)
    a, ta, sa, _ = orc.solve(U0, orc.Grid(48, 40), p)
    b, tb, sb, _ = orc.solve(U0, orc.Grid(48, 40), p, impl="ref")
    assert sa == sb and ta == tb == 0.05
    assert np.all(rel_l1(a, b) <= TOL)
    p.max_steps = 3
    for impl in ("oracle", "ref"):
        with pytest.raises(orc.OracleError) as e:
            orc.solve(U0, orc.Grid(48, 40), p, impl=impl)
        assert e.value.code == orc.EMAXSTEPS
