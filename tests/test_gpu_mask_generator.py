"""The device-side mask rasteriser (mhdb_configure_shapes) against the host rasterisation
(workloads.rasterize, the rule of the reference's gui/geometry.py:22-38, :130-156): bit for bit
at the masked workload's 2048^2 and at served sizes, with fluid paint over solid, rectangles
given by either pair of corners, more shapes than one launch carries, no shapes at all and a
domain other than the unit square; and a solve configured from shapes equals the same solve
configured from the host mask, bit for bit."""

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200 import workloads as wl
from oracle import oracle as orc
from tests.helpers import initial_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_device():
    if not _capi.cuda_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")


def device_mask(nx, ny, shapes, domain=(0.0, 1.0, 0.0, 1.0)):
    dev = _capi.DeviceSolver(nx, ny, *domain)
    try:
        dev.configure_shapes(_capi.BC_OUTFLOW, _capi.BC_PERIODIC, shapes)
        return dev.get_mask()
    finally:
        dev.close()


@pytest.mark.parametrize("n,seed", [(2048, 0), (2048, 3), (128, 1), (300, 7), (1000, 2)])
def test_seeded_circles_and_rectangles_bit_exact(n, seed):
    shapes = wl.circles_and_rectangles_shapes(seed)
    want = wl.circles_and_rectangles(n, n, seed)
    got = device_mask(n, n, shapes)
    assert got.dtype == np.uint8 and np.array_equal(got, want)
    assert (got == 0).any()


def _random_shapes(rng, count):
    shapes = []
    for _ in range(count):
        if rng.uniform() < 0.5:
            shapes.append((wl.CIRCLE, int(rng.uniform() < 0.7), *rng.uniform(-0.2, 1.2, size=2),
                           rng.uniform(0.0, 0.3), 0.0))
        else:  # corners in either order
            shapes.append((wl.RECTANGLE, int(rng.uniform() < 0.7), *rng.uniform(-0.2, 1.2, 4)))
    return [tuple(float(v) if i > 1 else int(v) for i, v in enumerate(s)) for s in shapes]


@pytest.mark.parametrize("nx,ny,count,domain", [
    (517, 263, 150, (0.0, 1.0, 0.0, 1.0)),   # three launches of shapes
    (64, 200, 64, (0.0, 1.0, 0.0, 1.0)),     # exactly one full launch
    (333, 97, 20, (-0.5, 1.5, 0.25, 0.75)),  # cell size and origin other than the unit square
])
def test_random_shapes_with_fluid_paint_bit_exact(nx, ny, count, domain):
    rng = np.random.Generator(np.random.PCG64(nx * 1000 + count))
    shapes = _random_shapes(rng, count)
    # shapes in the domain's coordinates
    x0, x1, y0, y1 = domain
    shapes = [(k, s, x0 + a * (x1 - x0), y0 + b * (y1 - y0), x0 + c * (x1 - x0) if k else
               c * (x1 - x0), y0 + d * (y1 - y0) if k else 0.0) for k, s, a, b, c, d in shapes]
    want = wl.rasterize(shapes, nx, ny, *domain)
    got = device_mask(nx, ny, shapes, domain)
    assert np.array_equal(got, want), int(np.sum(got != want))


def test_no_shapes_is_all_fluid():
    assert np.all(device_mask(40, 30, []) == 1)
    assert np.all(device_mask(40, 30, [(wl.CIRCLE, 0, 0.5, 0.5, 0.3, 0.0)]) == 1)


def test_solve_from_shapes_equals_solve_from_host_mask():
    n = 96
    bc = (orc.OUTFLOW, orc.PERIODIC)
    shapes = wl.circles_and_rectangles_shapes(5)
    mask = wl.rasterize(shapes, n, n)
    U0 = initial_state(wl.fourier_state(n, n, 4), 5.0 / 3.0, bc, mask)
    cp = _capi.make_params(limiter=_capi.VANLEER, ohmic=True, hall=True, ambipolar=True,
                           eta_ohm=1e-3, eta_hall=1e-2, eta_ambipolar=1e-3)
    outs = []
    for precision in (_capi.FP64, _capi.FP32):
        for from_shapes in (False, True):
            dev = _capi.DeviceSolver(n, n, precision=precision)
            try:
                if from_shapes:
                    dev.configure_shapes(bc[0], bc[1], shapes, True)
                else:
                    dev.configure(bc[0], bc[1], mask, True)
                dev.upload(U0)
                r = dev.solve_steps(cp, 12)
                outs.append((dev.download(), r.steps, r.t))
            finally:
                dev.close()
    for a, b in ((outs[0], outs[1]), (outs[2], outs[3])):
        assert a[1] == b[1] == 12 and a[2] == b[2]
        assert np.array_equal(a[0], b[0])
