"""Serving form: requests that arrive while others run are admitted under the memory cap, all
complete, and each result is the same alone and in the mix (bit for bit), and within the FP32-mixed
tolerance of the plain FP64 path."""

import numpy as np
import pytest

from mhd_gpu_solver_b200 import _capi
from mhd_gpu_solver_b200.batch import state_bytes
from mhd_gpu_solver_b200.serve import make_stream, serve, serve_one_at_a_time
from tests.helpers import assert_components

pytestmark = pytest.mark.gpu


def small_stream(n=12, seed=5):
    return make_stream(n, rate=400.0, seed=seed, side=(40, 160), t_end=(0.005, 0.02),
                       nonideal_frac=0.3)


def test_served_results_equal_alone_and_fp64_path():
    reqs = small_stream()
    mixed = serve(reqs, keep_states=True)
    assert len(mixed.completions) == len(reqs)
    assert mixed.max_active > 1  # requests overlapped on the device
    for req in reqs:
        alone = serve([req], keep_states=True)
        assert np.array_equal(alone.states[req.rid], mixed.states[req.rid]), req
    plain = serve_one_at_a_time(reqs, keep_states=True)
    steps_mixed = {c.rid: c.steps for c in mixed.completions}
    for c in plain.completions:
        assert abs(steps_mixed[c.rid] - c.steps) <= 1
        assert_components(mixed.states[c.rid], plain.states[c.rid], 1e-6, what=c.rid)


def test_admission_respects_the_memory_cap():
    reqs = small_stream(10, seed=9)
    cap = 2.5 * max(state_bytes(r.n, r.n) for r in reqs)
    stats = serve(reqs, memory_cap=cap)
    assert len(stats.completions) == len(reqs)
    assert stats.peak_bytes <= cap
    s = stats.summary()
    assert s["p99_ms"] >= s["p50_ms"] > 0.0


def test_shortest_first_admission_keeps_results_and_the_cells_cap():
    """Shortest-estimated-work-first admission under a cap of running cells: every request
    completes, no admission takes the running cells over the cap (one request always runs), and
    each result equals the arrival-order serve's bit for bit (a solve's values do not depend on
    the requests beside it)."""
    reqs = small_stream(14, seed=11)
    cap = 2 * max(r.n * r.n for r in reqs)
    fifo = serve(reqs, keep_states=True, order="arrival")
    sjf = serve(reqs, keep_states=True, order="shortest", cells_cap=cap)
    assert len(sjf.completions) == len(fifo.completions) == len(reqs)
    assert sjf.peak_cells <= cap
    for req in reqs:
        assert np.array_equal(sjf.states[req.rid], fifo.states[req.rid]), req
    steps = {c.rid: c.steps for c in fifo.completions}
    assert all(c.steps == steps[c.rid] for c in sjf.completions)


def test_online_server_equals_serve():
    """The online Server (worker thread, requests submitted while others run) gives every request
    the state serve() gives it, bit for bit, with the same step count."""
    import time

    from mhd_gpu_solver_b200.serve import Server

    reqs = small_stream(8, seed=13)
    want = serve(reqs, keep_states=True)
    steps = {c.rid: c.steps for c in want.completions}
    with Server(keep_states=True) as srv:
        of = {}
        for r in reqs:
            of[srv.submit(r.n, r.t_end, r.kind, r.seed, r.nonideal)] = r
            time.sleep(0.002)
        got = []
        deadline = time.time() + 300
        while len(got) < len(reqs) and time.time() < deadline:
            got += srv.poll(timeout=1.0)
        assert len(got) == len(reqs)
        for c in got:
            r = of[c.rid]
            assert c.steps == steps[r.rid]
            assert np.array_equal(srv.result(c.rid), want.states[r.rid]), r
        s = srv.summary()
        assert s["requests"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0.0
