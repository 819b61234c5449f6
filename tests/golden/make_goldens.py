"""Regenerate the golden fixtures in tests/golden/ (run where the reference checkout exists).

1. ``orszag_tang_32.npz`` and ``ohmic_sine_bz_32.npz``: the reference's own regression goldens
   (tests/goldens/*.golden, text format of tests/golden_io.hpp in the reference project),
   converted to numpy: interior fields of the final state and the step count. They pin the
   Orszag-Tang 32^2 MC run to t = 0.05 (36 steps) and the Ohmic decay of Bz = sin(2 pi x) with
   minmod, CFL 0.3, eta = 0.1 to t = 0.1 (137 steps).
2. ``quadrant128_seed<k>.npz`` (k = 0..4): output of the reference CPU solver itself (compiled
   from its headers into oracle/_ref) on the 128^2 four-quadrant outflow case, minmod, 200
   steps: per-component interior sum, absolute sum, min and max, a strided sample of every 37th
   interior cell, and t, steps, c_h.

Usage: python tests/golden/make_goldens.py
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mhd_gpu_solver_b200 import workloads as wl  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from oracle.build_oracle import REFERENCE_ROOT, build_oracle, build_ref  # noqa: E402

SAMPLE_STRIDE = 37


def read_reference_golden(path: str) -> tuple[dict, dict]:
    meta, fields = {}, {}
    with open(path) as f:
        tokens = f.read().split()
    if tokens[:2] != ["MHD_GOLDEN", "1"]:
        raise ValueError(f"bad golden header in {path}")
    i = 2
    while i < len(tokens):
        key = tokens[i]
        if key == "field":
            name, n = tokens[i + 1], int(tokens[i + 2])
            fields[name] = np.array([float(v) for v in tokens[i + 3:i + 3 + n]])
            i += 3 + n
        else:
            meta[key] = tokens[i + 1]
            i += 2
    return meta, fields


def convert_reference_goldens() -> None:
    src = os.path.join(REFERENCE_ROOT, "tests", "goldens")
    for name in ("orszag_tang_32", "ohmic_sine_bz_32"):
        meta, fields = read_reference_golden(os.path.join(src, name + ".golden"))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), meta=json.dumps(meta),
                            **{k: v.reshape(32, 32) for k, v in fields.items()})
        print("wrote", name, meta.get("steps"))


def quadrant_case(seed: int):
    n = 128
    prim = wl.four_quadrant(n, n, seed)
    gamma = 5.0 / 3.0
    bc = (orc.OUTFLOW, orc.OUTFLOW)
    U0 = wl.embed(wl.to_conservative(prim, gamma))
    U0 = orc.apply_bc(U0, orc.Grid(n, n), bc)
    params = orc.Params(cfl=0.4, gamma=gamma, glm_alpha=0.1, limiter=orc.MINMOD, max_steps=200,
                        fixed_steps=True)
    return U0, orc.Grid(n, n), params, bc


def summarize(U: np.ndarray) -> dict:
    inner = U[:, 2:-2, 2:-2].reshape(9, -1)
    return {"sum": inner.sum(axis=1), "abs_sum": np.abs(inner).sum(axis=1),
            "min": inner.min(axis=1), "max": inner.max(axis=1),
            "sample": inner[:, ::SAMPLE_STRIDE].copy()}


def make_quadrant_fixtures() -> None:
    for seed in range(5):
        U0, grid, params, bc = quadrant_case(seed)
        out, t, steps, c_h = orc.solve(U0, grid, params, bc, impl="ref")
        s = summarize(out)
        np.savez_compressed(os.path.join(HERE, f"quadrant128_seed{seed}.npz"), t=t, steps=steps,
                            c_h=c_h, simd=orc.ref_simd_backend(), **s)
        print("wrote quadrant seed", seed, steps, t)


if __name__ == "__main__":
    build_oracle()
    if not build_ref():
        sys.exit("the reference checkout is required to regenerate the fixtures")
    convert_reference_goldens()
    make_quadrant_fixtures()
