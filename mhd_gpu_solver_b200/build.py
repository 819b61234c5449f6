"""Build recipe of the CUDA backend: ``csrc/*.cu`` -> ``libmhd_b200.so`` (sm_100a only).

The library is built in-tree next to this file so that it travels with the repository; the
CUDA runtime is linked statically, so the library needs only the driver at run time.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libmhd_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2",
              "--expt-relaxed-constexpr"]


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


OBJ_DIR = os.path.join(PKG, "_build")
# The FP32-mixed kernels use the hardware's approximate FP32 division and square root; the FP32
# arithmetic of that form carries no more accuracy than these give, and FP64 code is unaffected.
UNIT_FLAGS = {"kernels_mixed.cu": ["-prec-div=false", "-prec-sqrt=false"]}


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every csrc/*.cu to an object in parallel, then link the shared library."""
    deps = _sources()
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    units = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    procs = []
    for u in units:
        obj = os.path.join(OBJ_DIR, os.path.basename(u) + ".o")
        cmd = [NVCC, *ARCH_FLAGS, *NVCC_FLAGS, *UNIT_FLAGS.get(os.path.basename(u), []), "-c",
               "-I", INCLUDE, u, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((cmd, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                 stderr=subprocess.PIPE, text=True)))
    objs = []
    for cmd, obj, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out + err)
        if verbose:
            sys.stderr.write(err)
        objs.append(obj)
    link = [NVCC, *ARCH_FLAGS, "-shared", *objs, "-o", LIB + ".tmp"]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + " ".join(link) + "\n" + res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
