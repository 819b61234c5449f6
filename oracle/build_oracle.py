"""Build recipe for the CPU oracle — test infrastructure only.

* ``oracle/libmhd_oracle.so``: the C restatement (``mhd_oracle.c``), built with gcc for
  baseline x86-64 (no FMA contraction is possible there, so every operation rounds once,
  in program order).
* ``oracle/_ref/libmhd_ref_<isa>.so``: the reference CPU solver compiled from its own
  headers where they lie (``REFERENCE_ROOT/include``), wrapped by ``ref_driver.cpp``, with
  the reference's release flags (``-O3 -ffp-contract=fast -fno-math-errno
  -fno-trapping-math``; cmake/MHDCompilerFlags.cmake:29-35) for two ISA levels
  (x86-64-v4 = AVX-512F, x86-64-v3 = AVX2+FMA). Built only where the reference checkout
  exists; the built files travel with the repository to machines that lack it.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REFERENCE_ROOT = os.environ.get("MHD_REFERENCE_ROOT", "/root/reference")

ORACLE_SO = os.path.join(HERE, "libmhd_oracle.so")
REF_ISAS = {"avx512": "x86-64-v4", "avx2": "x86-64-v3"}


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "mhd_oracle.c")
    hdr = os.path.join(HERE, "mhd_oracle.h")
    if force or _stale(ORACLE_SO, [src, hdr]):
        _run(["gcc", "-std=c99", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
              "-march=x86-64", "-Wall", "-Wextra", src, "-o", ORACLE_SO, "-lm"])
    return ORACLE_SO


def reference_available() -> bool:
    return os.path.isdir(os.path.join(REFERENCE_ROOT, "include", "mhd"))


def build_ref(force: bool = False) -> list[str]:
    """Compile the reference CPU path into oracle/_ref (no-op without the checkout)."""
    if not reference_available():
        return []
    os.makedirs(REF_DIR, exist_ok=True)
    src = os.path.join(HERE, "ref_driver.cpp")
    hdr = os.path.join(HERE, "mhd_oracle.h")
    inc = os.path.join(REFERENCE_ROOT, "include")
    ref_headers = []
    for root, _dirs, files in os.walk(inc):
        ref_headers += [os.path.join(root, f) for f in files if f.endswith(".hpp")]
    out = []
    for isa, march in REF_ISAS.items():
        so = os.path.join(REF_DIR, f"libmhd_ref_{isa}.so")
        if force or _stale(so, [src, hdr] + ref_headers):
            _run(["g++", "-std=c++20", "-O3", "-DNDEBUG", "-fno-math-errno", "-fno-trapping-math",
                  "-ffp-contract=fast", f"-march={march}", "-fPIC", "-shared", "-pthread",
                  "-I", inc, "-I", HERE, src, "-o", so])
        out.append(so)
    return out


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
