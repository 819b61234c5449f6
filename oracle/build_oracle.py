"""Build recipe for the CPU oracle — test infrastructure only.

* ``oracle/libmhd_oracle.so``: the C restatement (``mhd_oracle.c``), built with gcc for
  baseline x86-64 (no FMA contraction is possible there, so every operation rounds once,
  in program order) and OpenMP (its loops over cells and rows run on all host threads; the
  results do not depend on the thread count).
* ``oracle/_ref/libmhd_ref_<isa>.so``: the reference CPU solver compiled from its own
  headers where they lie (``$MHD_REFERENCE_ROOT/include``), wrapped by ``ref_driver.cpp``, with
  the reference's release flags (``-O3 -ffp-contract=fast -fno-math-errno
  -fno-trapping-math``; cmake/MHDCompilerFlags.cmake:29-35) for two ISA levels
  (x86-64-v4 = AVX-512F, x86-64-v3 = AVX2+FMA). Built only where the reference checkout
  exists; the built files travel with the repository to machines that lack it.
* ``oracle/_ref/cuda_bench_reference`` and ``oracle/_ref/cuda_bench_b200``: the timing driver
  ``cuda_backend_bench.cpp`` over the reference's DeviceSolver interface, linked with the
  reference's own CUDA backend (``src/cuda/cuda_solver.cu`` compiled by nvcc for sm_100a with the
  reference's flags: C++20, -O3; CMakeLists.txt:87-101) and with the B200 adapter: a same-box
  baseline of the reference's GPU path.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def reference_root() -> str | None:
    """The reference checkout named by MHD_REFERENCE_ROOT (unset: no reference build)."""
    return os.environ.get("MHD_REFERENCE_ROOT") or None

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
        _run(["gcc", "-std=c99", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              "-march=x86-64", "-Wall", "-Wextra", src, "-o", ORACLE_SO, "-lm"])
    return ORACLE_SO


def reference_available() -> bool:
    root = reference_root()
    return root is not None and os.path.isdir(os.path.join(root, "include", "mhd"))


def build_ref(force: bool = False) -> list[str]:
    """Compile the reference CPU path into oracle/_ref (no-op without the checkout)."""
    if not reference_available():
        return []
    os.makedirs(REF_DIR, exist_ok=True)
    src = os.path.join(HERE, "ref_driver.cpp")
    hdr = os.path.join(HERE, "mhd_oracle.h")
    inc = os.path.join(reference_root(), "include")
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


PKG_DIR = os.path.join(os.path.dirname(HERE), "mhd_gpu_solver_b200")
ADAPTER = os.path.join(PKG_DIR, "csrc", "reference_backend.cpp")
REPO_INCLUDE = os.path.join(os.path.dirname(HERE), "include")


def _build_info_header() -> str:
    """Stand-in for the CMake-generated include/mhd/build_info.hpp of the reference (its
    template include/mhd/build_info.hpp.in only defines build-provenance strings)."""
    gen = os.path.join(REF_DIR, "generated", "mhd")
    os.makedirs(gen, exist_ok=True)
    path = os.path.join(gen, "build_info.hpp")
    vals = {"COMPILER_ID": "GNU", "COMPILER_VERSION": "g++", "CXX_STANDARD": "20",
            "CMAKE_VERSION": "none", "TYPE": "Release", "GIT_COMMIT": "unknown",
            "SYSTEM_NAME": "Linux", "SYSTEM_PROCESSOR": "x86_64", "NATIVE_ARCH": "OFF",
            "SANITIZERS": "OFF"}
    text = "#pragma once\n" + "".join(f'#define MHD_BUILD_{k} "{v}"\n' for k, v in vals.items())
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)
    return os.path.dirname(gen)


def build_ref_with_b200(force: bool = False) -> list[str]:
    """The reference's own Python module (python/mhd_pybind.cpp) and GPU gate tool
    (tools/mhd_backend_compare.cpp), compiled from their sources with -DMHD_HAS_CUDA=1 and the
    B200 backend (mhd_gpu_solver_b200/csrc/reference_backend.cpp + libmhd_b200.so) as their
    CUDA backend. No-op without the reference checkout or the CUDA library."""
    lib = os.path.join(PKG_DIR, "libmhd_b200.so")
    if not reference_available() or not os.path.exists(lib):
        return []
    import sysconfig

    import pybind11

    os.makedirs(REF_DIR, exist_ok=True)
    inc = os.path.join(reference_root(), "include")
    gen = _build_info_header()
    common = ["g++", "-std=c++20", "-O3", "-DNDEBUG", "-fno-math-errno", "-fno-trapping-math",
              "-ffp-contract=fast", "-march=x86-64-v3", "-pthread", "-DMHD_HAS_CUDA=1",
              "-I", inc, "-I", gen, "-I", REPO_INCLUDE]
    link = ["-L", PKG_DIR, "-l:libmhd_b200.so", "-Wl,-rpath,$ORIGIN/../../mhd_gpu_solver_b200"]
    outs = []
    mod = os.path.join(REF_DIR, "mhd_solver" + sysconfig.get_config_var("EXT_SUFFIX"))
    src_mod = os.path.join(reference_root(), "python", "mhd_pybind.cpp")
    if force or _stale(mod, [src_mod, ADAPTER, lib]):
        _run(common + ["-fPIC", "-shared", "-I", pybind11.get_include(),
                       "-I", sysconfig.get_paths()["include"], src_mod, ADAPTER, "-o", mod] + link)
    outs.append(mod)
    gate = os.path.join(REF_DIR, "mhd_backend_compare")
    src_gate = os.path.join(reference_root(), "tools", "mhd_backend_compare.cpp")
    if force or _stale(gate, [src_gate, ADAPTER, lib]):
        _run(common + [src_gate, ADAPTER, "-o", gate] + link)
    outs.append(gate)
    return outs


def build_cuda_bench(force: bool = False) -> list[str]:
    """The DeviceSolver timing driver against both CUDA backends (no-op without the reference
    checkout, nvcc or the B200 library)."""
    lib = os.path.join(PKG_DIR, "libmhd_b200.so")
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    if not reference_available() or not os.path.exists(lib) or not os.path.exists(nvcc):
        return []
    os.makedirs(REF_DIR, exist_ok=True)
    inc = os.path.join(reference_root(), "include")
    drv = os.path.join(HERE, "cuda_backend_bench.cpp")
    host = ["g++", "-std=c++20", "-O3", "-DNDEBUG", "-fno-math-errno", "-fno-trapping-math",
            "-ffp-contract=fast", "-march=x86-64-v3", "-pthread", "-DMHD_HAS_CUDA=1", "-I", inc]
    outs = []
    src_cu = os.path.join(reference_root(), "src", "cuda", "cuda_solver.cu")
    obj = os.path.join(REF_DIR, "reference_cuda_solver.o")
    ref_bin = os.path.join(REF_DIR, "cuda_bench_reference")
    if force or _stale(ref_bin, [src_cu, drv]):
        _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++20", "-O3",
              "-DMHD_HAS_CUDA=1", "-I", inc, "-c", src_cu, "-o", obj])
        _run(host + [drv, obj, "-L/usr/local/cuda/lib64", "-lcudart", "-o", ref_bin])
    outs.append(ref_bin)
    b200_bin = os.path.join(REF_DIR, "cuda_bench_b200")
    if force or _stale(b200_bin, [drv, ADAPTER, lib]):
        _run(host + ["-I", REPO_INCLUDE, drv, ADAPTER, "-o", b200_bin, "-L", PKG_DIR,
                     "-l:libmhd_b200.so", "-Wl,-rpath,$ORIGIN/../../mhd_gpu_solver_b200"])
    outs.append(b200_bin)
    return outs


if __name__ == "__main__":
    if not reference_available():
        sys.stderr.write("MHD_REFERENCE_ROOT does not name a reference checkout: building the C "
                         "oracle only\n")
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
    print(build_ref_with_b200(force="--force" in sys.argv))
    print(build_cuda_bench(force="--force" in sys.argv))
