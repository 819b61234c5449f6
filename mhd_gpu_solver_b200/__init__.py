"""B200-native (sm_100a) backend for the 2D GLM-MHD finite-volume operator.

* ``mhd_gpu_solver_b200.mhd_solver``: the reference's ``mhd_solver`` Python surface
  (MHDSolver, SolveParams, NonIdealConfig, ...) running on the CUDA backend.
* ``mhd_gpu_solver_b200._capi``: ctypes binding of the C ABI (include/mhd_b200.h).
* ``mhd_gpu_solver_b200.workloads``: seeded synthetic initial states and masks (numpy).
* ``mhd_gpu_solver_b200.accuracy``: the per-component L1 error rule (numpy).
* ``mhd_gpu_solver_b200.batch`` / ``serve``: many solves in one persistent step, and the
  continuous-batching request loop over it; ``autotune``: per-size-class configuration choice.
* ``mhd_gpu_solver_b200.strips``: one grid split into y strips over several GPUs or solvers.

Every module that runs the operator imports ``_capi``, which loads ``libmhd_b200.so``; there is
no CPU fallback, so that import fails with ImportError when the library has not been built. The
numpy-only modules (workloads, accuracy) load no library.
"""

__all__ = ["_capi", "accuracy", "autotune", "batch", "mhd_solver", "serve", "strips",
           "workloads"]
