// Timing driver for a CUDA backend of the reference's DeviceSolver interface: same-box
// comparison infrastructure only (it measures; nothing in the product calls it).
//
// oracle/build_oracle.py compiles it from the reference's own, unmodified headers where they lie
// twice: linked with the reference's own CUDA backend (src/cuda/cuda_solver.cu, nvcc for
// sm_100a) into oracle/_ref/cuda_bench_reference, and with the B200 adapter
// (mhd_gpu_solver_b200/csrc/reference_backend.cpp + libmhd_b200.so) into
// oracle/_ref/cuda_bench_b200. Both binaries time the same calls of the reference interface
// (include/mhd/gpu/device_solver.hpp:57-75) on the Orszag-Tang state of the reference's speed
// comparison (tools/mhd_backend_compare.cpp:215-223: CFL 0.4, GLM alpha 0.1, MC limiter,
// periodic, ideal):
//   * "resident": DeviceSolver::solve(params) on a state uploaded beforehand,
//   * "run": configure + upload + solve + download per call, as MHDSolver::run drives a device
//     (include/mhd/solver_api.hpp:294-311),
// each after one warm-up call, with std::chrono::steady_clock around the call (solve returns
// after the device has finished). Output: one JSON object per line.
//
// usage: cuda_bench_<backend> <n> <fp64|fp32> <t_end> [reps]

#include "mhd/solver_api.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>

namespace {

double seconds_of(const std::chrono::steady_clock::time_point& a,
                  const std::chrono::steady_clock::time_point& b)
{
    return std::chrono::duration<double>(b - a).count();
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <n> <fp64|fp32> <t_end> [reps]\n", argv[0]);
        return 2;
    }
    const int n = std::atoi(argv[1]);
    const std::string prec_name = argv[2];
    const double t_end = std::atof(argv[3]);
    const int reps = argc > 4 ? std::atoi(argv[4]) : 3;
    const mhd::Precision prec = prec_name == "fp32" ? mhd::Precision::FP32 : mhd::Precision::FP64;
    try {
        MHDSolver s(n, n, 0.0, 1.0, 0.0, 1.0);
        s.set_cfl(0.4);
        s.set_glm_alpha(0.1);
        s.set_limiter_mc();
        s.set_periodic_bc();
        s.set_ideal();
        s.initialize("orszag_tang");
        const StateField U0 = s.state();
        const BoundaryConditions bc(BoundaryConditionType::Periodic,
                                    BoundaryConditionType::Periodic);
        SolveParams p = s.params();
        p.t_end = t_end;

        auto dev = mhd::make_cuda_solver(s.grid(), prec);
        dev->configure(bc, nullptr, true);
        dev->upload(U0);
        dev->solve(p); // warm-up: context, module load, first touch, graphs
        for (int r = 0; r < reps; ++r) {
            dev->upload(U0);
            const auto t0 = std::chrono::steady_clock::now();
            const SolveResult res = dev->solve(p);
            const auto t1 = std::chrono::steady_clock::now();
            const double sec = seconds_of(t0, t1);
            std::printf("{\"mode\": \"resident\", \"device\": \"%s\", \"n\": %d, \"precision\": "
                        "\"%s\", \"t_end\": %g, \"steps\": %d, \"seconds\": %.6f, "
                        "\"zone_updates_per_s\": %.6e}\n",
                        dev->device_name().c_str(), n, prec_name.c_str(), t_end, res.steps, sec,
                        static_cast<double>(n) * n * res.steps / sec);
        }
        StateField U = U0;
        for (int r = 0; r < reps; ++r) {
            U = U0;
            const auto t0 = std::chrono::steady_clock::now();
            dev->configure(bc, nullptr, true);
            dev->upload(U);
            const SolveResult res = dev->solve(p);
            dev->download(U);
            const auto t1 = std::chrono::steady_clock::now();
            const double sec = seconds_of(t0, t1);
            std::printf("{\"mode\": \"run\", \"device\": \"%s\", \"n\": %d, \"precision\": "
                        "\"%s\", \"t_end\": %g, \"steps\": %d, \"seconds\": %.6f, "
                        "\"zone_updates_per_s\": %.6e}\n",
                        dev->device_name().c_str(), n, prec_name.c_str(), t_end, res.steps, sec,
                        static_cast<double>(n) * n * res.steps / sec);
        }
        std::fflush(stdout);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
