// Drop-in CUDA backend for the reference project's accelerator seam.
//
// Compiled against the reference's unchanged header include/mhd/gpu/device_solver.hpp, this file
// defines the two symbols that header declares for a CUDA backend, mhd::cuda_available() and
// mhd::make_cuda_solver() (device_solver.hpp:78-82), and implements mhd::DeviceSolver
// (device_solver.hpp:57-75) on top of the C ABI in include/mhd_b200.h. Built with
// -DMHD_HAS_CUDA=1 (so the header's stubs are not compiled) and linked with libmhd_b200.so, it
// makes MHDSolver::set_backend("cuda", ...), the pybind module mhd_solver and the
// mhd_backend_compare gate of the reference run the B200 kernels.
//
// Errors map back to the reference's exception types and messages: MHDB_INVALID_ARGUMENT and
// MHDB_BAD_TIMESTEP -> std::invalid_argument, everything else -> std::runtime_error.

#include "mhd/gpu/device_solver.hpp"

#include "mhd_b200.h"

#include <memory>
#include <stdexcept>
#include <string>

namespace {

void raise_for(int rc, const mhdb_solver* h)
{
    if (rc == MHDB_OK) {
        return;
    }
    const std::string msg = mhdb_last_error(h);
    if (rc == MHDB_INVALID_ARGUMENT || rc == MHDB_BAD_TIMESTEP) {
        throw std::invalid_argument(msg);
    }
    throw std::runtime_error(msg);
}

class B200DeviceSolver final : public mhd::DeviceSolver {
  public:
    B200DeviceSolver(const Grid2D& grid, mhd::Precision precision) : grid_(grid)
    {
        const mhdb_grid g{grid.nx, grid.ny, grid.ng, grid.x_min, grid.x_max, grid.y_min, grid.y_max};
        const int prec = precision == mhd::Precision::FP32 ? MHDB_FP32 : MHDB_FP64;
        raise_for(mhdb_create(&g, prec, &h_), nullptr);
    }

    ~B200DeviceSolver() override
    {
        mhdb_destroy(h_);
    }

    B200DeviceSolver(const B200DeviceSolver&) = delete;
    B200DeviceSolver& operator=(const B200DeviceSolver&) = delete;

    std::string device_name() const override
    {
        char buf[256];
        raise_for(mhdb_device_name(h_, buf, sizeof buf), h_);
        return buf;
    }

    mhd::Precision precision() const override
    {
        return mhdb_precision(h_) == MHDB_FP32 ? mhd::Precision::FP32 : mhd::Precision::FP64;
    }

    void configure(const BoundaryConditions& bc, const FluidMask* mask,
                   bool reflective_walls) override
    {
        const std::uint8_t* m = nullptr;
        std::size_t len = 0;
        if (mask != nullptr && !mask->empty() && !mask->all_fluid()) {
            if (mask->nx != grid_.nx || mask->ny != grid_.ny) {
                throw std::invalid_argument("FluidMask size does not match Grid2D interior");
            }
            m = mask->fluid.data();
            len = mask->fluid.size();
        }
        raise_for(mhdb_configure(h_, static_cast<int>(bc.type_x), static_cast<int>(bc.type_y), m,
                                 len, reflective_walls ? 1 : 0),
                  h_);
    }

    void upload(const StateField& U) override
    {
        check_shape(U);
        const double* const c[9] = {U.rho.data(), U.mx.data(), U.my.data(),
                                    U.mz.data(),  U.energy.data(), U.bx.data(),
                                    U.by.data(),  U.bz.data(), U.psi.data()};
        raise_for(mhdb_upload(h_, c, U.rho.size()), h_);
    }

    void download(StateField& U) override
    {
        check_shape(U);
        double* const c[9] = {U.rho.data(), U.mx.data(), U.my.data(), U.mz.data(), U.energy.data(),
                              U.bx.data(),  U.by.data(), U.bz.data(), U.psi.data()};
        raise_for(mhdb_download(h_, c, U.rho.size()), h_);
    }

    SolveResult solve(const SolveParams& p) override
    {
        const mhdb_params cp{p.t_end,
                             p.cfl,
                             p.gamma,
                             p.glm_alpha,
                             p.limiter == SlopeLimiter::Minmod ? MHDB_MINMOD : MHDB_MC,
                             p.nonideal.ohmic ? 1 : 0,
                             p.nonideal.hall ? 1 : 0,
                             p.nonideal.ambipolar ? 1 : 0,
                             p.nonideal.eta_ohm,
                             p.nonideal.eta_hall,
                             p.nonideal.eta_ambipolar,
                             p.max_steps};
        mhdb_result r{};
        raise_for(mhdb_solve(h_, &cp, &r), h_);
        SolveResult out{};
        out.t = r.t;
        out.steps = r.steps;
        out.c_h = r.c_h;
        return out;
    }

  private:
    void check_shape(const StateField& U) const
    {
        if (U.nx != grid_.get_size_x() || U.ny != grid_.get_size_y()) {
            throw std::invalid_argument("StateField size does not match Grid2D");
        }
    }

    Grid2D grid_;
    mhdb_solver* h_ = nullptr;
};

} // namespace

bool mhd::cuda_available()
{
    return mhdb_cuda_available() != 0;
}

std::unique_ptr<mhd::DeviceSolver> mhd::make_cuda_solver(const Grid2D& grid, Precision precision)
{
    if (grid.ng < 2) {
        throw std::invalid_argument("CUDA solver requires grid.ng >= 2");
    }
    if (!cuda_available()) {
        throw std::runtime_error("CUDA: no device available");
    }
    return std::make_unique<B200DeviceSolver>(grid, precision);
}
