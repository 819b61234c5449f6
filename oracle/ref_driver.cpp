// Thin C-ABI driver around the reference CPU solver — TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/build_ref.py from the reference's own, unmodified headers where they lie
// (include path given on the command line) into oracle/_ref/libmhd_ref_<isa>.so. Nothing from
// the reference is copied into this repository. The library runs the reference's SIMD +
// thread-pool CPU path: solve() (include/mhd/time_integrator.hpp:62-106) for time-based runs,
// and the body of its step loop (time_integrator.hpp:84-104) for a fixed number of steps,
// followed by the same final ghost and wall fill. It is used to pin the C restatement in
// oracle/mhd_oracle.c and as the timed CPU baseline.
//
// Structs are the same as oracle/mhd_oracle.h so one ctypes binding serves both.

#include "mhd_oracle.h"

#include "boundary_conditions/boundary_conditions.hpp"
#include "grid/grid.hpp"
#include "mhd/cfl.hpp"
#include "mhd/mask.hpp"
#include "mhd/parallel.hpp"
#include "mhd/rhs.hpp"
#include "mhd/simd.hpp"
#include "mhd/solve_types.hpp"
#include "mhd/time_integrator.hpp"
#include "state/state_field.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <limits>
#include <stdexcept>

namespace {

BoundaryConditionType bc_of(int k)
{
    switch (k) {
    case MHDO_PERIODIC:
        return BoundaryConditionType::Periodic;
    case MHDO_OUTFLOW:
        return BoundaryConditionType::Outflow;
    default:
        return BoundaryConditionType::Reflective;
    }
}

bool to_params(const mhdo_params* p, SolveParams& sp)
{
    if (p->limiter == MHDO_MINMOD) {
        sp.limiter = SlopeLimiter::Minmod;
    } else if (p->limiter == MHDO_MC) {
        sp.limiter = SlopeLimiter::MC;
    } else {
        return false; // the reference has no van Leer limiter
    }
    sp.t_end = p->t_end;
    sp.cfl = p->cfl;
    sp.gamma = p->gamma;
    sp.glm_alpha = p->glm_alpha;
    sp.max_steps = p->max_steps;
    NonIdealConfig ni{};
    ni.ohmic = p->ohmic != 0;
    ni.hall = p->hall != 0;
    ni.ambipolar = p->ambipolar != 0;
    ni.eta_ohm = p->eta_ohm;
    ni.eta_hall = p->eta_hall;
    ni.eta_ambipolar = p->eta_ambipolar;
    sp.nonideal = ni;
    return true;
}

void load_state(StateField& S, const double* U)
{
    const std::size_t n = S.rho.size();
    std::vector<double>* c[9] = {&S.rho, &S.mx, &S.my, &S.mz, &S.energy,
                                 &S.bx,  &S.by, &S.bz, &S.psi};
    for (int k = 0; k < 9; ++k) {
        std::memcpy(c[k]->data(), U + k * n, n * sizeof(double));
    }
}

void store_state(const StateField& S, double* U)
{
    const std::size_t n = S.rho.size();
    const std::vector<double>* c[9] = {&S.rho, &S.mx, &S.my, &S.mz, &S.energy,
                                       &S.bx,  &S.by, &S.bz, &S.psi};
    for (int k = 0; k < 9; ++k) {
        std::memcpy(U + k * n, c[k]->data(), n * sizeof(double));
    }
}

// Wall-clock seconds of the step loop of the last mhdr_solve (state copies and workspace
// allocation excluded), as tools/mhd_backend_compare.cpp times run().
double g_loop_seconds = 0.0;

} // namespace

extern "C" {

double mhdr_last_loop_seconds()
{
    return g_loop_seconds;
}

int mhdr_set_threads(int n)
{
    mhd::set_num_threads(n);
    return mhd::num_threads();
}

const char* mhdr_simd_backend()
{
    return mhd::simd::kBackendName;
}

int mhdr_solve(const mhdo_grid* g, const mhdo_params* p, int bc_x, int bc_y, const uint8_t* mask,
               int reflective_walls, double* U, mhdo_result* out)
{
    try {
        SolveParams sp;
        if (!to_params(p, sp)) {
            return MHDO_EINVAL;
        }
        Grid2D grid(g->nx, g->ny, g->x_min, g->x_max, g->y_min, g->y_max, g->ng);
        BoundaryConditions bc(bc_of(bc_x), bc_of(bc_y));
        StateField S(grid.get_size_x(), grid.get_size_y());
        load_state(S, U);
        TimeIntegratorWorkspace work(grid);
        FluidMask fm(g->nx, g->ny, true);
        const FluidMask* mptr = nullptr;
        if (mask != nullptr) {
            fm.set_from_interior(mask, static_cast<std::size_t>(g->nx) * g->ny, g->nx, g->ny);
            mptr = &fm;
        }
        SolveResult r{};
        const auto t0 = std::chrono::steady_clock::now();
        if (p->fixed_steps == 0) {
            r = solve(S, work, grid, bc, sp, mptr, reflective_walls != 0);
        } else {
            // Body of the solve() loop, exactly N steps (time_integrator.hpp:84-104).
            const FluidMask* active = (mptr != nullptr && !fm.empty() && !fm.all_fluid()) ? mptr
                                                                                          : nullptr;
            for (int s = 0; s < p->max_steps; ++s) {
                const CFLResult cfl =
                    compute_cfl_dt(S, grid, sp.gamma, sp.cfl, sp.nonideal, active);
                r.c_h = cfl.c_h;
                const double dt = cfl.dt;
                ssp_rk2_step(S, work, grid, bc, sp.gamma, dt, cfl.c_h, sp.glm_alpha, sp.limiter,
                             sp.nonideal, active, reflective_walls != 0);
                r.t += dt;
                ++r.steps;
            }
            apply_boundary_conditions(S, grid, bc);
            if (active != nullptr && reflective_walls != 0) {
                apply_solid_wall_fill(S, grid, *active, sp.gamma);
            }
        }
        g_loop_seconds =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        store_state(S, U);
        out->t = r.t;
        out->steps = r.steps;
        out->c_h = r.c_h;
        return MHDO_OK;
    } catch (const std::runtime_error&) {
        return MHDO_EMAXSTEPS;
    } catch (const std::exception&) {
        return MHDO_EINVAL;
    }
}

int mhdr_rhs(const mhdo_grid* g, const mhdo_params* p, const uint8_t* mask, double c_h,
             const double* U, double* rhs)
{
    try {
        SolveParams sp;
        if (!to_params(p, sp)) {
            return MHDO_EINVAL;
        }
        Grid2D grid(g->nx, g->ny, g->x_min, g->x_max, g->y_min, g->y_max, g->ng);
        StateField S(grid.get_size_x(), grid.get_size_y());
        StateField R(grid.get_size_x(), grid.get_size_y());
        load_state(S, U);
        load_state(R, rhs);
        RHSWorkspace work(grid.get_size_x(), grid.get_size_y());
        FluidMask fm(g->nx, g->ny, true);
        const FluidMask* mptr = nullptr;
        if (mask != nullptr) {
            fm.set_from_interior(mask, static_cast<std::size_t>(g->nx) * g->ny, g->nx, g->ny);
            if (!fm.all_fluid()) {
                mptr = &fm;
            }
        }
        compute_rhs(S, R, grid, work, sp.gamma, c_h, sp.glm_alpha, sp.limiter, sp.nonideal, mptr);
        store_state(R, rhs);
        return MHDO_OK;
    } catch (const std::exception&) {
        return MHDO_EINVAL;
    }
}

} // extern "C"
