// FP64 diagnostics of the device state, reduced on the device in a fixed order.
//
// Quantities follow the reference's host-side diagnostics run on the state that solve() leaves
// (ghosts by the boundary rule, solid cells wall-filled): mass = sum(rho dx dy) and energy =
// sum(E dx dy) over interior cells (include/verification/diagnostics.hpp:41-52), min rho and
// min p with to_primitive's division form, finiteness of rho, p, E and B, and the central-
// difference divergence of B (include/initial_condition/inititial_condition.hpp:273-287) as its
// maximum and its root-mean-square over interior cells.
#pragma once

#include "runtime_types.cuh"
#include "stage_f64.cuh"
#include "stage_mixed.cuh"

namespace mhdb {

constexpr int kDiagThreads = 256;
constexpr int kDiagBlocks = 592; // 4 x 148 SMs
constexpr int kDiagFields = 7;   // mass, energy, div2, divmax, rhomin, pmin, nonfinite

struct DiagLoaderF64 {
    const double* u;
    __device__ void cell(const Geometry& g, const uint8_t* mask, int fill, double gm1, int x,
                         int y, double* out) const
    {
        if (fill && is_solid(mask, g, x, y)) {
            wall_fill_f64(u, mask, g, x, y, gm1, out);
        } else {
            load_cons_f64(u, g, x, y, out);
        }
    }
};

struct DiagLoaderMx {
    MixedState u;
    __device__ void cell(const Geometry& g, const uint8_t* mask, int fill, double gm1, int x,
                         int y, double* out) const
    {
        if (fill && is_solid(mask, g, x, y)) {
            wall_fill_mx(u, mask, g, x, y, gm1, out);
        } else {
            load_cons_mx(u, g, x, y, out);
        }
    }
};

template <class Loader>
__device__ __forceinline__ double b_component(const Loader& ld, const Geometry& g,
                                              const uint8_t* mask, int fill, double gm1, int x,
                                              int y, int comp)
{
    // Ghost neighbours hold the stored (pre-fill) value of the cell the boundary rule maps to.
    const bool interior = x >= 0 && x < g.nx && y >= 0 && y < g.ny;
    const int sx = map_index(x, g.nx, g.bc_x), sy = map_index(y, g.ny, g.bc_y);
    double v[9];
    ld.cell(g, mask, interior ? fill : 0, gm1, sx, sy, v);
    return v[comp];
}

template <class Loader>
__global__ void __launch_bounds__(kDiagThreads) diag_partial(Loader ld, const uint8_t* mask,
                                                            int fill, Geometry g, double gm1,
                                                            double inv_2dx, double inv_2dy,
                                                            double* partial)
{
    double acc[kDiagFields] = {0.0, 0.0, 0.0, 0.0, INFINITY, INFINITY, 0.0};
    const long long n = static_cast<long long>(g.nx) * (g.ry1 - g.ry0);
    for (long long c = blockIdx.x * static_cast<long long>(kDiagThreads) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * kDiagThreads) {
        const int x = static_cast<int>(c % g.nx), y = g.ry0 + static_cast<int>(c / g.nx);
        double u[9];
        ld.cell(g, mask, fill, gm1, x, y, u);
        const double rho = u[0], E = u[4];
        const double e_kin = 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / rho;
        const double e_mag = 0.5 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
        const double p = gm1 * (E - e_kin - e_mag);
        acc[0] += rho;
        acc[1] += E;
        const double dbx = (b_component(ld, g, mask, fill, gm1, x + 1, y, 5) -
                            b_component(ld, g, mask, fill, gm1, x - 1, y, 5)) * inv_2dx;
        const double dby = (b_component(ld, g, mask, fill, gm1, x, y + 1, 6) -
                            b_component(ld, g, mask, fill, gm1, x, y - 1, 6)) * inv_2dy;
        const double dv = dbx + dby;
        acc[2] += dv * dv;
        acc[3] = vmax(acc[3], fabs(dv));
        acc[4] = vmin(acc[4], rho);
        acc[5] = vmin(acc[5], p);
        if (!isfinite(rho) || !isfinite(p) || !isfinite(E) || !isfinite(u[5]) ||
            !isfinite(u[6]) || !isfinite(u[7])) {
            acc[6] = 1.0;
        }
    }
    __shared__ double sh[kDiagFields][kDiagThreads];
#pragma unroll
    for (int f = 0; f < kDiagFields; ++f) {
        sh[f][threadIdx.x] = acc[f];
    }
    __syncthreads();
    for (int s = kDiagThreads / 2; s > 0; s >>= 1) {
        if (static_cast<int>(threadIdx.x) < s) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
            sh[2][threadIdx.x] += sh[2][threadIdx.x + s];
            sh[3][threadIdx.x] = vmax(sh[3][threadIdx.x], sh[3][threadIdx.x + s]);
            sh[4][threadIdx.x] = vmin(sh[4][threadIdx.x], sh[4][threadIdx.x + s]);
            sh[5][threadIdx.x] = vmin(sh[5][threadIdx.x], sh[5][threadIdx.x + s]);
            sh[6][threadIdx.x] = vmax(sh[6][threadIdx.x], sh[6][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x < kDiagFields) {
        partial[threadIdx.x * gridDim.x + blockIdx.x] = sh[threadIdx.x][0];
    }
}

// One thread sums the block partials in block order (deterministic, nblocks <= kDiagBlocks).
__global__ void diag_final(const double* partial, int nblocks, double cell, long long ncell,
                           double* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) {
        return;
    }
    double m = 0.0, e = 0.0, d2 = 0.0, dmax = 0.0, rmin = INFINITY, pmin = INFINITY, nf = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        m += partial[0 * nblocks + b];
        e += partial[1 * nblocks + b];
        d2 += partial[2 * nblocks + b];
        dmax = vmax(dmax, partial[3 * nblocks + b]);
        rmin = vmin(rmin, partial[4 * nblocks + b]);
        pmin = vmin(pmin, partial[5 * nblocks + b]);
        nf = vmax(nf, partial[6 * nblocks + b]);
    }
    out[0] = m * cell;
    out[1] = e * cell;
    out[2] = dmax;
    out[3] = sqrt(d2 / static_cast<double>(ncell));
    out[4] = rmin;
    out[5] = pmin;
    out[6] = nf;
}

} // namespace mhdb
