// Plain FP64 form: state as 9 double planes, all arithmetic in FP64.
#pragma once

#include "physics.cuh"
#include "runtime_types.cuh"

namespace mhdb {

// Load the 9 conserved values of interior cell (x, y) from padded planes.
__device__ __forceinline__ void load_cons_f64(const double* __restrict__ u, const Geometry& g,
                                              int x, int y, double* out)
{
    const size_t k = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        out[c] = __ldg(u + static_cast<size_t>(c) * g.plane + k);
    }
}

__device__ __forceinline__ bool is_solid(const uint8_t* __restrict__ mask, const Geometry& g,
                                         int x, int y)
{
    return mask[static_cast<size_t>(y) * g.pitch + x] == 0;
}

// Wall fill of solid interior cell (x, y) (include/mhd/mask.hpp:100-146): first fluid interior
// neighbour in the order +x, -x, +y, -y; Load(x, y, out) reads one cell in full precision.
template <class Load>
__device__ __forceinline__ void wall_fill_any(const Load& load, const uint8_t* __restrict__ mask,
                                              const Geometry& g, int x, int y, double gm1,
                                              double* out)
{
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        const int nx = x + (k == 0 ? 1 : (k == 1 ? -1 : 0));
        const int ny = y + (k == 2 ? 1 : (k == 3 ? -1 : 0));
        if (nx < 0 || ny < 0 || nx >= g.nx || ny >= g.ny) {
            continue;
        }
        if (mask[static_cast<size_t>(ny) * g.pitch + nx] == 0) {
            continue;
        }
        double s[9];
        load(nx, ny, s);
        reflect_fill(s, k < 2 ? 0 : 1, gm1, out);
        return;
    }
    isolated_fill(gm1, out);
}

__device__ __forceinline__ void wall_fill_f64(const double* __restrict__ u,
                                              const uint8_t* __restrict__ mask, const Geometry& g,
                                              int x, int y, double gm1, double* out)
{
    wall_fill_any([&](int i, int j, double* s) { load_cons_f64(u, g, i, j, s); }, mask, g, x, y,
                  gm1, out);
}

struct StageArgsF64 {
    const double* uin;   // stage input (U^n for stage 1, U* for stage 2)
    double* out;         // U* (stage 1) or U^n updated in place (stage 2)
    const uint8_t* mask; // padded fluid mask or nullptr
    Ctrl* ctrl;
    Geometry geom;
    Consts k;
    int walls;           // reflective wall fill of solid cells
};

struct PolicyF64 {
    using T = double;
    using Args = StageArgsF64;

    static __device__ __forceinline__ void halo_prim(const double* u, const Geometry& g, int x,
                                                     int y, const Consts& k, double* w)
    {
        double c[9];
        load_cons_f64(u, g, x, y, c);
        cons_to_prim(c, k.gm1, w);
    }
    static __device__ __forceinline__ void prim_of(const double* f, const Consts& k, double* w)
    {
        cons_to_prim(f, k.gm1, w);
    }
    static __device__ __forceinline__ void wall_fill(const double* u, const uint8_t* mask,
                                                     const Geometry& g, int x, int y, double gm1,
                                                     double* out)
    {
        wall_fill_f64(u, mask, g, x, y, gm1, out);
    }
    static __device__ __forceinline__ void load_full(const double* u, const Geometry& g, int x,
                                                     int y, double* out)
    {
        load_cons_f64(u, g, x, y, out);
    }
    static __device__ __forceinline__ void store(double* u, const Geometry& g, size_t o,
                                                 const double* v)
    {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            u[static_cast<size_t>(c) * g.plane + o] = v[c];
        }
    }
    static __device__ __forceinline__ double signal_speed(const double* r, const Consts& k)
    {
        return cell_max_signal_speed(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], k.gamma);
    }
};

// Max signal speed of the current state (start of a solve): same reduction and tail as stage 2.
template <int NT>
__global__ void __launch_bounds__(NT) cfl_init_kernel_f64(const double* __restrict__ u,
                                                         const uint8_t* __restrict__ mask,
                                                         Geometry g, Consts k, Ctrl* ctrl,
                                                         int has_mask)
{
    double smax = 0.0;
    const long long ncell = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; c < ncell;
         c += static_cast<long long>(gridDim.x) * NT) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        if (has_mask && is_solid(mask, g, x, y)) {
            continue;
        }
        double r[9];
        load_cons_f64(u, g, x, y, r);
        smax = vmax(smax, PolicyF64::signal_speed(r, k));
    }
    reduce_signal_speed_and_finish(smax, ctrl, k, gridDim.x, false);
}

} // namespace mhdb
