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
    static constexpr int kLayout = 0; // MarchTmaLayout of the stored form
    struct Raw {
        double v[9];
    };
    static __device__ __forceinline__ void load_raw(const Args& a, const Geometry& g, int x, int y,
                                                    Raw& r)
    {
        load_cons_f64(a.uin, g, x, y, r.v);
    }
    template <int STAGE, bool MASK>
    static __device__ __forceinline__ void raw_prim(const Args&, const Geometry&, int, int,
                                                    const Raw& r, const Consts& k, double* w)
    {
        cons_to_prim(r.v, k.gm1, w);
    }
    static __device__ __forceinline__ void prim_of(const double* f, const Consts& k, double* w)
    {
        cons_to_prim(f, k.gm1, w);
    }
    template <int STAGE, bool MASK>
    static __device__ __forceinline__ void wall_fill(const Args& a, const Geometry& g, int x,
                                                     int y, double gm1, double* out)
    {
        wall_fill_f64(a.uin, a.mask, g, x, y, gm1, out);
    }
    static __device__ __forceinline__ double signal_speed(const double* r, const Consts& k)
    {
        return cell_max_signal_speed(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], k.gamma);
    }

    // Stage update of one owned cell: stage 1 U* = U + dt L (include/mhd/field_ops.hpp:51);
    // stage 2 U = (U + U*)/2 + (dt/2) L in place (field_ops.hpp:61). For a solid cell the stored
    // U* is the (wall-filled) U^n written by stage 1 and the stage input is the fill of U*.
    template <int STAGE, bool MASK>
    static __device__ __forceinline__ void update(const Args& a, const Geometry& g, int gx, int gy,
                                                  bool solid, double (&L)[9], double psi_in,
                                                  double psi_damp, double dt, const Consts& k,
                                                  double& smax)
    {
        if (psi_damp != 0.0) {
            L[8] -= psi_damp * psi_in; // include/mhd/rhs.hpp:219-225
        }
        if (solid) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                L[c] = 0.0;
            }
        }
        if (solid && a.walls) {
            double uin[9];
            wall_fill_f64(a.uin, a.mask, g, gx, gy, k.gm1, uin);
            // a solid cell's stored U* is the fill of U^n and U^n is the stage input
            update_ops<STAGE>(a, g, gx, gy, solid, L, dt, k, smax, [&](int i) {
                return i < 9 ? uin[i] : __ldg(a.uin + static_cast<size_t>(i - 9) * g.plane +
                                              static_cast<size_t>(gy) * g.pitch + gx);
            });
            return;
        }
        const size_t o = static_cast<size_t>(gy) * g.pitch + gx;
        const double* __restrict__ in = a.uin + o;
        // the stored U* of a solid cell (stage 2 input) stands in for its U^n
        const double* __restrict__ un = (solid ? a.uin : a.out) + o;
        const size_t pl = g.plane;
        update_ops<STAGE>(a, g, gx, gy, solid, L, dt, k, smax, [&](int i) {
            return i < 9 ? __ldg(in + static_cast<size_t>(i) * pl)
                         : un[static_cast<size_t>(i - 9) * pl];
        });
    }

    // The stage update of one cell from its own-cell operands op(i): plane i of the input (i < 9)
    // and, in stage 2, plane i - 9 of U^n (i < 18), which the stage overwrites; all are read
    // before any store.
    template <int STAGE, class Op>
    static __device__ __forceinline__ void update_ops(const Args& a, const Geometry& g, int gx,
                                                      int gy, bool solid, const double (&L)[9],
                                                      double dt, const Consts& k, double& smax,
                                                      const Op& op)
    {
        const size_t o = static_cast<size_t>(gy) * g.pitch + gx;
        double* __restrict__ out = a.out + o;
        const size_t pl = g.plane;
        double uin[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            uin[c] = op(c);
        }
        if constexpr (STAGE == 1) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                out[c * pl] = uin[c] + dt * L[c];
            }
        } else {
            double un[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                un[c] = op(9 + c);
            }
            const double half_dt = 0.5 * dt;
            double r2[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                r2[c] = 0.5 * (un[c] + uin[c]) + half_dt * L[c];
                out[c * pl] = r2[c];
            }
            if (!solid && reduce_row(g, gy)) {
                smax = vmax(smax, signal_speed(r2, k));
            }
        }
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
    const long long ncell = static_cast<long long>(g.nx) * (g.ry1 - g.ry0);
    for (long long c = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; c < ncell;
         c += static_cast<long long>(gridDim.x) * NT) {
        const int x = static_cast<int>(c % g.nx), y = g.ry0 + static_cast<int>(c / g.nx);
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
