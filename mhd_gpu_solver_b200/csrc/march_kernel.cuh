// Warp-synchronous strip-march stage kernel (ideal GLM-MHD, no solid mask).
//
// Each warp owns a strip of kMarchOwned = 28 columns and a segment of LY rows. Lane l holds
// column x0 - 2 + l (lanes 0, 1 and 30, 31 are the x halo) and the warp marches up the segment
// one row at a time, so the whole stencil lives in registers:
//   * the primitives of rows j and j+1, the y slope of row j and the y flux G(j-1/2) are carried
//     from one row to the next; row j+2 is converted from a load issued one row earlier;
//   * x neighbours come from warp shuffles: W(x+1), the left difference, the right neighbour's
//     slope and the left face's flux;
//   * every face is evaluated once per lane (x face x+1/2 and y face j+1/2), every slope is
//     limited once, exactly as in the shared-memory tile kernel, so both produce the same values.
// There is no shared memory and no barrier until the stage-2 signal-speed reduction. Boundary
// conditions are the same index maps (periodic wrap / outflow clamp) applied to every load.
//
// A block is NW warps side by side (NW * 28 columns x LY rows), so the host's tile grid
// arithmetic is the same as for the tile kernel.
#pragma once

#include "stage_kernel.cuh"

namespace mhdb {

constexpr int kMarchOwned = 28; // owned columns per warp (lanes 2..29)

template <class Policy, int L, int STAGE, int LY>
__device__ __forceinline__ double march_strip(const typename Policy::Args& a, int x0, int y0,
                                              int lane)
{
    using T = typename Policy::T;
    using Raw = typename Policy::Raw;
    constexpr unsigned kFull = 0xffffffffu;
    const Geometry& g = a.geom;
    const Consts& k = a.k;
    const double dt = a.ctrl->dt;
    const double c_h64 = a.ctrl->c_h;
    const T c_h = static_cast<T>(c_h64);
    const T gamma = static_cast<T>(k.gamma);
    const T inv_gm1 = static_cast<T>(k.inv_gm1);
    const T inv_dx = static_cast<T>(k.inv_dx), inv_dy = static_cast<T>(k.inv_dy);
    const double psi_damp = (c_h64 > 0.0 && k.glm_alpha > 0.0) ? (c_h64 * k.glm_alpha / k.h) : 0.0;

    const int gx = x0 - 2 + lane;
    const int sx = map_index(gx, g.nx, g.bc_x);
    const bool own = lane >= 2 && lane < 2 + kMarchOwned && gx < g.nx;
    const int y1 = min(y0 + LY, g.ny);

    auto load = [&](int y, Raw& r) { Policy::load_raw(a, g, sx, map_index(y, g.ny, g.bc_y), r); };
    auto prim = [&](int y, const Raw& r, T (&w)[9]) {
        Policy::template raw_prim<STAGE, false>(a, g, sx, map_index(y, g.ny, g.bc_y), r, k, w);
    };

    // Prologue: rows y0-2 .. y0+1, slopes of rows y0-1 and y0, flux G(y0 - 1/2).
    T Wm[9], Wp[9], sYc[9], Gm[9];
    Raw rn;
    {
        Raw r0, r1, r2, r3;
        load(y0 - 2, r0);
        load(y0 - 1, r1);
        load(y0, r2);
        load(y0 + 1, r3);
        load(y0 + 2, rn);
        T wa[9], wb[9], sYm[9];
        prim(y0 - 2, r0, wa);
        prim(y0 - 1, r1, wb);
        prim(y0, r2, Wm);
        prim(y0 + 1, r3, Wp);
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            sYm[c] = limit_slope<L>(wb[c] - wa[c], Wm[c] - wb[c]);
            sYc[c] = limit_slope<L>(Wm[c] - wb[c], Wp[c] - Wm[c]);
        }
        face_flux_regs<T, true>(wb, sYm, Wm, sYc, gamma, inv_gm1, c_h, Gm);
    }

    double smax = 0.0;
#pragma unroll 1
    for (int y = y0; y < y1; ++y) {
        // x sweep of row y: dF = F(x + 1/2) - F(x - 1/2) on the owned lanes
        T dF[9];
        {
            T Wn[9], sX[9], sXn[9], F[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                Wn[c] = __shfl_down_sync(kFull, Wm[c], 1);
                const T dR = Wn[c] - Wm[c];
                const T dL = __shfl_up_sync(kFull, dR, 1);
                sX[c] = limit_slope<L>(dL, dR);
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                sXn[c] = __shfl_down_sync(kFull, sX[c], 1);
            }
            face_flux_regs<T, false>(Wm, sX, Wn, sXn, gamma, inv_gm1, c_h, F);
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                dF[c] = F[c] - __shfl_up_sync(kFull, F[c], 1);
            }
        }
        // row y+3 in flight while row y+2 is converted and the y face y+1/2 is evaluated
        Raw rq;
        load(y + 3, rq);
        T W2[9], sYn[9], Gp[9];
        prim(y + 2, rn, W2);
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            sYn[c] = limit_slope<L>(Wp[c] - Wm[c], W2[c] - Wp[c]);
        }
        face_flux_regs<T, true>(Wm, sYc, Wp, sYn, gamma, inv_gm1, c_h, Gp);
        if (own) {
            T Lc[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                Lc[c] = -dF[c] * inv_dx - (Gp[c] - Gm[c]) * inv_dy; // include/mhd/rhs.hpp:121
            }
            Policy::template update<STAGE, false>(a, g, gx, y, false, Lc, Wm[8], psi_damp, dt, k,
                                                  smax);
        }
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            Wm[c] = Wp[c];
            Wp[c] = W2[c];
            sYc[c] = sYn[c];
            Gm[c] = Gp[c];
        }
        rn = rq;
    }
    return smax;
}

template <class Policy, int L, int STAGE, int LY, int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) march_kernel(const typename Policy::Args a)
{
    if (a.ctrl->finished != 0) {
        return;
    }
    const int lane = threadIdx.x & 31;
    const int strip = blockIdx.x * NW + (threadIdx.x >> 5);
    const int x0 = strip * kMarchOwned;
    double smax = 0.0;
    if (x0 < a.geom.nx) { // warp-uniform
        smax = march_strip<Policy, L, STAGE, LY>(a, x0, static_cast<int>(blockIdx.y) * LY, lane);
    }
    if constexpr (STAGE == 2) {
        reduce_signal_speed_and_finish(smax, a.ctrl, a.k, gridDim.x * gridDim.y, true);
    }
}

} // namespace mhdb
