// Warp-synchronous strip-march stage kernel (ideal or non-ideal GLM-MHD, no solid mask).
//
// Each warp owns a strip of kMarchOwned = 28 columns and a segment of LY rows. Lane l holds
// column x0 - 2 + l (lanes 0, 1 and 30, 31 are the x halo) and the warp marches up the segment
// one row at a time, so the whole stencil lives in registers:
//   * the primitives of rows j and j+1, the y slope of row j and the y flux G(j-1/2) are carried
//     from one row to the next; row j+2 is converted from a load issued one row earlier;
//   * x neighbours come from warp shuffles: W(x+1), the left difference, the right neighbour's
//     slope and the left face's flux;
//   * every face is evaluated once per lane (x face x+1/2 and y face j+1/2), every slope is
//     limited once, with the same per-face and per-cell functions as the shared-memory tile
//     kernel (both are held to the oracle at the same tolerances).
// There is no shared memory and no barrier until the stage-2 signal-speed reduction. Boundary
// conditions are the same index maps (periodic wrap / outflow clamp) applied to every load.
// Non-ideal terms (NI): the current J of row y is carried like the primitives; J of row y + 1 is
// formed from rows y, y + 1, y + 2 and the x neighbours by shuffles, and both face fluxes get the
// Ohm's-law correction from face-averaged J and B, as in the tile kernel.
//
// A block is NW warps side by side (NW * 28 columns x LY rows), so the host's tile grid
// arithmetic is the same as for the tile kernel.
#pragma once

#include "stage_kernel.cuh"

namespace mhdb {

constexpr int kMarchOwned = 28; // owned columns per warp (lanes 2..29)

// Current J of the cells of row c (rows s below and n above) of a strip: x neighbours by shuffle.
// Lanes 0 and 31 get wrong values (they have no neighbour lane); no used face reads them.
template <class T>
__device__ __forceinline__ void march_current(const T (&Ws)[9], const T (&Wc)[9],
                                              const T (&Wn)[9], T inv_2dx, T inv_2dy, T (&J)[3])
{
    constexpr unsigned kFull = 0xffffffffu;
    const T bz_e = __shfl_down_sync(kFull, Wc[7], 1), bz_w = __shfl_up_sync(kFull, Wc[7], 1);
    const T by_e = __shfl_down_sync(kFull, Wc[6], 1), by_w = __shfl_up_sync(kFull, Wc[6], 1);
    cell_current(Wn[7], Ws[7], bz_e, bz_w, by_e, by_w, Wn[5], Ws[5], inv_2dx, inv_2dy, J);
}

// Non-ideal correction of the x face between this lane's cell (J, W) and the next lane's.
template <class T>
__device__ __forceinline__ void march_nonideal_x(const T (&J)[3], const T (&W)[9],
                                                 const T (&Wn)[9], const NonIdealCoef& ni,
                                                 T (&F)[9])
{
    constexpr unsigned kFull = 0xffffffffu;
    const T jx = __shfl_down_sync(kFull, J[0], 1), jy = __shfl_down_sync(kFull, J[1], 1),
            jz = __shfl_down_sync(kFull, J[2], 1);
    add_nonideal_face<T, false>(J[0], J[1], J[2], jx, jy, jz, W[5], W[6], W[7], Wn[5], Wn[6],
                                Wn[7], ni, F);
}

// Non-ideal correction of the y face between row cells (Jb, Wb) below and (Ja, Wa) above.
template <class T>
__device__ __forceinline__ void march_nonideal_y(const T (&Jb)[3], const T (&Wb)[9],
                                                 const T (&Ja)[3], const T (&Wa)[9],
                                                 const NonIdealCoef& ni, T (&G)[9])
{
    add_nonideal_face<T, true>(Jb[0], Jb[1], Jb[2], Ja[0], Ja[1], Ja[2], Wb[5], Wb[6], Wb[7],
                               Wa[5], Wa[6], Wa[7], ni, G);
}

template <class Policy, int L, int STAGE, int LY, bool NI = false>
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
    const T inv_2dx = static_cast<T>(k.inv_2dx), inv_2dy = static_cast<T>(k.inv_2dy);

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
    T Jc[NI ? 3 : 1]; // current of row y (NI)
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
        if constexpr (NI) {
            T Jb[3];
            march_current(wa, wb, Wm, inv_2dx, inv_2dy, Jb);
            march_current(wb, Wm, Wp, inv_2dx, inv_2dy, Jc);
            march_nonideal_y(Jb, wb, Jc, Wm, k.ni, Gm);
        }
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
            if constexpr (NI) {
                march_nonideal_x(Jc, Wm, Wn, k.ni, F);
            }
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
        T Jn[NI ? 3 : 1];
        if constexpr (NI) {
            march_current(Wm, Wp, W2, inv_2dx, inv_2dy, Jn);
            march_nonideal_y(Jc, Wm, Jn, Wp, k.ni, Gp);
        }
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
        if constexpr (NI) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                Jc[c] = Jn[c];
            }
        }
        rn = rq;
    }
    return smax;
}

template <class Policy, int L, int STAGE, int LY, int NW, int MINB, bool NI = false>
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
        smax = march_strip<Policy, L, STAGE, LY, NI>(a, x0, static_cast<int>(blockIdx.y) * LY, lane);
    }
    if constexpr (STAGE == 2) {
        reduce_signal_speed_and_finish(smax, a.ctrl, a.k, gridDim.x * gridDim.y, true);
    }
}

// Persistent strip-march form over a block work-list of many independent solves (each item:
// solve index, block index; a block is NW strips of 28 columns by LY rows; Desc is any
// descriptor with stage[2], tiles_x and ntiles). Every CTA walks the
// list with a grid stride, like batch_stage_kernel in stage_kernel.cuh; a solve's signal-speed
// reduction completes when its last block arrives and that block advances the solve's clock.
template <class Policy, int L, bool NI, int STAGE, int LY, int NW, int MINB,
          class Desc = BatchSolve<Policy>>
__global__ void __launch_bounds__(NW * 32, MINB) batch_march_kernel(const Desc* solves,
                                                                     const int2* __restrict__ work,
                                                                     int nwork)
{
    using Args = typename Policy::Args;
    __shared__ __align__(16) Args sa;
    __shared__ int s_tiles_x, s_ntiles;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 it = work[w];
        __syncthreads(); // the previous item is done with sa
        {
            const int* src = reinterpret_cast<const int*>(&solves[it.x].stage[STAGE - 1]);
            int* dst = reinterpret_cast<int*>(&sa);
            for (int i = threadIdx.x; i < static_cast<int>(sizeof(Args) / sizeof(int)); i += NW * 32) {
                dst[i] = src[i];
            }
            if (threadIdx.x == 0) {
                s_tiles_x = solves[it.x].tiles_x;
                s_ntiles = solves[it.x].ntiles;
            }
        }
        __syncthreads();
        if (sa.ctrl->finished != 0) {
            continue;
        }
        const int x0 = ((it.y % s_tiles_x) * NW + warp) * kMarchOwned;
        const int y0 = (it.y / s_tiles_x) * LY;
        double smax = 0.0;
        if (x0 < sa.geom.nx) { // warp-uniform
            smax = march_strip<Policy, L, STAGE, LY, NI>(sa, x0, y0, lane);
        }
        if constexpr (STAGE == 2) {
            reduce_signal_speed_and_finish(smax, sa.ctrl, sa.k, static_cast<unsigned>(s_ntiles),
                                           true);
        }
    }
}

} // namespace mhdb
