// Fused SSP-RK2 stage kernel shared by both precision forms.
//
// One CTA owns a TX x TY tile of interior cells; a stage is one pass over HBM:
//   A. stage the tile plus its 2-cell halo of the 9 conserved fields into shared memory as
//      primitives; boundary conditions are index maps (periodic wrap / outflow clamp) applied
//      while loading, and solid cells are wall-filled from their fluid neighbours;
//   B. (non-ideal) cell-centred current J = curl B on the tile plus a 1-cell ring;
//   C. x sweep: every cell of the tile plus a 1-cell x ring limits its slope once per component
//      into shared memory; then every x-face flux (HLL + GLM + non-ideal E) is evaluated once
//      from the face states W(l) + s(l)/2 and W(r) - s(r)/2 of its two cells, and each owned
//      cell keeps dF = F(i+1/2) - F(i-1/2) in registers;
//   D. y sweep: the same for y, reusing the slope and flux buffers;
//   E. L = -dF/dx - dG/dy, Dedner psi damping, L = 0 on solids, and the stage update
//      (stage 1: U* = U + dt L; stage 2: U = (U + U*)/2 + (dt/2) L, written in place);
//   F. stage 2 reduces the next step's max signal speed (warp shuffles, one 64-bit atomic max
//      per CTA) and the last CTA to arrive turns it into the next dt (FP64 clock).
//
// Per-cell slopes give the same values as the reference's per-face reconstruction
// (include/mhd/kernels/muscl_hll.hpp:59-68): the left state of face i-1/2 is
// W(i-1) + lim(W(i-1) - W(i-2), W(i) - W(i-1))/2, built from cell i-1's slope, and the right
// state W(i) - lim(W(i) - W(i-1), W(i+1) - W(i))/2 from cell i's slope; each slope is limited
// once instead of once per adjacent face, with the same operations on the same operands.
//
// The arithmetic type T and the storage of the state come from the Policy (stage_f64.cuh:
// plain FP64; stage_mixed.cuh: FP32 arithmetic on a compensated hi/lo FP32 state).
#pragma once

#include "physics.cuh"
#include "runtime_types.cuh"

namespace mhdb {

template <int TX, int TY>
struct TileShape {
    static constexpr int HX = TX + 4;
    static constexpr int HY = TY + 4;
    static constexpr int NH = HX * HY;          // halo cells
    static constexpr int SXN = TY * (TX + 2);   // x-sweep face-state cells
    static constexpr int SYN = (TY + 2) * TX;   // y-sweep face-state cells
    static constexpr int SN = SXN > SYN ? SXN : SYN;
    static constexpr int NFX = (TX + 1) * TY;   // x-faces
    static constexpr int NFY = TX * (TY + 1);   // y-faces
    static constexpr int NF = NFX > NFY ? NFX : NFY;
    static constexpr int JX = TX + 2;
    static constexpr int JY = TY + 2;
    static constexpr int NJ = JX * JY;          // current cells
    static constexpr int NC = TX * TY;          // owned cells
};

// Shared memory of one tile. Separate sweeps reuse one slope buffer and one flux buffer for x
// and y; merged sweeps keep x and y buffers side by side.
template <class T, int TX, int TY, bool NI, bool MERGED = false>
constexpr size_t stage_smem_bytes()
{
    using S = TileShape<TX, TY>;
    const size_t slopes = MERGED ? (S::SXN + S::SYN) : S::SN;
    const size_t fluxes = MERGED ? (S::NFX + S::NFY) : S::NF;
    return sizeof(T) * (9 * S::NH + 9 * slopes + 9 * fluxes + (NI ? 3 * S::NJ : 0));
}

// One cell of a slope sweep: per component the limited slope s = lim(W - W_prev, W_next - W)
// (include/mhd/kernels/muscl_hll.hpp:64-65), stored at sS[c * sn + t]. Sweep regions: x: columns
// 1..TX+2 and rows 2..TY+1 of the halo tile; y: columns 2..TX+1 and rows 1..TY+2.
template <int L, class T, int TX, int TY, bool YDIR>
__device__ __forceinline__ void slope_item(const T* __restrict__ sW, T* __restrict__ sS, int sn,
                                           int t)
{
    using S = TileShape<TX, TY>;
    constexpr int HX = S::HX;
    constexpr int W = YDIR ? TX : TX + 2;
    constexpr int step = YDIR ? HX : 1;
    const int sx = t % W, sy = t / W;
    const int i = YDIR ? (sy + 1) * HX + (sx + 2) : (sy + 2) * HX + (sx + 1);
    if constexpr (L == kVanLeer && sizeof(T) == 8) {
        // the nine components at once: one division (limit_half_slopes), slope = 2 x half
        // slope (exact)
        T dm[9], dp[9], h[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const T* w = sW + c * S::NH + i;
            const T wm = w[-step], w0 = w[0], wp = w[step];
            dm[c] = w0 - wm;
            dp[c] = wp - w0;
        }
        limit_half_slopes<L>(dm, dp, h);
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            sS[c * sn + t] = T(2) * h[c];
        }
    } else {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const T* w = sW + c * S::NH + i;
            const T wm = w[-step], w0 = w[0], wp = w[step];
            sS[c * sn + t] = limit_slope<L>(w0 - wm, wp - w0);
        }
    }
}

template <int L, class T, int TX, int TY, int NT, bool YDIR>
__device__ __forceinline__ void face_states(const T* __restrict__ sW, T* __restrict__ sS)
{
    using S = TileShape<TX, TY>;
    constexpr int N = YDIR ? S::SYN : S::SXN;
    for (int t = threadIdx.x; t < N; t += NT) {
        slope_item<L, T, TX, TY, YDIR>(sW, sS, S::SN, t);
    }
}

// One face flux from the centre values lc, rc and limited slopes sl, sr (physical component
// order) of its two cells: left state W(l) + s(l)/2, right state W(r) - s(r)/2
// (include/mhd/kernels/muscl_hll.hpp:66-67), with the both-sides first-order fallback of
// muscl_hll.hpp:145-168. Output in physical component order. HALF: sl and sr hold half slopes
// s/2 (exact halves), so the face states are W(l) + s'(l) and W(r) - s'(r), the same values.
template <class T, bool YDIR, bool HALF = false>
__device__ __forceinline__ void face_flux_regs(const T (&lc)[9], const T (&sl)[9],
                                               const T (&rc)[9], const T (&sr)[9], T gamma,
                                               T inv_gm1, T c_h, T (&out)[9])
{
    // physical component feeding each rotated-frame slot (rho, vn, vt, vz, p, bn, bt, bz, psi)
    constexpr int comp[9] = {0, YDIR ? 2 : 1, YDIR ? 1 : 2, 3, 4, YDIR ? 6 : 5, YDIR ? 5 : 6, 7, 8};
    // Density and pressure of both states decide the fallback; then every component is
    // W + h s with h = 1/2 (second order) or h = 0 (first order: W + 0 s = W exactly for finite
    // slopes, and 0.5 s is exact, so both cases give the reference's values).
    const T inf = T(INFINITY);
    const T hs = HALF ? T(1) : T(0.5);
    const T l0 = lc[0] + hs * sl[0], l4 = lc[4] + hs * sl[4];
    const T r0 = rc[0] - hs * sr[0], r4 = rc[4] - hs * sr[4];
    const bool ok = (l0 > T(0)) && (l4 > T(0)) && (l0 < inf) && (l4 < inf) && (r0 > T(0)) &&
                    (r4 > T(0)) && (r0 < inf) && (r4 < inf);
    const T h = ok ? hs : T(0);
    T l[9], r[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        l[q] = lc[comp[q]] + h * sl[comp[q]];
        r[q] = rc[comp[q]] - h * sr[comp[q]];
    }
    const PrimN<T> WL{l[0], l[1], l[2], l[3], l[4], l[5], l[6], l[7], l[8]};
    const PrimN<T> WR{r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8]};
    const FluxN<T> f = hll_flux(WL, WR, gamma, inv_gm1, c_h);
    out[0] = f.rho;
    out[1] = YDIR ? f.mt : f.mn;
    out[2] = YDIR ? f.mn : f.mt;
    out[3] = f.mz;
    out[4] = f.e;
    out[5] = YDIR ? f.bt : f.bn;
    out[6] = YDIR ? f.bn : f.bt;
    out[7] = f.bz;
    out[8] = f.psi;
}

// The same from the shared-memory tile: centres sW[c * nh + wl|wr], slopes sS[c * sn + il|ir].
template <class T, bool YDIR>
__device__ __forceinline__ void face_flux(const T* __restrict__ sS, int sn, int il, int ir,
                                          const T* __restrict__ sW, int nh, int wl, int wr,
                                          T gamma, T inv_gm1, T c_h, T (&out)[9])
{
    T lc[9], rc[9], sl[9], sr[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        lc[c] = sW[c * nh + wl];
        rc[c] = sW[c * nh + wr];
        sl[c] = sS[c * sn + il];
        sr[c] = sS[c * sn + ir];
    }
    face_flux_regs<T, YDIR>(lc, sl, rc, sr, gamma, inv_gm1, c_h, out);
}

// Non-ideal correction of one face flux from the cell-centred current J and field B of its two
// cells (l: left/below, r: right/above): face averages, E from Ohm's law, then the x-face
// (F_by -= Ez, F_bz += Ey, F_E += By Ez - Bz Ey) or y-face (G_bx += Ez, G_bz -= Ex,
// G_E += Bz Ex - Bx Ez) update; include/mhd/rhs.hpp:75-114.
template <class T, bool YDIR>
__device__ __forceinline__ void add_nonideal_face(T jxl, T jyl, T jzl, T jxr, T jyr, T jzr, T bxl,
                                                  T byl, T bzl, T bxr, T byr, T bzr,
                                                  const NonIdealCoef& ni, T (&out)[9])
{
    const T Jx = T(0.5) * (jxl + jxr);
    const T Jy = T(0.5) * (jyl + jyr);
    const T Jz = T(0.5) * (jzl + jzr);
    const T Bx = T(0.5) * (bxl + bxr);
    const T By = T(0.5) * (byl + byr);
    const T Bz = T(0.5) * (bzl + bzr);
    T Ex, Ey, Ez;
    nonideal_e(Jx, Jy, Jz, Bx, By, Bz, ni, Ex, Ey, Ez);
    if (!YDIR) {
        out[6] += -Ez;
        out[7] += Ey;
        out[4] += By * Ez - Bz * Ey;
    } else {
        out[5] += Ez;
        out[7] += -Ex;
        out[4] += Bz * Ex - Bx * Ez;
    }
}

// Cell-centred current J = curl B of one cell from its four neighbours' field components
// (include/mhd/nonideal.hpp:30-60): Jx = dBz/dy, Jy = -dBz/dx, Jz = dBy/dx - dBx/dy, central
// differences.
template <class T>
__device__ __forceinline__ void cell_current(T bz_n, T bz_s, T bz_e, T bz_w, T by_e, T by_w,
                                             T bx_n, T bx_s, T inv_2dx, T inv_2dy, T (&J)[3])
{
    const T dbz_dy = (bz_n - bz_s) * inv_2dy;
    const T dbz_dx = (bz_e - bz_w) * inv_2dx;
    const T dby_dx = (by_e - by_w) * inv_2dx;
    const T dbx_dy = (bx_n - bx_s) * inv_2dy;
    J[0] = dbz_dy;
    J[1] = -dbz_dx;
    J[2] = dby_dx - dbx_dy;
}

// One face of a sweep: flux (HLL + GLM + non-ideal E) into sF[c * fn + t]; sS/sn are the
// slopes of the same sweep (x: region width TX+2; y: width TX).
template <class T, int TX, int TY, bool YDIR, bool NI>
__device__ __forceinline__ void face_item(const T* __restrict__ sW, const T* __restrict__ sS,
                                          int sn, T* __restrict__ sF, int fn,
                                          const T* __restrict__ sJ, const NonIdealCoef& ni,
                                          T gamma, T inv_gm1, T c_h, int t)
{
    using S = TileShape<TX, TY>;
    constexpr int HX = S::HX;
    constexpr int FW = YDIR ? TX : TX + 1;      // faces per row
    constexpr int SW = YDIR ? TX : TX + 2;      // slope region width
    const int fx = t % FW, fy = t / FW;
    // cells left/below (l) and right/above (r) of the face in slope-region coordinates
    const int ir = YDIR ? (fy + 1) * SW + fx : fy * SW + (fx + 1);
    const int il = fy * SW + fx;
    // the same two cells in halo coordinates
    const int wr = (fy + 2) * HX + (fx + 2);
    const int wl = wr - (YDIR ? HX : 1);
    T out[9];
    face_flux<T, YDIR>(sS, sn, il, ir, sW, S::NH, wl, wr, gamma, inv_gm1, c_h, out);
    if constexpr (NI) {
        const int jr = (fy + 1) * S::JX + (fx + 1);
        const int jl = jr - (YDIR ? S::JX : 1);
        add_nonideal_face<T, YDIR>(sJ[jl], sJ[S::NJ + jl], sJ[2 * S::NJ + jl], sJ[jr],
                                   sJ[S::NJ + jr], sJ[2 * S::NJ + jr], sW[5 * S::NH + wl],
                                   sW[6 * S::NH + wl], sW[7 * S::NH + wl], sW[5 * S::NH + wr],
                                   sW[6 * S::NH + wr], sW[7 * S::NH + wr], ni, out);
    }
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        sF[c * fn + t] = out[c];
    }
}

// Fluxes of all faces of one sweep into sF, then each owned cell's flux difference into dF.
template <class T, int TX, int TY, int NT, bool YDIR, bool NI>
__device__ __forceinline__ void face_sweep(const T* __restrict__ sW, const T* __restrict__ sS,
                                           T* __restrict__ sF, const T* __restrict__ sJ,
                                           const NonIdealCoef& ni, T gamma, T inv_gm1, T c_h,
                                           T (&dF)[(TX * TY + NT - 1) / NT][9])
{
    using S = TileShape<TX, TY>;
    constexpr int NFACE = YDIR ? S::NFY : S::NFX;
    for (int t = threadIdx.x; t < NFACE; t += NT) {
        face_item<T, TX, TY, YDIR, NI>(sW, sS, S::SN, sF, S::NF, sJ, ni, gamma, inv_gm1, c_h, t);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < (TX * TY + NT - 1) / NT; ++r) {
        const int t = threadIdx.x + r * NT;
        if (t < S::NC) {
            const int cx = t % TX, cy = t / TX;
            const int f0 = YDIR ? cy * TX + cx : cy * (TX + 1) + cx;
            const int f1 = f0 + (YDIR ? TX : 1);
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                dF[r][c] = sF[c * S::NF + f1] - sF[c * S::NF + f0];
            }
        }
    }
}

// Phases A-E for the tile with lower-left interior cell (x0, y0); returns the largest signal
// speed of the owned fluid cells after a stage-2 update (0 for stage 1).
template <class Policy, int L, bool NI, bool MASK, int STAGE, int TX, int TY, int NT,
          bool MERGED = false>
__device__ __forceinline__ double stage_tile(const typename Policy::Args& a, int x0, int y0,
                                             unsigned char* smem_raw)
{
    using T = typename Policy::T;
    using S = TileShape<TX, TY>;
    constexpr int HX = S::HX;
    constexpr int R = (TX * TY + NT - 1) / NT; // owned cells per thread
    const Ctrl* __restrict__ ctrl = a.ctrl;
    T* sW = reinterpret_cast<T*>(smem_raw); // [9][HY][HX] primitives
    T* sS = sW + 9 * S::NH;                 // [9][SN] limited slopes of the current sweep
    T* sF = sS + 9 * S::SN;                 // [9][NF] face fluxes
    T* sJ = sF + 9 * S::NF;                 // [3][JY][JX] current

    const Geometry& g = a.geom;
    const Consts& k = a.k;
    const double dt = ctrl->dt;
    const double c_h64 = ctrl->c_h;
    const T c_h = static_cast<T>(c_h64);
    const T gamma = static_cast<T>(k.gamma);
    const T inv_gm1 = static_cast<T>(k.inv_gm1);

    // A. tile + halo as primitives. All loads of a thread are issued before any conversion so
    // that they are in flight together.
    {
        constexpr int HR = (S::NH + NT - 1) / NT;
        typename Policy::Raw raw[HR];
        int src[HR][2];
        bool fill[HR];
#pragma unroll
        for (int r = 0; r < HR; ++r) {
            const int t = threadIdx.x + r * NT;
            fill[r] = false;
            if (t < S::NH) {
                const int lx = t % HX, ly = t / HX;
                const int gx = x0 - 2 + lx, gy = y0 - 2 + ly;
                const int sx = map_index(gx, g.nx, g.bc_x);
                const int sy = map_index(gy, g.ny, g.bc_y);
                const bool interior = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny;
                src[r][0] = sx;
                src[r][1] = sy;
                fill[r] = MASK && a.walls && interior && is_solid(a.mask, g, sx, sy);
                if (!fill[r]) {
                    Policy::load_raw(a, g, sx, sy, raw[r]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < HR; ++r) {
            const int t = threadIdx.x + r * NT;
            if (t < S::NH) {
                T w[9];
                if (fill[r]) {
                    double f[9];
                    Policy::template wall_fill<STAGE, MASK>(a, g, src[r][0], src[r][1], k.gm1, f);
                    Policy::prim_of(f, k, w);
                } else {
                    Policy::template raw_prim<STAGE, MASK>(a, g, src[r][0], src[r][1], raw[r], k, w);
                }
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    sW[c * S::NH + t] = w[c];
                }
            }
        }
    }
    __syncthreads();

    // B. current J (include/mhd/nonideal.hpp:30-60)
    auto current_item = [&](int t) {
        const T inv_2dx = static_cast<T>(k.inv_2dx), inv_2dy = static_cast<T>(k.inv_2dy);
        const int jx = t % S::JX + 1, jy = t / S::JX + 1;
        const int i = jy * HX + jx;
        const T* bx = sW + 5 * S::NH;
        const T* by = sW + 6 * S::NH;
        const T* bz = sW + 7 * S::NH;
        T J[3];
        cell_current(bz[i + HX], bz[i - HX], bz[i + 1], bz[i - 1], by[i + 1], by[i - 1],
                     bx[i + HX], bx[i - HX], inv_2dx, inv_2dy, J);
        sJ[0 * S::NJ + t] = J[0];
        sJ[1 * S::NJ + t] = J[1];
        sJ[2 * S::NJ + t] = J[2];
    };

    T dFx[R][9];
    T dGy[R][9];
    if constexpr (!MERGED) {
        if constexpr (NI) {
            for (int t = threadIdx.x; t < S::NJ; t += NT) {
                current_item(t);
            }
        }
        // C. x sweep
        face_states<L, T, TX, TY, NT, false>(sW, sS);
        __syncthreads();
        face_sweep<T, TX, TY, NT, false, NI>(sW, sS, sF, sJ, k.ni, gamma, inv_gm1, c_h, dFx);
        __syncthreads();
        // D. y sweep
        face_states<L, T, TX, TY, NT, true>(sW, sS);
        __syncthreads();
        face_sweep<T, TX, TY, NT, true, NI>(sW, sS, sF, sJ, k.ni, gamma, inv_gm1, c_h, dGy);
    } else {
        // Merged sweeps: J, x slopes and y slopes in one flat work list; then x and y faces in
        // one list (x faces padded to whole warps so that no warp straddles the two kinds).
        T* sSx = sS;
        T* sSy = sSx + 9 * S::SXN;
        T* sFx = sSy + 9 * S::SYN;
        T* sFy = sFx + 9 * S::NFX;
        T* sJm = sFy + 9 * S::NFY;
        sJ = sJm;
        constexpr int NJI = NI ? S::NJ : 0;
        for (int t = threadIdx.x; t < NJI + S::SXN + S::SYN; t += NT) {
            if (t < NJI) {
                current_item(t);
            } else if (t < NJI + S::SXN) {
                slope_item<L, T, TX, TY, false>(sW, sSx, S::SXN, t - NJI);
            } else {
                slope_item<L, T, TX, TY, true>(sW, sSy, S::SYN, t - NJI - S::SXN);
            }
        }
        __syncthreads();
        constexpr int NFXP = (S::NFX + 31) / 32 * 32;
        for (int t = threadIdx.x; t < NFXP + S::NFY; t += NT) {
            if (t < NFXP) {
                if (t < S::NFX) {
                    face_item<T, TX, TY, false, NI>(sW, sSx, S::SXN, sFx, S::NFX, sJ, k.ni,
                                                    gamma, inv_gm1, c_h, t);
                }
            } else {
                face_item<T, TX, TY, true, NI>(sW, sSy, S::SYN, sFy, S::NFY, sJ, k.ni, gamma,
                                               inv_gm1, c_h, t - NFXP);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = threadIdx.x + r * NT;
            if (t < S::NC) {
                const int cx = t % TX, cy = t / TX;
                const int fxi = cy * (TX + 1) + cx;
                const int fyi = cy * TX + cx;
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    dFx[r][c] = sFx[c * S::NFX + fxi + 1] - sFx[c * S::NFX + fxi];
                    dGy[r][c] = sFy[c * S::NFY + fyi + TX] - sFy[c * S::NFY + fyi];
                }
            }
        }
    }

    // E. divergence, psi damping, solid zeroing and the stage update
    const T inv_dx = static_cast<T>(k.inv_dx), inv_dy = static_cast<T>(k.inv_dy);
    const double psi_damp = (c_h64 > 0.0 && k.glm_alpha > 0.0) ? (c_h64 * k.glm_alpha / k.h) : 0.0;
    double smax = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int t = threadIdx.x + r * NT;
        if (t >= S::NC) {
            continue;
        }
        const int cx = t % TX, cy = t / TX;
        const int gx = x0 + cx, gy = y0 + cy;
        if (gx >= g.nx || gy >= g.ny) {
            continue;
        }
        const bool solid = MASK && is_solid(a.mask, g, gx, gy);
        T Lc[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            Lc[c] = -dFx[r][c] * inv_dx - dGy[r][c] * inv_dy; // include/mhd/rhs.hpp:121
        }
        const T psi_in = sW[8 * S::NH + (cy + 2) * HX + (cx + 2)];
        Policy::template update<STAGE, MASK>(a, g, gx, gy, solid, Lc, psi_in, psi_damp, dt, k,
                                             smax);
    }
    return smax;
}

// One CTA per tile of one grid.
template <class Policy, int L, bool NI, bool MASK, int STAGE, int TX, int TY, int NT, int MINB,
          bool MERGED = false>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(const typename Policy::Args a)
{
    if (a.ctrl->finished != 0) {
        return;
    }
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const double smax = stage_tile<Policy, L, NI, MASK, STAGE, TX, TY, NT, MERGED>(
        a, blockIdx.x * TX, blockIdx.y * TY, smem_raw);
    if constexpr (STAGE == 2) {
        reduce_signal_speed_and_finish(smax, a.ctrl, a.k, gridDim.x * gridDim.y, true);
    }
}

// One solve of a batch: its stage arguments and its tiling.
template <class Policy>
struct BatchSolve {
    typename Policy::Args stage[2]; // stage 1 and stage 2 arguments
    int tiles_x;                    // tiles per row
    int ntiles;                     // tiles of this solve
};

// Persistent form over a tile work-list of many independent solves (each item: solve index,
// tile index). Every CTA walks the list with a grid stride; a solve's signal-speed reduction
// completes when its last tile arrives, whichever CTA processes it, and that tile advances the
// solve's own FP64 clock. Finished solves are skipped.
template <class Policy, int L, bool NI, int STAGE, int TX, int TY, int NT, int MINB,
          bool MERGED = false>
__global__ void __launch_bounds__(NT, MINB) batch_stage_kernel(const BatchSolve<Policy>* solves,
                                                              const int2* __restrict__ work,
                                                              int nwork)
{
    using Args = typename Policy::Args;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) Args sa;
    __shared__ int s_tiles_x, s_ntiles;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 it = work[w];
        __syncthreads(); // the previous tile is done with shared memory
        {
            const int* src = reinterpret_cast<const int*>(&solves[it.x].stage[STAGE - 1]);
            int* dst = reinterpret_cast<int*>(&sa);
            for (int i = threadIdx.x; i < static_cast<int>(sizeof(Args) / sizeof(int)); i += NT) {
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
        const int x0 = (it.y % s_tiles_x) * TX;
        const int y0 = (it.y / s_tiles_x) * TY;
        const double smax =
            stage_tile<Policy, L, NI, false, STAGE, TX, TY, NT, MERGED>(sa, x0, y0, smem_raw);
        if constexpr (STAGE == 2) {
            reduce_signal_speed_and_finish(smax, sa.ctrl, sa.k, static_cast<unsigned>(s_ntiles),
                                           true);
        }
    }
}

} // namespace mhdb
