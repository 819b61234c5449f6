// Fused SSP-RK2 stage kernels, plain FP64 form.
//
// One CTA owns a TX x TY tile of interior cells. A stage is one pass over HBM:
//   1. stage the tile plus its 2-cell halo of the 9 conserved fields into shared memory as
//      primitives; boundary conditions are index maps (periodic wrap / outflow clamp) applied
//      while loading, and solid cells of the mask are wall-filled from their fluid neighbours;
//   2. (non-ideal) cell-centred current J = curl B on the tile plus a 1-cell ring;
//   3. every x- and y-face flux of the tile (MUSCL + HLL + GLM, plus the non-ideal E terms),
//      each face evaluated once, into shared memory;
//   4. L = -dF/dx - dG/dy, Dedner psi damping, L = 0 on solids, and the stage update
//      (stage 1: U* = U + dt L; stage 2: U = (U + U*)/2 + (dt/2) L, written in place);
//   5. stage 2 also reduces the next step's max signal speed (warp shuffles, one 64-bit atomic
//      max per CTA) and the last CTA to finish turns it into the next dt (FP64 clock).
//
// Reference semantics followed: ssp_rk2_step (include/mhd/time_integrator.hpp:36-60), BC
// before wall fill (ghosts see pre-fill values), compute_rhs (include/mhd/rhs.hpp:140-240),
// field_xpay / field_ssp_rk2_combine (include/mhd/field_ops.hpp:47-63), compute_cfl_dt
// (include/mhd/cfl.hpp:28-92) and the solve() loop condition (time_integrator.hpp:84-99).
#pragma once

#include "physics.cuh"
#include "runtime_types.cuh"

namespace mhdb {

template <int TX, int TY>
struct TileShape {
    static constexpr int HX = TX + 4;
    static constexpr int HY = TY + 4;
    static constexpr int NH = HX * HY;                 // halo cells
    static constexpr int NFX = (TX + 1) * TY;          // x-faces
    static constexpr int NFY = TX * (TY + 1);          // y-faces
    static constexpr int JX = TX + 2;
    static constexpr int JY = TY + 2;
    static constexpr int NJ = JX * JY;                 // current cells
    static constexpr int NC = TX * TY;                 // owned cells
};

template <int TX, int TY, bool NI>
constexpr size_t stage_smem_bytes_f64()
{
    using S = TileShape<TX, TY>;
    return sizeof(double) * (9 * S::NH + 9 * S::NFX + 9 * S::NFY + (NI ? 3 * S::NJ : 0));
}

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

// Wall fill of solid interior cell (x, y) from the state u (include/mhd/mask.hpp:100-146):
// first fluid interior neighbour in the order +x, -x, +y, -y.
__device__ __forceinline__ void wall_fill_f64(const double* __restrict__ u,
                                              const uint8_t* __restrict__ mask, const Geometry& g,
                                              int x, int y, double gm1, double* out)
{
    const int cx[4] = {x + 1, x - 1, x, x};
    const int cy[4] = {y, y, y + 1, y - 1};
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        const int nx = cx[k], ny = cy[k];
        if (nx < 0 || ny < 0 || nx >= g.nx || ny >= g.ny) {
            continue;
        }
        if (mask[static_cast<size_t>(ny) * g.pitch + nx] == 0) {
            continue;
        }
        double s[9];
        load_cons_f64(u, g, nx, ny, s);
        reflect_fill(s, k < 2 ? 0 : 1, gm1, out);
        return;
    }
    isolated_fill(gm1, out);
}

__device__ __forceinline__ bool is_solid(const uint8_t* __restrict__ mask, const Geometry& g,
                                         int x, int y)
{
    return mask[static_cast<size_t>(y) * g.pitch + x] == 0;
}

template <int L, bool NI, bool MASK, int STAGE, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 2) stage_kernel_f64(const StageArgsF64 a)
{
    using S = TileShape<TX, TY>;
    constexpr int HX = S::HX;
    const Ctrl* __restrict__ ctrl = a.ctrl;
    if (ctrl->finished != 0) {
        return;
    }
    extern __shared__ double smem[];
    double* sW = smem;                 // [9][HY][HX] primitives
    double* sFx = sW + 9 * S::NH;      // [9][TY][TX+1]
    double* sFy = sFx + 9 * S::NFX;    // [9][TY+1][TX]
    double* sJ = sFy + 9 * S::NFY;     // [3][TY+2][TX+2]

    const Geometry& g = a.geom;
    const Consts& k = a.k;
    const int x0 = blockIdx.x * TX;
    const int y0 = blockIdx.y * TY;
    const double* __restrict__ uin = a.uin;
    const double dt = ctrl->dt;
    const double c_h = ctrl->c_h;

    // 1. Stage tile + halo as primitives.
    for (int t = threadIdx.x; t < S::NH; t += NT) {
        const int lx = t % HX, ly = t / HX;
        const int gx = x0 - 2 + lx, gy = y0 - 2 + ly;
        const int sx = map_index(gx, g.nx, g.bc_x);
        const int sy = map_index(gy, g.ny, g.bc_y);
        double u[9];
        const bool interior = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny;
        if (MASK && a.walls && interior && is_solid(a.mask, g, sx, sy)) {
            wall_fill_f64(uin, a.mask, g, sx, sy, k.gm1, u);
        } else {
            load_cons_f64(uin, g, sx, sy, u);
        }
        double w[9];
        cons_to_prim(u, k.gm1, w);
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            sW[c * S::NH + t] = w[c];
        }
    }
    __syncthreads();

    // 2. Current J on the tile plus a 1-cell ring (include/mhd/nonideal.hpp:30-60).
    if constexpr (NI) {
        for (int t = threadIdx.x; t < S::NJ; t += NT) {
            const int jx = t % S::JX + 1, jy = t / S::JX + 1;
            const int i = jy * HX + jx;
            const double* bx = sW + 5 * S::NH;
            const double* by = sW + 6 * S::NH;
            const double* bz = sW + 7 * S::NH;
            const double dbz_dy = (bz[i + HX] - bz[i - HX]) * k.inv_2dy;
            const double dbz_dx = (bz[i + 1] - bz[i - 1]) * k.inv_2dx;
            const double dby_dx = (by[i + 1] - by[i - 1]) * k.inv_2dx;
            const double dbx_dy = (bx[i + HX] - bx[i - HX]) * k.inv_2dy;
            sJ[0 * S::NJ + t] = dbz_dy;
            sJ[1 * S::NJ + t] = -dbz_dx;
            sJ[2 * S::NJ + t] = dby_dx - dbx_dy;
        }
        __syncthreads();
    }

    // 3. Face fluxes: x-faces then y-faces in one flat work list.
    for (int t = threadIdx.x; t < S::NFX + S::NFY; t += NT) {
        const bool ydir = t >= S::NFX;
        const int tt = ydir ? t - S::NFX : t;
        const int w = ydir ? TX : TX + 1;
        const int fx = tt % w, fy = tt / w;
        const int base = (fy + 2) * HX + (fx + 2); // right / upper cell of the face
        const int stride = ydir ? HX : 1;
        const int pn = ydir ? 2 : 1, pt = ydir ? 1 : 2;
        const int bn = ydir ? 6 : 5, bt = ydir ? 5 : 6;
        PrimN<double> W[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int i = base + (s - 2) * stride;
            W[s].rho = sW[0 * S::NH + i];
            W[s].vn = sW[pn * S::NH + i];
            W[s].vt = sW[pt * S::NH + i];
            W[s].vz = sW[3 * S::NH + i];
            W[s].p = sW[4 * S::NH + i];
            W[s].bn = sW[bn * S::NH + i];
            W[s].bt = sW[bt * S::NH + i];
            W[s].bz = sW[7 * S::NH + i];
            W[s].psi = sW[8 * S::NH + i];
        }
        const FluxN<double> f =
            muscl_hll_face<L>(W[0], W[1], W[2], W[3], k.gamma, k.inv_gm1, c_h);
        double out[9];
        out[0] = f.rho;
        out[1] = ydir ? f.mt : f.mn;
        out[2] = ydir ? f.mn : f.mt;
        out[3] = f.mz;
        out[4] = f.e;
        out[5] = ydir ? f.bt : f.bn;
        out[6] = ydir ? f.bn : f.bt;
        out[7] = f.bz;
        out[8] = f.psi;
        if constexpr (NI) {
            {
                // Face-averaged J and B (include/mhd/rhs.hpp:75-114).
                const int jr = (fy + 1) * S::JX + (fx + 1);
                const int jl = jr - (ydir ? S::JX : 1);
                const int il = base - stride;
                const double Jx = 0.5 * (sJ[jl] + sJ[jr]);
                const double Jy = 0.5 * (sJ[S::NJ + jl] + sJ[S::NJ + jr]);
                const double Jz = 0.5 * (sJ[2 * S::NJ + jl] + sJ[2 * S::NJ + jr]);
                const double Bx = 0.5 * (sW[5 * S::NH + il] + sW[5 * S::NH + base]);
                const double By = 0.5 * (sW[6 * S::NH + il] + sW[6 * S::NH + base]);
                const double Bz = 0.5 * (sW[7 * S::NH + il] + sW[7 * S::NH + base]);
                double Ex, Ey, Ez;
                nonideal_e(Jx, Jy, Jz, Bx, By, Bz, k.ni, Ex, Ey, Ez);
                if (!ydir) {
                    out[6] += -Ez;
                    out[7] += Ey;
                    out[4] += By * Ez - Bz * Ey;
                } else {
                    out[5] += Ez;
                    out[7] += -Ex;
                    out[4] += Bz * Ex - Bx * Ez;
                }
            }
        }
        double* dst = ydir ? (sFy + tt) : (sFx + tt);
        const int pstride = ydir ? S::NFY : S::NFX;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            dst[c * pstride] = out[c];
        }
    }
    __syncthreads();

    // 4. Divergence, psi damping, solid zeroing and the stage update of owned cells.
    const double psi_damp = (c_h > 0.0 && k.glm_alpha > 0.0) ? (c_h * k.glm_alpha / k.h) : 0.0;
    double smax = 0.0;
    for (int t = threadIdx.x; t < S::NC; t += NT) {
        const int cx = t % TX, cy = t / TX;
        const int gx = x0 + cx, gy = y0 + cy;
        if (gx >= g.nx || gy >= g.ny) {
            continue;
        }
        const bool solid = MASK && is_solid(a.mask, g, gx, gy);
        double Lc[9];
        const int fxi = cy * (TX + 1) + cx;
        const int fyi = cy * TX + cx;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            Lc[c] = -(sFx[c * S::NFX + fxi + 1] - sFx[c * S::NFX + fxi]) * k.inv_dx -
                    (sFy[c * S::NFY + fyi + TX] - sFy[c * S::NFY + fyi]) * k.inv_dy;
        }
        if (psi_damp != 0.0) {
            Lc[8] -= psi_damp * sW[8 * S::NH + (cy + 2) * HX + (cx + 2)];
        }
        if (solid) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                Lc[c] = 0.0;
            }
        }
        const size_t o = static_cast<size_t>(gy) * g.pitch + gx;
        if constexpr (STAGE == 1) {
            double u[9];
            if (solid && a.walls) {
                wall_fill_f64(uin, a.mask, g, gx, gy, k.gm1, u);
            } else {
                load_cons_f64(uin, g, gx, gy, u);
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                a.out[static_cast<size_t>(c) * g.plane + o] = u[c] + dt * Lc[c];
            }
        } else {
            // uin = U*, out = U^n (updated in place). For solid cells U*'s stored value is the
            // (wall-filled) U^n written by stage 1, and the stage input is the wall fill of U*.
            double us[9], un[9];
            if (solid) {
                if (a.walls) {
                    wall_fill_f64(uin, a.mask, g, gx, gy, k.gm1, us);
                } else {
                    load_cons_f64(uin, g, gx, gy, us);
                }
                load_cons_f64(uin, g, gx, gy, un);
            } else {
                load_cons_f64(uin, g, gx, gy, us);
                load_cons_f64(a.out, g, gx, gy, un);
            }
            const double half_dt = 0.5 * dt;
            double r[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                r[c] = 0.5 * (un[c] + us[c]) + half_dt * Lc[c];
                a.out[static_cast<size_t>(c) * g.plane + o] = r[c];
            }
            if (!solid) {
                const double s = cell_max_signal_speed(r[0], r[1], r[2], r[3], r[4], r[5], r[6],
                                                       r[7], k.gamma);
                smax = vmax(smax, s);
            }
        }
    }

    if constexpr (STAGE == 2) {
        reduce_signal_speed_and_finish(smax, a.ctrl, a.k, gridDim.x * gridDim.y, true);
    }
}

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
        smax = vmax(smax, cell_max_signal_speed(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7],
                                                k.gamma));
    }
    reduce_signal_speed_and_finish(smax, ctrl, k, gridDim.x, false);
}

} // namespace mhdb
