// Fused SSP-RK2 stage kernels, FP32-mixed form.
//
// Same tile algorithm as the FP64 form (stage_f64.cuh), with these precision rules:
//   * the state is carried as a compensated pair of FP32 planes, value = hi + lo with
//     |lo| <= ulp(hi)/2, so it holds ~48 significant bits; the stage update is done in FP64 on
//     (hi + lo) and split again, so the RK2 combination loses no bits;
//   * reconstruction, HLL fluxes, non-ideal terms and the divergence run in FP32 on hi;
//   * pressure recovery p = (gamma-1)(E - rho v^2/2 - B^2/2) is redone in FP64 from hi + lo in
//     cells where the FP32 subtraction cancels (p / (gamma-1) < E / kCancelRatio): low-beta or
//     high-Mach cells;
//   * the wall fill of solid cells is done in FP64 from hi + lo, like the plain form;
//   * the clock, dt and the CFL step control stay in FP64 (runtime_types.cuh); the per-cell
//     signal speed is evaluated in FP32.
#pragma once

#include "physics.cuh"
#include "runtime_types.cuh"
#include "stage_f64.cuh"

namespace mhdb {

// FP64 pressure recovery when E / (p/(gamma-1)) exceeds this ratio (>= 3 bits cancelled).
constexpr float kCancelRatio = 8.0f;

struct MixedState {
    float* hi; // 9 planes
    float* lo; // 9 planes
};

struct StageArgsMx {
    MixedState uin; // stage input (U^n for stage 1, U* for stage 2)
    MixedState out; // U* (stage 1) or U^n updated in place (stage 2)
    const uint8_t* mask;
    Ctrl* ctrl;
    Geometry geom;
    Consts k;
    int walls;
};

// One state buffer of 9 * plane * 8 bytes viewed as 9 hi planes followed by 9 lo planes.
inline MixedState mixed_view(void* base, const Geometry& g)
{
    float* f = static_cast<float*>(base);
    return MixedState{f, f + 9 * g.plane};
}

__device__ __forceinline__ void split_store(const MixedState& s, size_t off, double v)
{
    const float h = __double2float_rn(v);
    const float l = __double2float_rn(v - static_cast<double>(h));
    s.hi[off] = h;
    s.lo[off] = l;
}

__device__ __forceinline__ void load_cons_mx(const MixedState& u, const Geometry& g, int x, int y,
                                             double* out)
{
    const size_t k = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const size_t o = static_cast<size_t>(c) * g.plane + k;
        out[c] = static_cast<double>(__ldg(u.hi + o)) + static_cast<double>(__ldg(u.lo + o));
    }
}

__device__ __forceinline__ void load_hi_mx(const MixedState& u, const Geometry& g, int x, int y,
                                           float* out)
{
    const size_t k = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        out[c] = __ldg(u.hi + static_cast<size_t>(c) * g.plane + k);
    }
}

// FP64 wall fill from hi + lo of the neighbour (include/mhd/mask.hpp:100-146).
__device__ __forceinline__ void wall_fill_mx(const MixedState& u, const uint8_t* __restrict__ mask,
                                             const Geometry& g, int x, int y, double gm1,
                                             double* out)
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
        load_cons_mx(u, g, nx, ny, s);
        reflect_fill(s, k < 2 ? 0 : 1, gm1, out);
        return;
    }
    isolated_fill(gm1, out);
}

template <int TX, int TY, bool NI>
constexpr size_t stage_smem_bytes_mixed()
{
    using S = TileShape<TX, TY>;
    return sizeof(float) * (9 * S::NH + 9 * S::NFX + 9 * S::NFY + (NI ? 3 * S::NJ : 0));
}

// Primitive of one halo cell in FP32 with the FP64 pressure fallback.
__device__ __forceinline__ void halo_prim_mx(const MixedState& u, const Geometry& g, int sx,
                                             int sy, const double* filled, const Consts& k,
                                             float* w)
{
    float uf[9];
    if (filled != nullptr) {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            uf[c] = __double2float_rn(filled[c]);
        }
    } else {
        load_hi_mx(u, g, sx, sy, uf);
    }
    const float gm1 = static_cast<float>(k.gm1);
    cons_to_prim(uf, gm1, w);
    const float eint = w[4] * static_cast<float>(k.inv_gm1);
    if (!(eint * kCancelRatio >= uf[4])) {
        // Cancellation (or a non-finite value): recover p in FP64 from the full-precision state.
        double d[9];
        if (filled != nullptr) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                d[c] = filled[c];
            }
        } else {
            load_cons_mx(u, g, sx, sy, d);
        }
        const double inv_rho = 1.0 / d[0];
        const double ekin = 0.5 * (d[1] * d[1] + d[2] * d[2] + d[3] * d[3]) * inv_rho;
        const double emag = 0.5 * (d[5] * d[5] + d[6] * d[6] + d[7] * d[7]);
        w[4] = __double2float_rn(k.gm1 * (d[4] - ekin - emag));
    }
}

template <int L, bool NI, bool MASK, int STAGE, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 3) stage_kernel_mixed(const StageArgsMx a)
{
    using S = TileShape<TX, TY>;
    constexpr int HX = S::HX;
    const Ctrl* __restrict__ ctrl = a.ctrl;
    if (ctrl->finished != 0) {
        return;
    }
    extern __shared__ float smemf[];
    float* sW = smemf;
    float* sFx = sW + 9 * S::NH;
    float* sFy = sFx + 9 * S::NFX;
    float* sJ = sFy + 9 * S::NFY;

    const Geometry& g = a.geom;
    const Consts& k = a.k;
    const int x0 = blockIdx.x * TX;
    const int y0 = blockIdx.y * TY;
    const double dt = ctrl->dt;
    const double c_h64 = ctrl->c_h;
    const float c_h = static_cast<float>(c_h64);
    const float gamma = static_cast<float>(k.gamma);
    const float inv_gm1 = static_cast<float>(k.inv_gm1);

    for (int t = threadIdx.x; t < S::NH; t += NT) {
        const int lx = t % HX, ly = t / HX;
        const int gx = x0 - 2 + lx, gy = y0 - 2 + ly;
        const int sx = map_index(gx, g.nx, g.bc_x);
        const int sy = map_index(gy, g.ny, g.bc_y);
        const bool interior = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny;
        float w[9];
        if (MASK && a.walls && interior && is_solid(a.mask, g, sx, sy)) {
            double f[9];
            wall_fill_mx(a.uin, a.mask, g, sx, sy, k.gm1, f);
            halo_prim_mx(a.uin, g, sx, sy, f, k, w);
        } else {
            halo_prim_mx(a.uin, g, sx, sy, nullptr, k, w);
        }
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            sW[c * S::NH + t] = w[c];
        }
    }
    __syncthreads();

    if constexpr (NI) {
        const float inv_2dx = static_cast<float>(k.inv_2dx), inv_2dy = static_cast<float>(k.inv_2dy);
        for (int t = threadIdx.x; t < S::NJ; t += NT) {
            const int jx = t % S::JX + 1, jy = t / S::JX + 1;
            const int i = jy * HX + jx;
            const float* bx = sW + 5 * S::NH;
            const float* by = sW + 6 * S::NH;
            const float* bz = sW + 7 * S::NH;
            const float dbz_dy = (bz[i + HX] - bz[i - HX]) * inv_2dy;
            const float dbz_dx = (bz[i + 1] - bz[i - 1]) * inv_2dx;
            const float dby_dx = (by[i + 1] - by[i - 1]) * inv_2dx;
            const float dbx_dy = (bx[i + HX] - bx[i - HX]) * inv_2dy;
            sJ[0 * S::NJ + t] = dbz_dy;
            sJ[1 * S::NJ + t] = -dbz_dx;
            sJ[2 * S::NJ + t] = dby_dx - dbx_dy;
        }
        __syncthreads();
    }

    for (int t = threadIdx.x; t < S::NFX + S::NFY; t += NT) {
        const bool ydir = t >= S::NFX;
        const int tt = ydir ? t - S::NFX : t;
        const int w = ydir ? TX : TX + 1;
        const int fx = tt % w, fy = tt / w;
        const int base = (fy + 2) * HX + (fx + 2);
        const int stride = ydir ? HX : 1;
        const int pn = ydir ? 2 : 1, pt = ydir ? 1 : 2;
        const int bn = ydir ? 6 : 5, bt = ydir ? 5 : 6;
        PrimN<float> W[4];
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
        const FluxN<float> f = muscl_hll_face<L>(W[0], W[1], W[2], W[3], gamma, inv_gm1, c_h);
        float out[9];
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
            const int jr = (fy + 1) * S::JX + (fx + 1);
            const int jl = jr - (ydir ? S::JX : 1);
            const int il = base - stride;
            const float Jx = 0.5f * (sJ[jl] + sJ[jr]);
            const float Jy = 0.5f * (sJ[S::NJ + jl] + sJ[S::NJ + jr]);
            const float Jz = 0.5f * (sJ[2 * S::NJ + jl] + sJ[2 * S::NJ + jr]);
            const float Bx = 0.5f * (sW[5 * S::NH + il] + sW[5 * S::NH + base]);
            const float By = 0.5f * (sW[6 * S::NH + il] + sW[6 * S::NH + base]);
            const float Bz = 0.5f * (sW[7 * S::NH + il] + sW[7 * S::NH + base]);
            float Ex, Ey, Ez;
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
        float* dst = ydir ? (sFy + tt) : (sFx + tt);
        const int pstride = ydir ? S::NFY : S::NFX;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            dst[c * pstride] = out[c];
        }
    }
    __syncthreads();

    const float inv_dx = static_cast<float>(k.inv_dx), inv_dy = static_cast<float>(k.inv_dy);
    const double psi_damp = (c_h64 > 0.0 && k.glm_alpha > 0.0) ? (c_h64 * k.glm_alpha / k.h) : 0.0;
    float smax = 0.0f;
    for (int t = threadIdx.x; t < S::NC; t += NT) {
        const int cx = t % TX, cy = t / TX;
        const int gx = x0 + cx, gy = y0 + cy;
        if (gx >= g.nx || gy >= g.ny) {
            continue;
        }
        const bool solid = MASK && is_solid(a.mask, g, gx, gy);
        const int fxi = cy * (TX + 1) + cx;
        const int fyi = cy * TX + cx;
        double Lc[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const float l = -(sFx[c * S::NFX + fxi + 1] - sFx[c * S::NFX + fxi]) * inv_dx -
                            (sFy[c * S::NFY + fyi + TX] - sFy[c * S::NFY + fyi]) * inv_dy;
            Lc[c] = static_cast<double>(l);
        }
        const size_t o = static_cast<size_t>(gy) * g.pitch + gx;
        double uin[9];
        if (solid && a.walls) {
            wall_fill_mx(a.uin, a.mask, g, gx, gy, k.gm1, uin);
        } else {
            load_cons_mx(a.uin, g, gx, gy, uin);
        }
        if (psi_damp != 0.0) {
            Lc[8] -= psi_damp * uin[8];
        }
        if (solid) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                Lc[c] = 0.0;
            }
        }
        if constexpr (STAGE == 1) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                split_store(a.out, static_cast<size_t>(c) * g.plane + o, uin[c] + dt * Lc[c]);
            }
        } else {
            double un[9];
            if (solid) {
                load_cons_mx(a.uin, g, gx, gy, un); // stored U* of a solid cell = filled U^n
            } else {
                load_cons_mx(a.out, g, gx, gy, un);
            }
            const double half_dt = 0.5 * dt;
            float rf[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                const double r = 0.5 * (un[c] + uin[c]) + half_dt * Lc[c];
                split_store(a.out, static_cast<size_t>(c) * g.plane + o, r);
                rf[c] = __double2float_rn(r);
            }
            if (!solid) {
                smax = vmax(smax, cell_max_signal_speed(rf[0], rf[1], rf[2], rf[3], rf[4], rf[5],
                                                        rf[6], rf[7], gamma));
            }
        }
    }
    if constexpr (STAGE == 2) {
        reduce_signal_speed_and_finish(static_cast<double>(smax), a.ctrl, a.k,
                                       gridDim.x * gridDim.y, true);
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) cfl_init_kernel_mixed(const MixedState u,
                                                           const uint8_t* __restrict__ mask,
                                                           Geometry g, Consts k, Ctrl* ctrl,
                                                           int has_mask)
{
    float smax = 0.0f;
    const float gamma = static_cast<float>(k.gamma);
    const long long ncell = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; c < ncell;
         c += static_cast<long long>(gridDim.x) * NT) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        if (has_mask && is_solid(mask, g, x, y)) {
            continue;
        }
        double r[9];
        load_cons_mx(u, g, x, y, r);
        float rf[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            rf[q] = __double2float_rn(r[q]);
        }
        smax = vmax(smax, cell_max_signal_speed(rf[0], rf[1], rf[2], rf[3], rf[4], rf[5], rf[6],
                                                rf[7], gamma));
    }
    reduce_signal_speed_and_finish(static_cast<double>(smax), ctrl, k, gridDim.x, false);
}

__global__ void unpack_mixed(const double* __restrict__ stg, MixedState u, Geometry g, int ng,
                             int nxt, size_t ntot)
{
    const long long n = static_cast<long long>(g.nx) * g.ny;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(c % g.nx), y = static_cast<int>(c / g.nx);
        const size_t s = static_cast<size_t>(y + ng) * nxt + (x + ng);
        const size_t d = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            split_store(u, q * g.plane + d, stg[q * ntot + s]);
        }
    }
}

__global__ void pack_mixed(const MixedState u, const uint8_t* __restrict__ mask,
                           double* __restrict__ stg, Geometry g, int ng, int nxt, int nyt,
                           size_t ntot, int fill, double gm1)
{
    const long long n = static_cast<long long>(nxt) * nyt;
    for (long long c = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; c < n;
         c += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(c % nxt), j = static_cast<int>(c / nxt);
        const int gx = i - ng, gy = j - ng;
        const int sx = map_index(gx, g.nx, g.bc_x), sy = map_index(gy, g.ny, g.bc_y);
        const bool interior = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny;
        double v[9];
        if (fill && interior && is_solid(mask, g, sx, sy)) {
            wall_fill_mx(u, mask, g, sx, sy, gm1, v);
        } else {
            load_cons_mx(u, g, sx, sy, v);
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            stg[q * ntot + static_cast<size_t>(c)] = v[q];
        }
    }
}

using StageFnMx = void (*)(StageArgsMx);

template <int L, bool NI, bool MASK>
void stage_pair_mixed(StageFnMx& s1, StageFnMx& s2)
{
    s1 = stage_kernel_mixed<L, NI, MASK, 1, 32, 16, 256>;
    s2 = stage_kernel_mixed<L, NI, MASK, 2, 32, 16, 256>;
}

inline void select_mixed(int lim, bool ni, bool mask, StageFnMx& s1, StageFnMx& s2)
{
#define MHDB_SELM(LL)                                                                              \
    if (ni) {                                                                                      \
        if (mask) stage_pair_mixed<LL, true, true>(s1, s2);                                        \
        else stage_pair_mixed<LL, true, false>(s1, s2);                                            \
    } else {                                                                                       \
        if (mask) stage_pair_mixed<LL, false, true>(s1, s2);                                       \
        else stage_pair_mixed<LL, false, false>(s1, s2);                                           \
    }
    if (lim == kMinmod) {
        MHDB_SELM(kMinmod)
    } else if (lim == kMC) {
        MHDB_SELM(kMC)
    } else {
        MHDB_SELM(kVanLeer)
    }
#undef MHDB_SELM
}

} // namespace mhdb
