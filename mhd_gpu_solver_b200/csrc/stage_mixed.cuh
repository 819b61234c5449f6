// FP32-mixed form: the state is carried as a compensated pair of FP32 planes, value = hi + lo
// with |lo| <= ulp(hi)/2 (~48 significant bits). Precision rules:
//   * reconstruction, HLL fluxes, non-ideal terms and the divergence run in FP32 on hi;
//   * the stage updates U* = U^n + dt L (include/mhd/field_ops.hpp:51) and
//     U^{n+1} = (U^n + U*)/2 + (dt/2) L (field_ops.hpp:61) add an FP32 stage increment (dt L,
//     resp. (U* - U^n)/2 + (dt/2) L) to the (hi, lo) pair of U^n with error-free two-sums, so
//     the RK2 combination loses no bits of the state (only the increment carries FP32 rounding,
//     relative to its own size);
//   * pressure recovery p = (gamma-1)(E - rho v^2/2 - B^2/2) is redone in FP64 from hi + lo in
//     cells where the FP32 subtraction cancels (p/(gamma-1) < E / kCancelRatio: low beta or high
//     Mach) or is not finite;
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

__device__ __forceinline__ void wall_fill_mx(const MixedState& u, const uint8_t* __restrict__ mask,
                                             const Geometry& g, int x, int y, double gm1,
                                             double* out)
{
    wall_fill_any([&](int i, int j, double* s) { load_cons_mx(u, g, i, j, s); }, mask, g, x, y,
                  gm1, out);
}

// FP64 pressure from a full-precision conserved state (the reference's primitive formula,
// include/mhd/kernels/cpu_rows.hpp:145-152).
__device__ __forceinline__ float pressure_f64(const double* d, double gm1)
{
    const double inv_rho = 1.0 / d[0];
    const double ekin = 0.5 * (d[1] * d[1] + d[2] * d[2] + d[3] * d[3]) * inv_rho;
    const double emag = 0.5 * (d[5] * d[5] + d[6] * d[6] + d[7] * d[7]);
    return __double2float_rn(gm1 * (d[4] - ekin - emag));
}

__device__ __forceinline__ bool cancels(const float* w, const float* uf, const Consts& k)
{
    const float eint = w[4] * static_cast<float>(k.inv_gm1);
    return !(eint * kCancelRatio >= uf[4]);
}

// Error-free transformation a + b = s + e (Knuth's two-sum; six FP32 additions, none of them
// contractible).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Renormalise s + t (|t| small against s) into a (hi, lo) pair (Dekker's fast two-sum).
__device__ __forceinline__ void fast_two_sum(float s, float t, float& h, float& l)
{
    h = s + t;
    l = t - (h - s);
}

struct PolicyMixed {
    using T = float;
    using Args = StageArgsMx;
    static constexpr int kLayout = 0; // MarchTmaLayout of the stored form
    struct Raw {
        float v[9];
    };
    // Full-precision value of the stage input at (x, y): hi + lo.
    template <int STAGE, bool MASK>
    static __device__ __forceinline__ void full(const Args& a, const Geometry& g, int x, int y,
                                                double* out)
    {
        load_cons_mx(a.uin, g, x, y, out);
    }

    static __device__ __forceinline__ void load_raw(const Args& a, const Geometry& g, int x, int y,
                                                    Raw& r)
    {
        const size_t o = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            r.v[c] = __ldg(a.uin.hi + static_cast<size_t>(c) * g.plane + o);
        }
    }
    template <int STAGE, bool MASK>
    static __device__ __forceinline__ void raw_prim(const Args& a, const Geometry& g, int x, int y,
                                                    const Raw& r, const Consts& k, float* w)
    {
        cons_to_prim(r.v, static_cast<float>(k.gm1), w);
        if (cancels(w, r.v, k)) {
            double d[9];
            full<STAGE, MASK>(a, g, x, y, d);
            w[4] = pressure_f64(d, k.gm1);
        }
    }
    static __device__ __forceinline__ void prim_of(const double* f, const Consts& k, float* w)
    {
        float uf[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            uf[c] = __double2float_rn(f[c]);
        }
        cons_to_prim(uf, static_cast<float>(k.gm1), w);
        if (cancels(w, uf, k)) {
            w[4] = pressure_f64(f, k.gm1);
        }
    }
    // FP64 wall fill of a solid cell from its fluid neighbours' full-precision stage input.
    template <int STAGE, bool MASK>
    static __device__ __forceinline__ void wall_fill(const Args& a, const Geometry& g, int x,
                                                     int y, double gm1, double* out)
    {
        wall_fill_mx(a.uin, a.mask, g, x, y, gm1, out);
    }
    static __device__ __forceinline__ float signal_speed_f(const float* r, const Consts& k)
    {
        return cell_max_signal_speed(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7],
                                     static_cast<float>(k.gamma));
    }
    static __device__ __forceinline__ double signal_speed(const double* r, const Consts& k)
    {
        float rf[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            rf[c] = __double2float_rn(r[c]);
        }
        return static_cast<double>(signal_speed_f(rf, k));
    }

    template <int STAGE, bool MASK>
    static __device__ __forceinline__ void update(const Args& a, const Geometry& g, int gx, int gy,
                                                  bool solid, float (&L)[9], float psi_in,
                                                  double psi_damp, double dt, const Consts& k,
                                                  double& smax)
    {
        if (psi_damp != 0.0) {
            L[8] -= static_cast<float>(psi_damp) * psi_in; // include/mhd/rhs.hpp:219-225
        }
        if (solid) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                L[c] = 0.0f;
            }
        }
        const size_t o = static_cast<size_t>(gy) * g.pitch + gx;
        if (MASK && solid && a.walls) {
            // Rare path in FP64: stage 1 stores fill(U^n); stage 2 stores
            // (U*_stored + fill(U*)) / 2, where the stored U* of a solid cell is fill(U^n).
            double f[9];
            wall_fill<STAGE, MASK>(a, g, gx, gy, k.gm1, f);
            if constexpr (STAGE == 2) {
                double un[9];
                load_cons_mx(a.uin, g, gx, gy, un);
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    f[c] = 0.5 * (un[c] + f[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                split_store(a.out, static_cast<size_t>(c) * g.plane + o, f[c]);
            }
            return;
        }
        const float* __restrict__ ih = a.uin.hi + o;
        const float* __restrict__ il = a.uin.lo + o;
        const float* __restrict__ oh = a.out.hi + o;
        const float* __restrict__ ol = a.out.lo + o;
        const size_t pl = g.plane;
        update_ops<STAGE>(a, g, gx, gy, solid, L, dt, k, smax, [&](int i) {
            const size_t q = static_cast<size_t>(i % 9) * pl;
            return i < 9 ? __ldg(ih + q) : (i < 18 ? __ldg(il + q) : (i < 27 ? oh[q] : ol[q]));
        });
    }

    // The stage update of one cell from its own-cell operands op(i): plane i % 9 of the input hi
    // (i < 9) and lo (i < 18) planes and, in stage 2, of the U^n hi (i < 27) and lo (i < 36)
    // planes, which the stage overwrites; all are read before any store.
    template <int STAGE, class Op>
    static __device__ __forceinline__ void update_ops(const Args& a, const Geometry& g, int gx,
                                                      int gy, bool solid, const float (&L)[9],
                                                      double dt, const Consts& k, double& smax,
                                                      const Op& op)
    {
        // Plane bases are the same for every thread; the cell offset within a plane fits 32 bits
        // (it is below the plane size), so each store address is one wide multiply-add.
        const uint32_t o = static_cast<uint32_t>(gy) * static_cast<uint32_t>(g.pitch) +
                           static_cast<uint32_t>(gx);
        const size_t pl = g.plane;
        update_ops<STAGE>(a, solid || !reduce_row(g, gy), L, dt, k, smax, op,
                          [&](int c, float h, float l) {
            (a.out.hi + static_cast<size_t>(c) * pl)[o] = h;
            (a.out.lo + static_cast<size_t>(c) * pl)[o] = l;
        });
    }
    // The same with the results handed to st(c, hi, lo) instead of stored to the output planes;
    // no_speed (a solid cell, or a row outside the reduction rows) keeps the cell out of the
    // signal-speed max.
    template <int STAGE, class Op, class St>
    static __device__ __forceinline__ void update_ops(const Args& a, bool no_speed,
                                                      const float (&L)[9], double dt,
                                                      const Consts& k, double& smax, const Op& op,
                                                      const St& st)
    {
        const float dtf = static_cast<float>(dt);
        float xh[9], xl[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            xh[c] = op(c);
            xl[c] = op(9 + c);
        }
        if constexpr (STAGE == 1) {
            // U* = U^n + dt L
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                float s, e, h, l;
                two_sum(xh[c], __fmul_rn(dtf, L[c]), s, e); // product rounded first: exact two-sum
                fast_two_sum(s, xl[c] + e, h, l);
                st(c, h, l);
            }
        } else {
            // U^{n+1} = (U^n + U*)/2 + (dt/2) L = U^n + d with d = (U* - U^n)/2 + (dt/2) L,
            // U^n read from the output buffer (own cell). d is a stage increment: it is formed
            // in FP32 (its rounding is relative to d, like that of dt L in stage 1) and added to
            // the (hi, lo) pair of U^n exactly.
            float nh[9], nl[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                nh[c] = op(18 + c);
                nl[c] = op(27 + c);
            }
            const float half_dt = 0.5f * dtf;
            float rf[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                float s, e, h, l;
                const float d = __fmaf_rn(half_dt, L[c],
                                          __fmul_rn(0.5f, __fadd_rn(__fsub_rn(xh[c], nh[c]),
                                                                    __fsub_rn(xl[c], nl[c]))));
                two_sum(nh[c], d, s, e);
                fast_two_sum(s, nl[c] + e, h, l);
                st(c, h, l);
                rf[c] = h;
            }
            if (!no_speed) {
                smax = vmax(smax, static_cast<double>(signal_speed_f(rf, k)));
            }
        }
    }
};

template <int NT>
__global__ void __launch_bounds__(NT) cfl_init_kernel_mixed(const MixedState u,
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
        load_cons_mx(u, g, x, y, r);
        smax = vmax(smax, PolicyMixed::signal_speed(r, k));
    }
    reduce_signal_speed_and_finish(smax, ctrl, k, gridDim.x, false);
}

} // namespace mhdb
