// FP32-mixed form: the state is carried as a compensated pair of FP32 planes, value = hi + lo
// with |lo| <= ulp(hi)/2 (~48 significant bits). Precision rules:
//   * reconstruction, HLL fluxes, non-ideal terms and the divergence run in FP32 on hi;
//   * the stage update is done in FP64 on hi + lo and split again, so the RK2 combination
//     loses no bits;
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

struct PolicyMixed {
    using T = float;
    using Args = StageArgsMx;

    static __device__ __forceinline__ void halo_prim(const MixedState& u, const Geometry& g,
                                                     int x, int y, const Consts& k, float* w)
    {
        const size_t o = static_cast<size_t>(y) * g.pitch + x;
        float uf[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            uf[c] = __ldg(u.hi + static_cast<size_t>(c) * g.plane + o);
        }
        cons_to_prim(uf, static_cast<float>(k.gm1), w);
        if (cancels(w, uf, k)) {
            double d[9];
            load_cons_mx(u, g, x, y, d);
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
    static __device__ __forceinline__ void wall_fill(const MixedState& u, const uint8_t* mask,
                                                     const Geometry& g, int x, int y, double gm1,
                                                     double* out)
    {
        wall_fill_mx(u, mask, g, x, y, gm1, out);
    }
    static __device__ __forceinline__ void load_full(const MixedState& u, const Geometry& g,
                                                     int x, int y, double* out)
    {
        load_cons_mx(u, g, x, y, out);
    }
    static __device__ __forceinline__ void store(const MixedState& u, const Geometry& g, size_t o,
                                                 const double* v)
    {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            split_store(u, static_cast<size_t>(c) * g.plane + o, v[c]);
        }
    }
    static __device__ __forceinline__ double signal_speed(const double* r, const Consts& k)
    {
        float rf[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            rf[c] = __double2float_rn(r[c]);
        }
        return static_cast<double>(cell_max_signal_speed(rf[0], rf[1], rf[2], rf[3], rf[4], rf[5],
                                                         rf[6], rf[7],
                                                         static_cast<float>(k.gamma)));
    }
};

template <int NT>
__global__ void __launch_bounds__(NT) cfl_init_kernel_mixed(const MixedState u,
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
        load_cons_mx(u, g, x, y, r);
        smax = vmax(smax, PolicyMixed::signal_speed(r, k));
    }
    reduce_signal_speed_and_finish(smax, ctrl, k, gridDim.x, false);
}

} // namespace mhdb
