// FP32-mixed form with the stage increment stored instead of U* (the increment form).
//
// Stage 1 of the FP32-mixed form adds the FP32 increment delta = fl(dt L) to the (hi, lo) pair
// of U^n exactly (stage_mixed.cuh), so U* - U^n = delta. This form stores delta itself (9 FP32
// planes) instead of U*'s 18 hi and lo planes, and stage 2 rebuilds what it needs:
//   * the stencil of stage 2 reads U*'s hi values as fl(hi(U^n) + delta) (FP32 inputs of the
//     FP32 fluxes, as in the stored form), the FP64 pressure recovery (hi + lo)(U^n) + delta;
//   * the update U^{n+1} = U^n + d with d = delta/2 + (dt/2) L (include/mhd/field_ops.hpp:61:
//     (U^n + U*)/2 + (dt/2) L = U^n + (U* - U^n)/2 + (dt/2) L) adds d to the (hi, lo) pair of
//     U^n with error-free two-sums, as the stored form does.
// U* itself is exact here (the stored form rounds its lo word once), so the state loses no bits
// in either stage. Stage 1 reads only U^n's hi planes (the lo planes only where the FP64 pressure
// recovery needs them) and writes 9 planes: 72 B per cell instead of 144; stage 2 reads U^n and
// delta and writes U^{n+1}: 180 B instead of 216. Stage 2's stencil reads U^n of neighbouring
// cells, so U^{n+1} goes to the other state buffer (the two buffers alternate step by step).
// With a mask, a solid cell's stored U* is the wall fill of U^n, so stage 1 stores the increment
// fill(U^n) - U^n rounded to FP32 (the stored form rounds that fill to its FP32 primitives too);
// the FP64 wall fill reads U^n, or U^n + delta in stage 2, from global memory.
#pragma once

#include "stage_mixed.cuh"

namespace mhdb {

struct StageArgsDelta {
    MixedState un;       // U^n: read by both stages
    MixedState out;      // U^{n+1}: written by stage 2 (the other state buffer)
    float* delta;        // 9 planes: fl(dt L) of stage 1 (U* = U^n + delta exactly)
    const uint8_t* mask; // padded fluid mask or nullptr
    Ctrl* ctrl;
    Geometry geom;
    Consts k;
    int walls;
};

// LAYOUT: MarchTmaLayout kind of the TMA strip march (1: own cells' delta through the own
// stream; 2: through the halo stream, kept in a ring per lane).
template <int STAGE, int LAYOUT = 1>
struct PolicyDelta {
    using T = float;
    using Args = StageArgsDelta;
    static constexpr int kLayout = LAYOUT;
    struct Raw {
        float v[9];
    };
    // Full-precision stage input at (x, y): U^n, or U^n + delta in stage 2.
    static __device__ __forceinline__ void full(const Args& a, const Geometry& g, int x, int y,
                                                double* out)
    {
        load_cons_mx(a.un, g, x, y, out);
        if constexpr (STAGE == 2) {
            const size_t k = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                out[c] += static_cast<double>(__ldg(a.delta + static_cast<size_t>(c) * g.plane + k));
            }
        }
    }
    // hi values of the stage input: hi(U^n), or fl(hi(U^n) + delta) in stage 2.
    static __device__ __forceinline__ void load_raw(const Args& a, const Geometry& g, int x, int y,
                                                    Raw& r)
    {
        const size_t o = static_cast<size_t>(y) * g.pitch + x;
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            r.v[c] = __ldg(a.un.hi + static_cast<size_t>(c) * g.plane + o);
            if constexpr (STAGE == 2) {
                r.v[c] = __fadd_rn(r.v[c], __ldg(a.delta + static_cast<size_t>(c) * g.plane + o));
            }
        }
    }
    template <int S, bool MASK>
    static __device__ __forceinline__ void raw_prim(const Args& a, const Geometry& g, int x, int y,
                                                    const Raw& r, const Consts& k, float* w)
    {
        cons_to_prim(r.v, static_cast<float>(k.gm1), w);
        if (cancels(w, r.v, k)) {
            double d[9];
            full(a, g, x, y, d);
            w[4] = pressure_f64(d, k.gm1);
        }
    }
    static __device__ __forceinline__ float signal_speed_f(const float* r, const Consts& k)
    {
        return PolicyMixed::signal_speed_f(r, k);
    }
    static __device__ __forceinline__ void prim_of(const double* f, const Consts& k, float* w)
    {
        PolicyMixed::prim_of(f, k, w);
    }
    // FP64 wall fill of a solid cell from its fluid neighbours' full-precision stage input.
    template <int S, bool MASK>
    static __device__ __forceinline__ void wall_fill(const Args& a, const Geometry& g, int x,
                                                     int y, double gm1, double* out)
    {
        wall_fill_any([&](int i, int j, double* s) { full(a, g, i, j, s); }, a.mask, g, x, y,
                      gm1, out);
    }
    // Stage update of one cell. Stage 1 stores delta = fl(dt L). Stage 2 reads its own-cell
    // operands op(i): delta (i < 9), hi(U^n) (i < 18) and lo(U^n) (i < 27), and stores U^{n+1}.
    template <int S, class Op>
    static __device__ __forceinline__ void update_ops(const Args& a, const Geometry& g, int gx,
                                                      int gy, bool solid, const float (&L)[9],
                                                      double dt, const Consts& k, double& smax,
                                                      const Op& op)
    {
        const uint32_t o = static_cast<uint32_t>(gy) * static_cast<uint32_t>(g.pitch) +
                           static_cast<uint32_t>(gx);
        const size_t pl = g.plane;
        const float dtf = static_cast<float>(dt);
        if constexpr (STAGE == 1) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                (a.delta + static_cast<size_t>(c) * pl)[o] = __fmul_rn(dtf, L[c]);
            }
        } else {
            const float half_dt = 0.5f * dtf;
            float rf[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                const float dl = op(c), nh = op(9 + c), nl = op(18 + c);
                const float d = __fmaf_rn(half_dt, L[c], __fmul_rn(0.5f, dl));
                float s, e, h, l;
                two_sum(nh, d, s, e);
                fast_two_sum(s, nl + e, h, l);
                (a.out.hi + static_cast<size_t>(c) * pl)[o] = h;
                (a.out.lo + static_cast<size_t>(c) * pl)[o] = l;
                rf[c] = h;
            }
            if (!solid && reduce_row(g, gy)) {
                smax = vmax(smax, static_cast<double>(signal_speed_f(rf, k)));
            }
        }
    }
};

} // namespace mhdb
