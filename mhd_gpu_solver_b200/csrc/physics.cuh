// Point-wise GLM-MHD numerics for the sm_100a stage kernels.
//
// Written for this project from the reference's numerical method; each function names the
// reference file:line whose arithmetic (operation order included) it follows, so the FP64 form
// agrees with the reference CPU path to round-off. All functions are templated on the
// arithmetic type T (double for the plain form, float for the FP32-mixed form).
#pragma once

#include <cstdint>

namespace mhdb {

enum LimiterKind : int { kMinmod = 0, kMC = 1, kVanLeer = 2 };

// Rotated frame: n = face normal, t = in-plane tangential (x-faces: n=x, t=y; y-faces: n=y,
// t=x); include/mhd/kernels/muscl_hll.hpp:11-13,23-31.
template <class T>
struct PrimN {
    T rho, vn, vt, vz, p, bn, bt, bz, psi;
};

template <class T>
struct FluxN {
    T rho, mn, mt, mz, e, bn, bt, bz, psi;
};

// Reciprocal and square root. FP64: IEEE division and sqrt, as the reference computes them.
// FP32 (the FP32-mixed form): the hardware approximations rcp.approx.ftz / sqrt.approx.ftz (PTX
// ISA; about 1 ulp), used only where the operand is a positive normal number or the result is
// discarded by a select (inverse densities, 1/(sR - sL) with sR - sL >= 2 c_h, |B|, the van
// Leer denominator a + b with ab > 0, and the non-negative fast-speed discriminants).
template <class T>
__device__ __forceinline__ T fast_rcp(T x)
{
    return T(1) / x;
}
template <>
__device__ __forceinline__ float fast_rcp<float>(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <class T>
__device__ __forceinline__ T fast_sqrt(T x)
{
    return sqrt(x);
}
template <>
__device__ __forceinline__ float fast_sqrt<float>(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// mhd::simd scalar min/max (include/mhd/simd.hpp:40-47): the first operand wins ties and
// NaN comparisons, exactly as (b < a) ? b : a.
template <class T>
__device__ __forceinline__ T vmin(T a, T b)
{
    return (b < a) ? b : a;
}
template <class T>
__device__ __forceinline__ T vmax(T a, T b)
{
    return (a < b) ? b : a;
}
// FP32 (the FP32-mixed form): the single-instruction IEEE minNum/maxNum, which agree with the
// reference's selection for every pair of numbers and differ only in which operand a NaN yields.
template <>
__device__ __forceinline__ float vmin<float>(float a, float b)
{
    return fminf(a, b);
}
template <>
__device__ __forceinline__ float vmax<float>(float a, float b)
{
    return fmaxf(a, b);
}

template <class T>
__device__ __forceinline__ T tabs(T a)
{
    return a < T(0) ? -a : a;
}

// include/mhd/kernels/muscl_hll.hpp:33-38
template <class T>
__device__ __forceinline__ T minmod(T a, T b)
{
    return (a * b <= T(0)) ? T(0) : ((fabs(a) < fabs(b)) ? a : b);
}

// include/mhd/kernels/muscl_hll.hpp:41-47
template <class T>
__device__ __forceinline__ T mc_limiter(T a, T b)
{
    return minmod(T(0.5) * (a + b), minmod(T(2) * a, T(2) * b));
}

// van Leer (1974) harmonic limiter 2ab/(a+b) for same-sign slopes, else 0. The reference has
// no van Leer limiter (include/mhd/mhd_types.hpp:44); this is the published formula. FP64 takes
// the quotient as 2ab * (1 / (a + b)): within an ulp or two of the division and measured 8 %
// faster for the whole FP64 step at 4096^2 (nvcc's reciprocal sequence is shorter than its
// division's).
template <class T>
__device__ __forceinline__ T vanleer_limiter(T a, T b)
{
    const T p = a * b;
    return (p <= T(0)) ? T(0) : (T(2) * p) * (T(1) / (a + b));
}
// FP32: 2ab * rcp(a + b) without a branch. When ab > 0 after rounding, a and b share their sign
// and max(|a|, |b|) >= 2^-74.5, so a + b is a normal number and the approximate reciprocal is
// within its stated error; otherwise the select returns 0.
template <>
__device__ __forceinline__ float vanleer_limiter<float>(float a, float b)
{
    const float p = a * b;
    const float q = (p + p) * fast_rcp(a + b);
    return (p <= 0.0f) ? 0.0f : q;
}

template <int L, class T>
__device__ __forceinline__ T limit_slope(T a, T b)
{
    if constexpr (L == kMinmod) {
        return minmod(a, b);
    } else if constexpr (L == kMC) {
        return mc_limiter(a, b);
    } else {
        return vanleer_limiter(a, b);
    }
}

// Half of the limited slope, lim(a, b) / 2, computed directly (halving is exact, so this is the
// same value as 0.5 * limit_slope): van Leer ab / (a + b) (as ab * (1 / (a + b)), as above), MC
// minmod((a + b) / 4, minmod(a, b)), minmod minmod(a / 2, b / 2).
template <int L, class T>
__device__ __forceinline__ T limit_half_slope(T a, T b)
{
    if constexpr (L == kMinmod) {
        return minmod(T(0.5) * a, T(0.5) * b);
    } else if constexpr (L == kMC) {
        return minmod(T(0.25) * (a + b), minmod(a, b));
    } else if constexpr (sizeof(T) == 4) {
        const float p = a * b;
        const float q = p * fast_rcp(a + b);
        return (p <= 0.0f) ? 0.0f : q;
    } else {
        const T p = a * b;
        return (p <= T(0)) ? T(0) : p * (T(1) / (a + b));
    }
}

// 1/x for a normal or infinite FP64 x without a division: the hardware approximation
// rcp.approx.ftz.f64 refined by two Newton-Raphson steps e = 1 - x y, y += y e (the classical
// iteration, each step squaring the relative error), so within a few ulp of 1/x; 0 for |x| of
// 2^1022 and above. Used only where a product of slopes left the normal range.
__device__ __forceinline__ double newton_rcp(double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// limit_half_slope of nine components (a[c], b[c]). FP64 van Leer takes one division for all
// nine (simultaneous inversion over a two-level product tree: groups g_j = s_3j s_3j+1 s_3j+2,
// q = 1 / (g_0 g_1 g_2), 1/g_2 = (g_0 g_1) q, 1/g_0 = g_1 (g_2 q), 1/g_1 = g_0 (g_2 q), then the
// same within each group; s = a + b if ab > 0 and 1 where the slope is 0 anyway), each reciprocal
// within 6 ulp of 1/s. If the product leaves the normal range, every component takes its own
// reciprocal (newton_rcp). Every other limiter and precision: component by component.
template <int L, class T>
__device__ __forceinline__ void limit_half_slopes(const T (&a)[9], const T (&b)[9], T (&out)[9])
{
    if constexpr (L == kVanLeer && sizeof(T) == 8) {
        T p[9], s[9], r[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            p[c] = a[c] * b[c];
            s[c] = (p[c] > T(0)) ? a[c] + b[c] : T(1);
        }
        T p01[3], g[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            p01[j] = s[3 * j] * s[3 * j + 1];
            g[j] = p01[j] * s[3 * j + 2];
        }
        const T g01 = g[0] * g[1];
        const T prod = g01 * g[2];
        const T mag = fabs(prod);
        if (mag >= 2.2250738585072014e-308 && mag <= 1.7976931348623157e308) {
            const T inv = T(1) / prod;
            T ig[3];
            ig[2] = g01 * inv;
            const T i01 = g[2] * inv;
            ig[0] = g[1] * i01;
            ig[1] = g[0] * i01;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                r[3 * j + 2] = p01[j] * ig[j];
                const T t = s[3 * j + 2] * ig[j];
                r[3 * j] = s[3 * j + 1] * t;
                r[3 * j + 1] = s[3 * j] * t;
            }
        } else {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                r[c] = newton_rcp(s[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            out[c] = (p[c] <= T(0)) ? T(0) : p[c] * r[c];
        }
    } else {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            out[c] = limit_half_slope<L>(a[c], b[c]);
        }
    }
}

// Face i-1/2 from cells (i-2, i-1, i, i+1); include/mhd/kernels/muscl_hll.hpp:59-68.
template <int L, class T>
__device__ __forceinline__ void reconstruct(T wmm, T wm, T w0, T wp, T& left, T& right)
{
    const T dm = limit_slope<L>(wm - wmm, w0 - wm);
    const T d0 = limit_slope<L>(w0 - wm, wp - w0);
    left = wm + T(0.5) * dm;
    right = w0 - T(0.5) * d0;
}

// Fast magnetosonic speed along n; include/mhd/kernels/muscl_hll.hpp:70-87.
template <class T>
__device__ __forceinline__ T fast_speed_n_inv(const PrimN<T>& W, T inv_rho, T gamma)
{
    const T cs2 = gamma * W.p * inv_rho;
    const T bn2 = W.bn * W.bn;
    const T b2 = bn2 + W.bt * W.bt + W.bz * W.bz;
    const T va2 = b2 * inv_rho;
    const T van2 = bn2 * inv_rho;
    const T sum = cs2 + va2;
    const T disc = vmax(sum * sum - T(4) * cs2 * van2, T(0));
    const T cf2 = T(0.5) * (sum + fast_sqrt(disc));
    return fast_sqrt(vmax(cf2, T(0)));
}
template <class T>
__device__ __forceinline__ T fast_speed_n(const PrimN<T>& W, T gamma)
{
    return fast_speed_n_inv(W, fast_rcp(W.rho), gamma);
}

// Conserved state and GLM-MHD flux along n; include/mhd/kernels/muscl_hll.hpp:89-124.
template <class T>
__device__ __forceinline__ void conserved_and_flux(const PrimN<T>& W, T inv_gm1, T ch2,
                                                   FluxN<T>& U, FluxN<T>& F)
{
    const T mn = W.rho * W.vn;
    const T mt = W.rho * W.vt;
    const T mz = W.rho * W.vz;
    const T v2 = W.vn * W.vn + W.vt * W.vt + W.vz * W.vz;
    const T b2 = W.bn * W.bn + W.bt * W.bt + W.bz * W.bz;
    const T pmag = T(0.5) * b2;
    const T energy = W.p * inv_gm1 + T(0.5) * W.rho * v2 + pmag;
    const T pstar = W.p + pmag;
    const T vb = W.vn * W.bn + W.vt * W.bt + W.vz * W.bz;

    U.rho = W.rho;
    U.mn = mn;
    U.mt = mt;
    U.mz = mz;
    U.e = energy;
    U.bn = W.bn;
    U.bt = W.bt;
    U.bz = W.bz;
    U.psi = W.psi;

    F.rho = mn;
    F.mn = mn * W.vn + pstar - W.bn * W.bn;
    F.mt = mn * W.vt - W.bn * W.bt;
    F.mz = mn * W.vz - W.bn * W.bz;
    F.e = (energy + pstar) * W.vn - W.bn * vb + W.psi * W.bn;
    F.bn = W.psi;
    F.bt = W.vn * W.bt - W.vt * W.bn;
    F.bz = W.vn * W.bz - W.vz * W.bn;
    F.psi = ch2 * W.bn;
}

// HLL flux with Dedner GLM wave-speed bounds (-c_h, +c_h) from the two face states, with the
// upwind and degenerate (|sR - sL| < 1e-14) branches; include/mhd/kernels/muscl_hll.hpp:170-208.
template <class T>
__device__ __forceinline__ FluxN<T> hll_flux(const PrimN<T>& WL, const PrimN<T>& WR, T gamma,
                                             T inv_gm1, T c_h)
{
    const T cfL = fast_speed_n(WL, gamma);
    const T cfR = fast_speed_n(WR, gamma);
    const T sL = vmin(vmin(WL.vn - cfL, WR.vn - cfR), -c_h);
    const T sR = vmax(vmax(WL.vn + cfL, WR.vn + cfR), c_h);

    const T ch2 = c_h * c_h;
    FluxN<T> UL, UR, FL, FR;
    conserved_and_flux(WL, inv_gm1, ch2, UL, FL);
    conserved_and_flux(WR, inv_gm1, ch2, UR, FR);

    const T denom = sR - sL;
    const T inv_denom = fast_rcp(denom);
    const T sLsR = sL * sR;
    const bool use_left = sL >= T(0);
    const bool use_right = sR <= T(0);
    const bool degenerate = fabs(denom) < T(1.0e-14);

    // FP64: the reference's operation order. FP32: the three weights folded into 1/(sR - sL)
    // once per face, four operations per component.
    const T wR = sR * inv_denom, wL = sL * inv_denom, wLR = sLsR * inv_denom;
    auto hll = [&](T fl, T fr, T ul, T ur) {
        if constexpr (sizeof(T) == 4) {
            return wR * fl - wL * fr + wLR * (ur - ul);
        } else {
            return (sR * fl - sL * fr + sLsR * (ur - ul)) * inv_denom;
        }
    };
    auto combine = [&](T fl, T fr, T ul, T ur) {
        const T mid = degenerate ? T(0.5) * (fl + fr) : hll(fl, fr, ul, ur);
        return use_left ? fl : (use_right ? fr : mid);
    };

    FluxN<T> F;
    if (c_h >= T(1.0e-14)) {
        // sL <= -c_h < 0 < c_h <= sR (or NaN) and sR - sL >= 2 c_h > 1e-14: neither upwind
        // branch nor the degenerate one can be taken, so the selection below returns the HLL
        // average for every component (NaN included). c_h is the same for every face of a
        // launch, so this branch does not diverge.
        F.rho = hll(FL.rho, FR.rho, UL.rho, UR.rho);
        F.mn = hll(FL.mn, FR.mn, UL.mn, UR.mn);
        F.mt = hll(FL.mt, FR.mt, UL.mt, UR.mt);
        F.mz = hll(FL.mz, FR.mz, UL.mz, UR.mz);
        F.e = hll(FL.e, FR.e, UL.e, UR.e);
        F.bn = hll(FL.bn, FR.bn, UL.bn, UR.bn);
        F.bt = hll(FL.bt, FR.bt, UL.bt, UR.bt);
        F.bz = hll(FL.bz, FR.bz, UL.bz, UR.bz);
        F.psi = hll(FL.psi, FR.psi, UL.psi, UR.psi);
        return F;
    }
    F.rho = combine(FL.rho, FR.rho, UL.rho, UR.rho);
    F.mn = combine(FL.mn, FR.mn, UL.mn, UR.mn);
    F.mt = combine(FL.mt, FR.mt, UL.mt, UR.mt);
    F.mz = combine(FL.mz, FR.mz, UL.mz, UR.mz);
    F.e = combine(FL.e, FR.e, UL.e, UR.e);
    F.bn = combine(FL.bn, FR.bn, UL.bn, UR.bn);
    F.bt = combine(FL.bt, FR.bt, UL.bt, UR.bt);
    F.bz = combine(FL.bz, FR.bz, UL.bz, UR.bz);
    F.psi = combine(FL.psi, FR.psi, UL.psi, UR.psi);
    return F;
}

// max(|vx| + cf_x, |vy| + cf_y) from conserved values; include/mhd/kernels/muscl_hll.hpp:211-239.
template <class T>
__device__ __forceinline__ T cell_max_signal_speed(T rho, T mx, T my, T mz, T energy, T bx, T by,
                                                   T bz, T gamma)
{
    const T inv_rho = fast_rcp(rho);
    PrimN<T> W;
    W.rho = rho;
    W.vn = mx * inv_rho;
    W.vt = my * inv_rho;
    W.vz = mz * inv_rho;
    const T ekin = T(0.5) * (mx * mx + my * my + mz * mz) * inv_rho;
    const T emag = T(0.5) * (bx * bx + by * by + bz * bz);
    W.p = (gamma - T(1)) * (energy - ekin - emag);
    W.bn = bx;
    W.bt = by;
    W.bz = bz;
    W.psi = T(0);
    const T sx = fabs(W.vn) + fast_speed_n_inv(W, inv_rho, gamma);
    PrimN<T> Wy = W;
    Wy.vn = W.vt;
    Wy.vt = W.vn;
    Wy.bn = by;
    Wy.bt = bx;
    const T sy = fabs(Wy.vn) + fast_speed_n_inv(Wy, inv_rho, gamma);
    return vmax(sx, sy);
}

// Conserved -> primitive as the reference RHS does it (reciprocal of rho, then products);
// include/mhd/kernels/cpu_rows.hpp:129-155. Writes rho, vx, vy, vz, p, bx, by, bz, psi.
template <class T>
__device__ __forceinline__ void cons_to_prim(const T* u, T gm1, T* w)
{
    const T rho = u[0], mx = u[1], my = u[2], mz = u[3], e = u[4];
    const T bx = u[5], by = u[6], bz = u[7];
    const T inv_rho = fast_rcp(rho);
    const T ekin = T(0.5) * (mx * mx + my * my + mz * mz) * inv_rho;
    const T emag = T(0.5) * (bx * bx + by * by + bz * bz);
    w[0] = rho;
    w[1] = mx * inv_rho;
    w[2] = my * inv_rho;
    w[3] = mz * inv_rho;
    w[4] = gm1 * (e - ekin - emag);
    w[5] = bx;
    w[6] = by;
    w[7] = bz;
    w[8] = u[8];
}

// Reflective copy of one fluid neighbour into a solid cell: to_primitive (division form), negate
// the normal velocity, floor rho and p at 1e-12, to_conservative;
// include/mhd/mask.hpp:123-137 with include/mhd/mhd_physics.hpp:23-57. axis 0 = x neighbour.
template <class T>
__device__ __forceinline__ void reflect_fill(const T* s, int axis, T gm1, T* out)
{
    const T rho = s[0], mx = s[1], my = s[2], mz = s[3], E = s[4];
    const T bx = s[5], by = s[6], bz = s[7];
    T vx = mx / rho;
    T vy = my / rho;
    const T vz = mz / rho;
    const T e_kin = T(0.5) * (mx * mx + my * my + mz * mz) / rho;
    const T e_mag = T(0.5) * (bx * bx + by * by + bz * bz);
    T p = gm1 * (E - e_kin - e_mag);
    T r = rho;
    if (axis == 0) {
        vx = -vx;
    } else {
        vy = -vy;
    }
    if (r < T(1e-12)) {
        r = T(1e-12);
    }
    if (p < T(1e-12)) {
        p = T(1e-12);
    }
    const T ek = T(0.5) * r * (vx * vx + vy * vy + vz * vz);
    const T em = T(0.5) * (bx * bx + by * by + bz * bz);
    out[0] = r;
    out[1] = r * vx;
    out[2] = r * vy;
    out[3] = r * vz;
    out[4] = p / gm1 + ek + em;
    out[5] = bx;
    out[6] = by;
    out[7] = bz;
    out[8] = s[8];
}

// Benign state of a solid cell without fluid neighbours: rho = p = 1 at rest, zero B and psi
// (include/mhd/mask.hpp:141-146).
template <class T>
__device__ __forceinline__ void isolated_fill(T gm1, T* out)
{
    out[0] = T(1);
    out[1] = T(0);
    out[2] = T(0);
    out[3] = T(0);
    out[4] = T(1) / gm1; // p / (gamma - 1) + 0 kinetic + 0 magnetic
    out[5] = T(0);
    out[6] = T(0);
    out[7] = T(0);
    out[8] = T(0);
}

// Generalised Ohm's law E = eta_O J + eta_H J x B / |B| + eta_A (J x B) x B / |B|^2, Hall and
// ambipolar skipped where |B|^2 < 1e-14; include/mhd/nonideal.hpp:63-102.
struct NonIdealCoef {
    int ohmic, hall, ambipolar;
    double eta_ohm, eta_hall, eta_ambipolar;
};

template <class T>
__device__ __forceinline__ void nonideal_e(T Jx, T Jy, T Jz, T Bx, T By, T Bz,
                                           const NonIdealCoef& c, T& Ex, T& Ey, T& Ez)
{
    Ex = T(0);
    Ey = T(0);
    Ez = T(0);
    if (c.ohmic) {
        const T eo = T(c.eta_ohm);
        Ex += eo * Jx;
        Ey += eo * Jy;
        Ez += eo * Jz;
    }
    if (!(c.hall || c.ambipolar)) {
        return;
    }
    const T B2 = Bx * Bx + By * By + Bz * Bz;
    if (B2 < T(1.0e-14)) {
        return;
    }
    const T cx = Jy * Bz - Jz * By;
    const T cy = Jz * Bx - Jx * Bz;
    const T cz = Jx * By - Jy * Bx;
    if (c.hall) {
        const T invB = fast_rcp(fast_sqrt(B2));
        const T eh = T(c.eta_hall);
        Ex += eh * cx * invB;
        Ey += eh * cy * invB;
        Ez += eh * cz * invB;
    }
    if (c.ambipolar) {
        const T dx = cy * Bz - cz * By;
        const T dy = cz * Bx - cx * Bz;
        const T dz = cx * By - cy * Bx;
        const T invB2 = fast_rcp(B2);
        const T ea = T(c.eta_ambipolar);
        Ex += ea * dx * invB2;
        Ey += ea * dy * invB2;
        Ez += ea * dz * invB2;
    }
}

} // namespace mhdb
