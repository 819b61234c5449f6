// TMA-fed warp strip-march stage kernel of the FP32-mixed form (ideal or non-ideal GLM-MHD, with
// or without a solid mask).
//
// The arithmetic is that of march_kernel.cuh (register-resident stencil, shuffle x sweep, every
// slope limited once and every face evaluated once; here the limiters return half slopes, the
// same values): ideal solves give the register march's values bit for bit, non-ideal ones agree
// to FP32 rounding (the compiler may contract the Ohm's-law products differently). What changes
// is how rows reach the warp: each warp runs a two-slot TMA pipeline per stream of rows, driven
// by lane 0 and completed on mbarriers:
//   * halo stream: the stage input's 9 hi planes of row y + 2, columns x0 - 4 .. x0 + 31
//     (box 36 x 1 x 9; the x origin x0 - 4 is a multiple of 4 floats, 16 bytes), issued two
//     rows ahead of its use; lane l reads column x0 - 2 + l at offset l + 2;
//   * own stream: the hi and lo planes of row y, owned columns x0 .. x0 + 27 (box 28 x 1 x 18),
//     of the stage input and, in stage 2, of U^n (updated in place), issued two rows ahead.
// Results leave through plain stores (ST = 0) or through TMA row stores from 1 or 2 staging
// slots (ST = 1, 2). Rows are addressed through the boundary map (periodic wrap / outflow clamp in
// y), so the copies never leave the interior in y. Lanes whose column lies outside [0, nx) (x
// halo of the first and last strips) load their values directly through the x map instead of
// from the box. With a mask (MASK), solid cells are wall-filled when their row is converted to
// primitives, and a solid cell's update stores the conservative form of those filled
// primitives (through plain stores). Each mbarrier wait is bounded (tma.cuh); on a timeout the warp records
// kStatusWaitTimeout in the Ctrl block, waits (bounded) for its copies still in flight and stops
// its strip.
#pragma once

#include "march_kernel.cuh"
#include "stage_delta.cuh"
#include "stage_mixed.cuh"
#include "tma.cuh"

namespace mhdb {

// Shared memory of one warp: 2 halo slots, 2 own slots, ST staging slots for the row stores
// (ST = 0: results are stored by the lanes; 1 or 2: TMA row stores through 1 or 2 staging slots),
// then the 4 mbarriers. ELEM is the size of a stored value: 4 for the FP32-mixed state (a row
// box holds 18 hi and lo planes), 8 for the FP64 state (9 planes). KIND 1 is the increment form
// (stage_delta.cuh): stage 1 has no own stream (its update needs no own-cell operand); stage 2
// has two halo boxes (hi(U^n), then delta) and own boxes delta (9 planes), then U^n (18).
// KIND 2 is the increment form whose stage 2 takes the own cells' delta from the halo stream: each
// owned lane keeps the 9 delta values of its column of the halo row in a 3-row ring of its own
// (the row is its own row two iterations later), so the own stream copies U^n alone (one box of
// 18 planes per row instead of two boxes of 27).
template <int STAGE, int ST, int ELEM = 4, int KIND = 0>
struct MarchTmaLayout {
    static constexpr bool kDelta = KIND >= 1;
    static constexpr bool kStash = KIND == 2 && STAGE == 2;
    static constexpr int kOwnPlanes = ELEM == 4 ? 18 : 9;
    static constexpr int kHaloBoxBytes = 9 * kTmaHaloW * ELEM;   // 1296 B (FP32), 2592 B (FP64)
    static constexpr int kHaloBoxSlot = (kHaloBoxBytes + 127) / 128 * 128;
    static constexpr int kHaloBoxes = (kDelta && STAGE == 2) ? 2 : 1;
    static constexpr int kHaloBytes = kHaloBoxes * kHaloBoxBytes; // transaction bytes per row
    static constexpr int kHaloSlot = kHaloBoxes * kHaloBoxSlot;
    static constexpr int kOwnBoxBytes = kOwnPlanes * kTmaOwnW * ELEM; // 2016 B per box
    static constexpr int kOwnBoxSlot = (kOwnBoxBytes + 127) / 128 * 128; // 2048 B
    // own box A (the stage input's own cells; delta in the increment form) and box B (U^n)
    static constexpr int kOwnPlanesA = kStash ? 0 : (kDelta ? 9 : kOwnPlanes);
    static constexpr int kOwnABytes = kOwnPlanesA * kTmaOwnW * ELEM;
    static constexpr int kOwnBOff = (kOwnABytes + 127) / 128 * 128; // byte offset of box B
    static constexpr int kOwnBoxes =
        kStash ? 1 : (kDelta ? (STAGE == 1 ? 0 : 2) : (STAGE == 1 ? 1 : 2));
    static constexpr int kOwnSlot = kOwnBoxes == 0 ? 0 : (kOwnBoxes == 1 ? kOwnBoxSlot
                                                                        : kOwnBOff + kOwnBoxSlot);
    static constexpr int kOwnTx = kOwnBoxes == 0 ? 0 : (kOwnBoxes == 1 ? kOwnBoxBytes
                                                                      : kOwnABytes + kOwnBoxBytes);
    static constexpr int kStageOff = 2 * kHaloSlot + 2 * kOwnSlot;
    // delta ring (kStash): 3 rows x 9 planes x the owned columns
    static constexpr int kStashRow = 9 * kTmaOwnW;
    static constexpr int kStashOff = kStageOff + ST * kOwnBoxSlot;
    static constexpr int kStashBytes = kStash ? (3 * kStashRow * 4 + 127) / 128 * 128 : 0;
    static constexpr int kBarOff = kStashOff + kStashBytes;
    static constexpr int kWarpBytes = kBarOff + 128;             // 4 mbarriers, padded
};

template <int STAGE, int ST, int ELEM = 4, int KIND = 0>
constexpr size_t march_tma_smem_bytes(int warps)
{
    return static_cast<size_t>(warps) * MarchTmaLayout<STAGE, ST, ELEM, KIND>::kWarpBytes + 128;
}

// The FP32-mixed one-warp configurations run 16 blocks per SM: their shared memory (plus the
// 1 KB an SM reserves per block) must fit the SM's 228 KB, or occupancy drops.
constexpr bool fits_16_blocks(size_t bytes) { return 16 * (bytes + 1024) <= 228 * 1024; }
static_assert(fits_16_blocks(march_tma_smem_bytes<1, 1>(1)) &&
                  fits_16_blocks(march_tma_smem_bytes<2, 0>(1)) &&
                  fits_16_blocks(march_tma_smem_bytes<1, 0, 4, 1>(1)) &&
                  fits_16_blocks(march_tma_smem_bytes<2, 0, 4, 1>(1)) &&
                  fits_16_blocks(march_tma_smem_bytes<2, 0, 4, 2>(1)),
              "a one-warp FP32-mixed strip-march layout no longer fits 16 blocks per SM");

template <int L, int STAGE, int LY, bool HF, int ST, bool NI, bool MASK = false,
          class Policy = PolicyMixed>
__device__ __forceinline__ double march_tma_strip(const typename Policy::Args& a,
                                                  const MarchTmaMaps& m,
                                                  int x0, int y0, int lane, unsigned char* wbase,
                                                  bool& failed_out)
{
    using T = typename Policy::T;
    using Raw = typename Policy::Raw;
    using Lay = MarchTmaLayout<STAGE, ST, sizeof(T), Policy::kLayout>;
    static_assert(sizeof(T) == 4 || ST == 0, "the FP64 TMA strip march stores through the lanes");
    static_assert(!Lay::kDelta || ST == 0, "the increment form stores through the lanes");
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
    const bool in_x = gx >= 0 && gx < g.nx;
    const bool own = lane >= 2 && lane < 2 + kMarchOwned && gx < g.nx;
    const int y1 = min(y0 + LY, g.ny);
    const int nrows = y1 - y0;

    const T* halo_f = reinterpret_cast<const T*>(wbase);
    const T* own_f = reinterpret_cast<const T*>(wbase + 2 * Lay::kHaloSlot);
    float* stg_f = reinterpret_cast<float*>(wbase + Lay::kStageOff);
    // delta ring (kStash): row item j in slot j % 3, this lane's owned column at lane - 2
    float* stash_f = reinterpret_cast<float*>(wbase + Lay::kStashOff) + (lane >= 2 ? lane - 2 : 0);
    const uint32_t halo_s = smem_addr(wbase);
    const uint32_t own_s = halo_s + 2 * Lay::kHaloSlot;
    const uint32_t stg_s = halo_s + Lay::kStageOff;
    const uint32_t bar_s = halo_s + Lay::kBarOff; // halo: +0, +8; own: +16, +24

    if (lane == 0) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            mbar_init(bar_s + 8 * b, 1);
        }
        fence_mbar_init();
    }
    __syncwarp();

    // Consts::stall_tx (timeout tests only): extra transaction bytes on the first halo copy of
    // the strip at the origin, which no copy delivers; every copy itself stays well-formed.
    const uint32_t stall = (x0 == 0 && y0 == 0) ? static_cast<uint32_t>(k.stall_tx) : 0u;
    // Item i of the halo stream is row y0 + 2 + i; item i of the own stream is row y0 + i; both
    // use slot i & 1, whose (i >> 1)-th phase completes it.
    auto issue_halo = [&](int i) {
        const uint32_t slot = static_cast<uint32_t>(i & 1);
        const uint32_t bar = bar_s + 8 * slot;
        const int yy = map_index(y0 + 2 + i, g.ny, g.bc_y);
        mbar_arrive_expect_tx(bar, Lay::kHaloBytes + (i == 0 ? stall : 0u));
        tma_load_3d(halo_s + slot * Lay::kHaloSlot, &m.in_halo, bar, x0 - 4, yy, 0);
        if constexpr (Lay::kHaloBoxes == 2) {
            tma_load_3d(halo_s + slot * Lay::kHaloSlot + Lay::kHaloBoxSlot, &m.delta_halo, bar,
                        x0 - 4, yy, 0);
        }
    };
    auto issue_own = [&](int i) {
        if constexpr (Lay::kOwnBoxes > 0) {
            const uint32_t slot = static_cast<uint32_t>(i & 1);
            const uint32_t bar = bar_s + 16 + 8 * slot;
            const uint32_t dst = own_s + slot * Lay::kOwnSlot;
            mbar_arrive_expect_tx(bar, Lay::kOwnTx);
            if constexpr (Lay::kOwnPlanesA > 0) {
                tma_load_3d(dst, &m.in_own, bar, x0, y0 + i, 0);
            }
            if constexpr (STAGE == 2) {
                tma_load_3d(dst + Lay::kOwnBOff, &m.out_own, bar, x0, y0 + i, 0);
            }
        }
    };
    int halo_issued = 0, own_issued = 0, halo_done = 0, own_done = 0;
    if (lane == 0) {
        issue_halo(0);
        issue_own(0);
        if (nrows > 1) {
            issue_halo(1);
            issue_own(1);
        }
    }
    halo_issued = nrows > 1 ? 2 : 1;
    own_issued = Lay::kOwnBoxes > 0 ? halo_issued : 0;

    auto load = [&](int y, Raw& r) { Policy::load_raw(a, g, sx, map_index(y, g.ny, g.bc_y), r); };
    // Primitives of this lane's cell of row y. With a mask, an interior solid cell (by its own,
    // unmapped coordinates: ghosts keep the stored values, include/mhd/time_integrator.hpp:46-49)
    // is wall-filled from its first fluid interior neighbour in the order +x, -x, +y, -y, or set
    // to the isolated state (include/mhd/mask.hpp:100-146). Filled values feed FP32 fluxes only,
    // so the x neighbours' primitives come from the neighbour lanes (reflected: normal velocity
    // negated, density and pressure floored at 1e-12), an isolated cell takes rho = p = 1 at rest
    // with zero B and psi, and the remaining cases (a fluid y neighbour, or an x neighbour outside
    // this warp) take the FP64 fill of the tile kernel from global memory.
    auto prim = [&](int y, const Raw& r, T (&w)[9]) {
        const int sy = map_index(y, g.ny, g.bc_y);
        Policy::template raw_prim<STAGE, MASK>(a, g, sx, sy, r, k, w);
        if constexpr (MASK) {
            if (!a.walls || y < 0 || y >= g.ny) { // warp-uniform
                return;
            }
            const bool solid = in_x && is_solid(a.mask, g, sx, sy);
            if constexpr (sizeof(T) == 8) {
                // FP64: every solid cell takes the FP64 fill of the tile kernel (its operations
                // and order, so the filled values are those of the oracle)
                if (solid) {
                    double f[9];
                    Policy::template wall_fill<STAGE, true>(a, g, sx, sy, k.gm1, f);
                    Policy::prim_of(f, k, w);
                }
                return;
            }
            if (!__any_sync(kFull, solid)) {
                return;
            }
            const bool fluid = in_x && !solid;
            const bool fluid_e = __shfl_down_sync(kFull, fluid, 1) && lane < 31;
            const bool fluid_w = __shfl_up_sync(kFull, fluid, 1) && lane > 0;
            T we[9], ww[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                we[c] = __shfl_down_sync(kFull, w[c], 1);
                ww[c] = __shfl_up_sync(kFull, w[c], 1);
            }
            if (!solid) {
                return;
            }
            const T tiny = T(1e-12);
            if (fluid_e || (fluid_w && lane > 0 && lane < 31 && !fluid_e)) {
                // lane 31 never gets here (its +x neighbour is outside the warp); lane 0 only
                // through fluid_e
                const T* s = fluid_e ? we : ww;
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    w[c] = s[c];
                }
                w[1] = -w[1];
                w[0] = w[0] < tiny ? tiny : w[0];
                w[4] = w[4] < tiny ? tiny : w[4];
                return;
            }
            const bool edge = lane == 31 || (lane == 0 && !fluid_e);
            const bool fluid_n = y + 1 < g.ny && !is_solid(a.mask, g, sx, y + 1);
            const bool fluid_s = y > 0 && !is_solid(a.mask, g, sx, y - 1);
            if (edge || fluid_n || fluid_s) {
                double f[9];
                Policy::template wall_fill<STAGE, true>(a, g, sx, sy, k.gm1, f);
                Policy::prim_of(f, k, w);
                return;
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                w[c] = T(0);
            }
            w[0] = T(1);
            w[4] = T(1);
        }
    };

    // Prologue (direct loads): rows y0-2 .. y0+1, slopes of rows y0-1 and y0, flux G(y0 - 1/2).
    T Wm[9], Wp[9], sYc[9], Gm[9];
    T Jc[NI ? 3 : 1]; // current of row y (NI)
    {
        Raw r0, r1, r2, r3;
        load(y0 - 2, r0);
        load(y0 - 1, r1);
        load(y0, r2);
        load(y0 + 1, r3);
        T wa[9], wb[9], sYm[9];
        prim(y0 - 2, r0, wa);
        prim(y0 - 1, r1, wb);
        prim(y0, r2, Wm);
        prim(y0 + 1, r3, Wp);
        {
            T d0[9], d1[9], d2[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                d0[c] = wb[c] - wa[c];
                d1[c] = Wm[c] - wb[c];
                d2[c] = Wp[c] - Wm[c];
            }
            limit_half_slopes<L>(d0, d1, sYm);
            limit_half_slopes<L>(d1, d2, sYc);
        }
        face_flux_regs<T, true, true>(wb, sYm, Wm, sYc, gamma, inv_gm1, c_h, Gm);
        if constexpr (Lay::kStash) {
            // the own cells' delta of rows y0 and y0 + 1 (the ring's first two items)
            if (own) {
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    if (r < nrows) {
                        const size_t o = static_cast<size_t>(y0 + r) * g.pitch + gx;
#pragma unroll
                        for (int c = 0; c < 9; ++c) {
                            stash_f[r * Lay::kStashRow + c * kTmaOwnW] =
                                __ldg(a.delta + static_cast<size_t>(c) * g.plane + o);
                        }
                    }
                }
            }
        }
        if constexpr (NI) {
            T Jb[3];
            march_current(wa, wb, Wm, inv_2dx, inv_2dy, Jb);
            march_current(wb, Wm, Wp, inv_2dx, inv_2dy, Jc);
            march_nonideal_y(Jb, wb, Jc, Wm, k.ni, Gm);
        }
    }

    double smax = 0.0;
    bool failed = false;
    int ring_rd = 0, ring_wr = 2; // delta ring slots of rows y and y + 2 (kStash)
#pragma unroll 1
    for (int i = 0; i < nrows; ++i) {
        const int y = y0 + i;
        // x sweep of row y: dF = F(x + 1/2) - F(x - 1/2) on the owned lanes
        T dF[9];
        auto x_sweep = [&]() {
            T Wn[9], sX[9], sXn[9], F[9];
            {
                T dL[9], dR[9];
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    Wn[c] = __shfl_down_sync(kFull, Wm[c], 1);
                    dR[c] = Wn[c] - Wm[c];
                    dL[c] = __shfl_up_sync(kFull, dR[c], 1);
                }
                limit_half_slopes<L>(dL, dR, sX);
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                sXn[c] = __shfl_down_sync(kFull, sX[c], 1);
            }
            face_flux_regs<T, false, true>(Wm, sX, Wn, sXn, gamma, inv_gm1, c_h, F);
            if constexpr (NI) {
                march_nonideal_x(Jc, Wm, Wn, k.ni, F);
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                dF[c] = F[c] - __shfl_up_sync(kFull, F[c], 1);
            }
        };
        if constexpr (!HF) {
            x_sweep();
        }
        // row y + 2 from the halo stream
        Raw rn;
        {
            const uint32_t slot = static_cast<uint32_t>(i & 1);
            const bool ok = mbar_wait(bar_s + 8 * slot, static_cast<uint32_t>((i >> 1) & 1));
            if (__any_sync(kFull, !ok)) {
                failed = true;
                break;
            }
            halo_done = i + 1;
            if (in_x) {
                const T* src = halo_f + slot * (Lay::kHaloSlot / sizeof(T)) + lane + 2;
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    rn.v[c] = src[c * kTmaHaloW];
                    if constexpr (Lay::kHaloBoxes == 2) { // U* hi = fl(hi(U^n) + delta)
                        const T dl = src[Lay::kHaloBoxSlot / sizeof(T) + c * kTmaHaloW];
                        if constexpr (Lay::kStash) {
                            if (own && i + 2 < nrows) {
                                stash_f[ring_wr * Lay::kStashRow + c * kTmaOwnW] = dl;
                            }
                        }
                        rn.v[c] = __fadd_rn(rn.v[c], dl);
                    }
                }
            } else {
                load(y + 2, rn);
            }
            __syncwarp();
            if (i + 2 < nrows) {
                if (lane == 0) {
                    issue_halo(i + 2);
                }
                halo_issued = i + 3;
            }
        }
        T W2[9], sYn[9], Gp[9];
        prim(y + 2, rn, W2);
        if constexpr (HF) {
            x_sweep(); // after the halo wait: the x and y fluxes share one scheduling region
        }
        {
            T dm[9], dp[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                dm[c] = Wp[c] - Wm[c];
                dp[c] = W2[c] - Wp[c];
            }
            limit_half_slopes<L>(dm, dp, sYn);
        }
        face_flux_regs<T, true, true>(Wm, sYc, Wp, sYn, gamma, inv_gm1, c_h, Gp);
        T Jn[NI ? 3 : 1];
        if constexpr (NI) {
            march_current(Wm, Wp, W2, inv_2dx, inv_2dy, Jn);
            march_nonideal_y(Jc, Wm, Jn, Wp, k.ni, Gp);
        }
        // own-cell operands of row y from the own stream, then the stage update
        {
            const uint32_t slot = static_cast<uint32_t>(i & 1);
            if constexpr (Lay::kOwnBoxes > 0) {
                const bool ok = mbar_wait(bar_s + 16 + 8 * slot,
                                          static_cast<uint32_t>((i >> 1) & 1));
                if (__any_sync(kFull, !ok)) {
                    failed = true;
                    break;
                }
                own_done = i + 1;
            }
            if constexpr (ST > 0) {
                if (lane == 0) {
                    bulk_wait_read<ST - 1>(); // the store that last used this slot has read it
                }
                __syncwarp();
            }
            const T* src = own_f + slot * (Lay::kOwnSlot / sizeof(T)) + (lane - 2);
            // own-cell operand q: plane q of box A (the stage input; delta in the increment
            // form), then (stage 2) plane q - kOwnPlanesA of box B (U^n)
            auto op = [&](int q) {
                if constexpr (Lay::kStash) { // delta from the ring, U^n from box B
                    return q < 9 ? stash_f[ring_rd * Lay::kStashRow + q * kTmaOwnW]
                                 : src[(q - 9) * kTmaOwnW];
                }
                return q < Lay::kOwnPlanesA
                           ? src[q * kTmaOwnW]
                           : src[Lay::kOwnBOff / sizeof(T) + (q - Lay::kOwnPlanesA) * kTmaOwnW];
            };
            const bool solid = MASK && own && is_solid(a.mask, g, gx, y);
            if constexpr (!MASK) {
                // no solid cells
            } else if constexpr (sizeof(T) == 8) {
                if (solid) {
                    // FP64: the tile kernel's solid update, from global memory: L = 0; with walls
                    // stage 1 stores fill(U^n) and stage 2 (U*_stored + fill(U*)) / 2
                    T Lz[9] = {};
                    Policy::template update<STAGE, true>(a, g, gx, y, true, Lz, T(0), 0.0, dt,
                                                         k, smax);
                }
            } else if constexpr (Lay::kDelta) {
                if (solid && a.walls) {
                    // The stored U* of a solid cell is the fill of U^n: stage 1 stores the
                    // increment fill(U^n) - U^n (rounded to FP32; U^n of the cell from global
                    // memory, as stage 1 has no own stream); stage 2 stores (U*_stored +
                    // fill(U*)) / 2 into U^{n+1}, with U*_stored = U^n + increment. The fill is
                    // this row's filled primitives Wm, made conservative in FP64.
                    const double rho = Wm[0], vx = Wm[1], vy = Wm[2], vz = Wm[3];
                    const double bx = Wm[5], by = Wm[6], bz = Wm[7];
                    double f[9] = {rho, rho * vx, rho * vy, rho * vz,
                                   static_cast<double>(Wm[4]) * k.inv_gm1 +
                                       0.5 * rho * (vx * vx + vy * vy + vz * vz) +
                                       0.5 * (bx * bx + by * by + bz * bz),
                                   bx, by, bz, static_cast<double>(Wm[8])};
                    const size_t o = static_cast<size_t>(y) * g.pitch + gx;
                    if constexpr (STAGE == 1) {
                        double un[9];
                        load_cons_mx(a.un, g, gx, y, un);
#pragma unroll
                        for (int c = 0; c < 9; ++c) {
                            a.delta[static_cast<size_t>(c) * g.plane + o] =
                                __double2float_rn(f[c] - un[c]);
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 9; ++c) {
                            const double us = (static_cast<double>(op(9 + c)) +
                                               static_cast<double>(op(18 + c))) +
                                              static_cast<double>(op(c));
                            split_store(a.out, static_cast<size_t>(c) * g.plane + o,
                                        0.5 * (us + f[c]));
                        }
                    }
                } else if (solid) {
                    // without walls a solid cell only has L = 0
                    const T Lz[9] = {};
                    Policy::template update_ops<STAGE>(a, g, gx, y, true, Lz, dt, k, smax, op);
                }
            } else if (solid && a.walls) {
                // L = 0 and the stored value is the wall fill of the stage input (tile kernel:
                // PolicyMixed::update): stage 1 stores fill(U^n), stage 2 (U*_stored +
                // fill(U*)) / 2. The fill is this row's filled primitives Wm, made conservative
                // in FP64; plain stores only (ST == 0).
                const double rho = Wm[0], vx = Wm[1], vy = Wm[2], vz = Wm[3];
                const double bx = Wm[5], by = Wm[6], bz = Wm[7];
                double f[9] = {rho, rho * vx, rho * vy, rho * vz,
                               static_cast<double>(Wm[4]) * k.inv_gm1 +
                                   0.5 * rho * (vx * vx + vy * vy + vz * vz) +
                                   0.5 * (bx * bx + by * by + bz * bz),
                               bx, by, bz, static_cast<double>(Wm[8])};
                const size_t o = static_cast<size_t>(y) * g.pitch + gx;
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    if constexpr (STAGE == 2) {
                        f[c] = 0.5 * ((static_cast<double>(src[c * kTmaOwnW]) +
                                       static_cast<double>(src[(9 + c) * kTmaOwnW])) + f[c]);
                    }
                    split_store(a.out, static_cast<size_t>(c) * g.plane + o, f[c]);
                }
            } else if (solid) {
                // without walls a solid cell only has L = 0
                const T Lz[9] = {};
                Policy::template update_ops<STAGE>(a, g, gx, y, true, Lz, dt, k, smax, op);
            }
            if (own && !solid) {
                T Lc[9];
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    Lc[c] = -dF[c] * inv_dx - (Gp[c] - Gm[c]) * inv_dy; // include/mhd/rhs.hpp:121
                }
                if (psi_damp != 0.0) {
                    Lc[8] -= static_cast<T>(psi_damp) * Wm[8]; // include/mhd/rhs.hpp:219-225
                }
                if constexpr (ST > 0) {
                    float* dst = stg_f + (i % (ST > 0 ? ST : 1)) * (Lay::kOwnBoxSlot / 4) + (lane - 2);
                    Policy::template update_ops<STAGE>(a, !reduce_row(g, y), Lc, dt, k, smax, op,
                                                       [&](int c, float h, float l) {
                                                           dst[c * kTmaOwnW] = h;
                                                           dst[(9 + c) * kTmaOwnW] = l;
                                                       });
                    fence_async_smem();
                } else {
                    Policy::template update_ops<STAGE>(a, g, gx, y, false, Lc, dt, k, smax, op);
                }
            }
            __syncwarp();
            if (lane == 0) {
                if constexpr (ST > 0) {
                    tma_store_3d(&m.out_own,
                                 stg_s + static_cast<uint32_t>(i % (ST > 0 ? ST : 1)) * Lay::kOwnBoxSlot,
                                 x0, y, 0);
                    bulk_commit();
                }
                if (i + 2 < nrows) {
                    issue_own(i + 2);
                }
            }
            if (i + 2 < nrows && Lay::kOwnBoxes > 0) {
                own_issued = i + 3;
            }
        }
        if constexpr (Lay::kStash) {
            ring_rd = ring_rd == 2 ? 0 : ring_rd + 1;
            ring_wr = ring_wr == 2 ? 0 : ring_wr + 1;
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
    }
    if constexpr (ST > 0) {
        if (lane == 0) {
            bulk_wait_all(); // the row stores have written global memory and read their source
        }
        __syncwarp();
    }
    if (failed) {
        // Record the failure and let every copy of this warp land before the CTA can exit; the
        // caller processes no further strips with these barriers.
        if (lane == 0) {
            atomicOr(&a.ctrl->status, static_cast<int>(kStatusWaitTimeout));
        }
        for (int j = halo_done; j < halo_issued; ++j) {
            mbar_wait(bar_s + 8 * (j & 1), static_cast<uint32_t>((j >> 1) & 1));
        }
        for (int j = own_done; j < own_issued; ++j) {
            mbar_wait(bar_s + 16 + 8 * (j & 1), static_cast<uint32_t>((j >> 1) & 1));
        }
        failed_out = true;
        return 0.0;
    }
    __syncwarp();
    if (lane == 0) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            mbar_inval(bar_s + 8 * b); // every phase completed; the next strip initialises anew
        }
    }
    __syncwarp();
    return smax;
}

template <int L, int STAGE, int LY, int NW, int MINB, bool HF, int ST, bool NI, bool MASK = false,
          class Policy = PolicyMixed>
__global__ void __launch_bounds__(NW * 32, MINB) march_tma_kernel(const typename Policy::Args a,
                                                                   const __grid_constant__ MarchTmaMaps m)
{
    if (a.ctrl->finished != 0) {
        return;
    }
    extern __shared__ unsigned char march_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // 128-byte aligned start, derived from the shared array itself so that every access through
    // it compiles to a shared-memory load
    unsigned char* base = march_smem + ((128u - (smem_addr(march_smem) & 127u)) & 127u);
    const int x0 = (blockIdx.x * NW + warp) * kMarchOwned;
    double smax = 0.0;
    bool failed = false;
    if (x0 < a.geom.nx) { // warp-uniform
        static_assert(!MASK || ST == 0, "masked strips store through the lanes");
        smax = march_tma_strip<L, STAGE, LY, HF, ST, NI, MASK, Policy>(
            a, m, x0, static_cast<int>(blockIdx.y) * LY, lane,
            base + warp * MarchTmaLayout<STAGE, ST, sizeof(typename Policy::T),
                                         Policy::kLayout>::kWarpBytes,
            failed);
    }
    if constexpr (STAGE == 2) {
        reduce_signal_speed_and_finish(smax, a.ctrl, a.k, gridDim.x * gridDim.y, true);
    }
}

// One solve of a TMA batch: stage arguments, the tensor maps of both stages, its tiling. For the
// increment form (stage_delta.cuh) the arguments and maps of both state-buffer parities: parity
// q holds U^n in buffer q (0: U, 1: U*'s buffer), and a solve that has run s steps is in parity
// s & 1.
struct BatchSolveTma {
    MarchTmaMaps maps[2]; // stage 1 and stage 2
    StageArgsMx stage[2];
    MarchTmaMaps dmaps[2][2]; // increment form: [parity][stage - 1]
    StageArgsDelta dstage[2]; // increment form: [parity]
    int tiles_x; // blocks per row
    int ntiles;  // blocks of this solve
};

// Persistent TMA strip march over a block work-list of many independent solves (items: solve
// index, block index), as batch_march_kernel; the tensor maps come from the descriptor array in
// global memory (lane 0 acquires them before its copies). A warp whose copies timed out processes
// no further items: the solves of the items it would have run report kStatusWaitTimeout too.
template <int L, bool NI, int STAGE, int LY, int NW, int MINB, bool HF, int ST>
__global__ void __launch_bounds__(NW * 32, MINB) batch_march_tma_kernel(
    const BatchSolveTma* solves, const int2* __restrict__ work, int nwork)
{
    __shared__ __align__(16) StageArgsMx sa;
    __shared__ int s_tiles_x, s_ntiles;
    extern __shared__ unsigned char march_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = march_smem + ((128u - (smem_addr(march_smem) & 127u)) & 127u);
    unsigned char* wbase = base + warp * MarchTmaLayout<STAGE, ST>::kWarpBytes;
    bool failed = false;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 it = work[w];
        __syncthreads(); // the previous item is done with sa
        {
            const int* src = reinterpret_cast<const int*>(&solves[it.x].stage[STAGE - 1]);
            int* dst = reinterpret_cast<int*>(&sa);
            for (int i = threadIdx.x; i < static_cast<int>(sizeof(StageArgsMx) / sizeof(int));
                 i += NW * 32) {
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
        const MarchTmaMaps& m = solves[it.x].maps[STAGE - 1];
        const int x0 = ((it.y % s_tiles_x) * NW + warp) * kMarchOwned;
        const int y0 = (it.y / s_tiles_x) * LY;
        double smax = 0.0;
        if (x0 < sa.geom.nx && failed) { // warp-uniform
            // this warp's barriers are unusable after a timed-out wait, so it cannot advance the
            // item: its solve reports the timeout instead of skipping cells
            if (lane == 0) {
                atomicOr(&sa.ctrl->status, static_cast<int>(kStatusWaitTimeout));
            }
        } else if (x0 < sa.geom.nx) { // warp-uniform
            if (lane == 0) {
                tensormap_acquire(&m.in_halo);
                tensormap_acquire(&m.in_own);
                tensormap_acquire(&m.out_own);
            }
            __syncwarp();
            smax = march_tma_strip<L, STAGE, LY, HF, ST, NI>(sa, m, x0, y0, lane, wbase, failed);
        }
        if constexpr (STAGE == 2) {
            reduce_signal_speed_and_finish(smax, sa.ctrl, sa.k, static_cast<unsigned>(s_ntiles),
                                           true);
        }
    }
}

// The batch kernel of the increment form: as batch_march_tma_kernel, with each solve's
// arguments and tensor maps taken for the state-buffer parity of its step counter (read before
// the stage; it only changes when the solve's stage-2 reduction completes).
template <int L, bool NI, int STAGE, int LY, int NW, int MINB, bool HF>
__global__ void __launch_bounds__(NW * 32, MINB) batch_march_delta_kernel(
    const BatchSolveTma* solves, const int2* __restrict__ work, int nwork)
{
    __shared__ __align__(16) StageArgsDelta sa;
    __shared__ int s_tiles_x, s_ntiles, s_q;
    extern __shared__ unsigned char march_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = march_smem + ((128u - (smem_addr(march_smem) & 127u)) & 127u);
    unsigned char* wbase = base + warp * MarchTmaLayout<STAGE, 0, 4, 2>::kWarpBytes;
    bool failed = false;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 it = work[w];
        __syncthreads(); // the previous item is done with sa
        if (threadIdx.x == 0) {
            s_q = solves[it.x].dstage[0].ctrl->steps & 1;
            s_tiles_x = solves[it.x].tiles_x;
            s_ntiles = solves[it.x].ntiles;
        }
        __syncthreads();
        {
            const int* src = reinterpret_cast<const int*>(&solves[it.x].dstage[s_q]);
            int* dst = reinterpret_cast<int*>(&sa);
            for (int i = threadIdx.x; i < static_cast<int>(sizeof(StageArgsDelta) / sizeof(int));
                 i += NW * 32) {
                dst[i] = src[i];
            }
        }
        __syncthreads();
        if (sa.ctrl->finished != 0) {
            continue;
        }
        const MarchTmaMaps& m = solves[it.x].dmaps[s_q][STAGE - 1];
        const int x0 = ((it.y % s_tiles_x) * NW + warp) * kMarchOwned;
        const int y0 = (it.y / s_tiles_x) * LY;
        double smax = 0.0;
        if (x0 < sa.geom.nx && failed) { // warp-uniform: as in batch_march_tma_kernel
            if (lane == 0) {
                atomicOr(&sa.ctrl->status, static_cast<int>(kStatusWaitTimeout));
            }
        } else if (x0 < sa.geom.nx) { // warp-uniform
            if (lane == 0) {
                tensormap_acquire(&m.in_halo);
                if constexpr (STAGE == 2) {
                    tensormap_acquire(&m.in_own);
                    tensormap_acquire(&m.out_own);
                    tensormap_acquire(&m.delta_halo);
                }
            }
            __syncwarp();
            smax = march_tma_strip<L, STAGE, LY, HF, 0, NI, false, PolicyDelta<STAGE, 2>>(
                sa, m, x0, y0, lane, wbase, failed);
        }
        if constexpr (STAGE == 2) {
            reduce_signal_speed_and_finish(smax, sa.ctrl, sa.k, static_cast<unsigned>(s_ntiles),
                                           true);
        }
    }
}

} // namespace mhdb
