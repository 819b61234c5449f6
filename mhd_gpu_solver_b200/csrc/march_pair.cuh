// Two-column TMA strip march of the FP32-mixed increment form (unmasked solves, ideal or
// non-ideal).
//
// The single-column strip march (march_tma.cuh) gives each lane one column: a warp covers 32
// columns of which 28 are its own, and the 4 x-halo lanes run the whole stencil for nothing
// (12.5 % of the issue slots of an issue-bound kernel). Here lane l holds two neighbouring
// columns, A = x0 - 2 + 2l and B = A + 1, so a warp covers 64 columns and owns the 60 of lanes
// 1..30 (6 % halo). Per row each lane evaluates four faces: the x faces A + 1/2 (inside the lane)
// and B + 1/2 (to the next lane's A), and the y faces of both columns. The arithmetic of every
// slope, face and update is that of the single-column march, operand for operand, so ideal
// solves give its values bit for bit; x neighbours come from the other column of the lane or
// from one shuffle, which halves the shuffles per cell.
//
// Rows reach the warp as in march_tma.cuh, through two-slot TMA rings completed on mbarriers:
//   * halo stream: row y + 2, columns x0 - 4 .. x0 + 63 (box 68 x 1 x 9; x0 is a multiple of 60,
//     so x0 - 4 is a multiple of 4 floats, 16 bytes), of hi(U^n) and, in stage 2, of the
//     increment delta; lane l reads its two columns as one 8-byte word at offset 2l + 2;
//   * own stream (stage 2): row y, owned columns x0 .. x0 + 59 (box 60 x 1 x 9 of delta and
//     60 x 1 x 18 of U^n's hi and lo planes).
// Lanes whose column lies outside [0, nx) (the first and last strips) load it through the x map.
// Every mbarrier wait is bounded (tma.cuh); on a timeout the warp records kStatusWaitTimeout,
// waits (bounded) for its copies in flight and stops. Consts::stall_tx arms the first halo copy
// of the strip at the origin as in march_tma.cuh.
#pragma once

#include "march_tma.cuh"

namespace mhdb {

constexpr int kPairOwned = 60;  // owned columns per warp (lanes 1..30, two each)
constexpr int kPairHaloW = 68;  // halo box: columns x0 - 4 .. x0 + 63
constexpr int kPairOwnW = 60;   // own box: columns x0 .. x0 + 59

// Shared memory of one warp: 2 halo slots (1 box in stage 1; hi(U^n) and delta in stage 2),
// 2 own slots (stage 2: delta, then U^n's hi and lo planes), 4 mbarriers.
template <int STAGE>
struct MarchPairLayout {
    static constexpr int kHaloBoxBytes = 9 * kPairHaloW * 4; // 2448 B
    static constexpr int kHaloBoxSlot = (kHaloBoxBytes + 127) / 128 * 128;
    static constexpr int kHaloBoxes = STAGE == 2 ? 2 : 1;
    static constexpr int kHaloBytes = kHaloBoxes * kHaloBoxBytes; // transaction bytes per row
    static constexpr int kHaloSlot = kHaloBoxes * kHaloBoxSlot;
    static constexpr int kOwnABytes = 9 * kPairOwnW * 4;  // delta, 2160 B
    static constexpr int kOwnBOff = (kOwnABytes + 127) / 128 * 128;
    static constexpr int kOwnBBytes = 18 * kPairOwnW * 4; // U^n hi and lo, 4320 B
    static constexpr int kOwnSlot = STAGE == 2 ? kOwnBOff + (kOwnBBytes + 127) / 128 * 128 : 0;
    static constexpr int kOwnTx = STAGE == 2 ? kOwnABytes + kOwnBBytes : 0;
    static constexpr int kBarOff = 2 * kHaloSlot + 2 * kOwnSlot;
    static constexpr int kWarpBytes = kBarOff + 128;
};

template <int STAGE>
constexpr size_t march_pair_smem_bytes()
{
    return static_cast<size_t>(MarchPairLayout<STAGE>::kWarpBytes) + 128;
}

// Current J of the two columns of row c (rows s below and n above): x neighbours from the other
// column of the lane or from the neighbour lane. Lane 0's column A and lane 31's column B get
// wrong values (their outer neighbour is outside the warp); no used face reads them.
template <class T>
__device__ __forceinline__ void pair_current(const T (&Ws)[2][9], const T (&Wc)[2][9],
                                             const T (&Wn)[2][9], T inv_2dx, T inv_2dy,
                                             T (&J)[2][3])
{
    constexpr unsigned kFull = 0xffffffffu;
    const T bz_w = __shfl_up_sync(kFull, Wc[1][7], 1), by_w = __shfl_up_sync(kFull, Wc[1][6], 1);
    const T bz_e = __shfl_down_sync(kFull, Wc[0][7], 1), by_e = __shfl_down_sync(kFull, Wc[0][6], 1);
    cell_current(Wn[0][7], Ws[0][7], Wc[1][7], bz_w, Wc[1][6], by_w, Wn[0][5], Ws[0][5], inv_2dx,
                 inv_2dy, J[0]);
    cell_current(Wn[1][7], Ws[1][7], bz_e, Wc[0][7], by_e, Wc[0][6], Wn[1][5], Ws[1][5], inv_2dx,
                 inv_2dy, J[1]);
}

template <int L, int STAGE, int LY, bool NI>
__device__ __forceinline__ double march_pair_strip(const StageArgsDelta& a, const MarchTmaMaps& m,
                                                   int x0, int y0, int lane, unsigned char* wbase)
{
    using T = float;
    using P = PolicyDelta<STAGE>;
    using Raw = typename P::Raw;
    using Lay = MarchPairLayout<STAGE>;
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

    int gx[2], sx[2];
    bool in_x[2], own[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        gx[j] = x0 - 2 + 2 * lane + j;
        sx[j] = map_index(gx[j], g.nx, g.bc_x);
        in_x[j] = gx[j] >= 0 && gx[j] < g.nx;
        own[j] = lane >= 1 && lane <= 30 && gx[j] < g.nx;
    }
    const int y1 = min(y0 + LY, g.ny);
    const int nrows = y1 - y0;

    const T* halo_f = reinterpret_cast<const T*>(wbase);
    const T* own_f = reinterpret_cast<const T*>(wbase + 2 * Lay::kHaloSlot);
    const uint32_t halo_s = smem_addr(wbase);
    const uint32_t own_s = halo_s + 2 * Lay::kHaloSlot;
    const uint32_t bar_s = halo_s + Lay::kBarOff; // halo: +0, +8; own: +16, +24

    if (lane == 0) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            mbar_init(bar_s + 8 * b, 1);
        }
        fence_mbar_init();
    }
    __syncwarp();

    const uint32_t stall = (x0 == 0 && y0 == 0) ? static_cast<uint32_t>(k.stall_tx) : 0u;
    // Item i of the halo stream is row y0 + 2 + i, of the own stream row y0 + i; both use slot
    // i & 1, whose (i >> 1)-th phase completes it.
    auto issue_halo = [&](int i) {
        const uint32_t slot = static_cast<uint32_t>(i & 1);
        const uint32_t bar = bar_s + 8 * slot;
        const int yy = map_index(y0 + 2 + i, g.ny, g.bc_y);
        mbar_arrive_expect_tx(bar, Lay::kHaloBytes + (i == 0 ? stall : 0u));
        tma_load_3d(halo_s + slot * Lay::kHaloSlot, &m.in_halo, bar, x0 - 4, yy, 0);
        if constexpr (STAGE == 2) {
            tma_load_3d(halo_s + slot * Lay::kHaloSlot + Lay::kHaloBoxSlot, &m.delta_halo, bar,
                        x0 - 4, yy, 0);
        }
    };
    auto issue_own = [&](int i) {
        if constexpr (STAGE == 2) {
            const uint32_t slot = static_cast<uint32_t>(i & 1);
            const uint32_t bar = bar_s + 16 + 8 * slot;
            const uint32_t dst = own_s + slot * Lay::kOwnSlot;
            mbar_arrive_expect_tx(bar, Lay::kOwnTx);
            tma_load_3d(dst, &m.in_own, bar, x0, y0 + i, 0);
            tma_load_3d(dst + Lay::kOwnBOff, &m.out_own, bar, x0, y0 + i, 0);
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
    own_issued = STAGE == 2 ? halo_issued : 0;

    auto load = [&](int j, int y, Raw& r) {
        P::load_raw(a, g, sx[j], map_index(y, g.ny, g.bc_y), r);
    };
    auto prim = [&](int j, int y, const Raw& r, T (&w)[9]) {
        P::template raw_prim<STAGE, false>(a, g, sx[j], map_index(y, g.ny, g.bc_y), r, k, w);
    };

    // Prologue (direct loads): rows y0-2 .. y0+1, slopes of rows y0-1 and y0, flux G(y0 - 1/2).
    T Wm[2][9], Wp[2][9], sYc[2][9], Gm[2][9];
    T Jc[2][NI ? 3 : 1];
    {
        T wa[2][9], wb[2][9], sYm[2][9];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            Raw r0, r1, r2, r3;
            load(j, y0 - 2, r0);
            load(j, y0 - 1, r1);
            load(j, y0, r2);
            load(j, y0 + 1, r3);
            prim(j, y0 - 2, r0, wa[j]);
            prim(j, y0 - 1, r1, wb[j]);
            prim(j, y0, r2, Wm[j]);
            prim(j, y0 + 1, r3, Wp[j]);
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                sYm[j][c] = limit_half_slope<L>(wb[j][c] - wa[j][c], Wm[j][c] - wb[j][c]);
                sYc[j][c] = limit_half_slope<L>(Wm[j][c] - wb[j][c], Wp[j][c] - Wm[j][c]);
            }
            face_flux_regs<T, true, true>(wb[j], sYm[j], Wm[j], sYc[j], gamma, inv_gm1, c_h,
                                          Gm[j]);
        }
        if constexpr (NI) {
            T Jb[2][3];
            pair_current(wa, wb, Wm, inv_2dx, inv_2dy, Jb);
            pair_current(wb, Wm, Wp, inv_2dx, inv_2dy, Jc);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                march_nonideal_y(Jb[j], wb[j], Jc[j], Wm[j], k.ni, Gm[j]);
            }
        }
    }

    double smax = 0.0;
    bool failed = false;
    // own-box column of column A (lanes 1..30; the other lanes read no own operand)
    const int oc = (lane >= 1 && lane <= 30) ? 2 * lane - 2 : 0;
#pragma unroll 1
    for (int i = 0; i < nrows; ++i) {
        const int y = y0 + i;
        // row y + 2 from the halo stream
        Raw rn[2];
        {
            const uint32_t slot = static_cast<uint32_t>(i & 1);
            const bool ok = mbar_wait(bar_s + 8 * slot, static_cast<uint32_t>((i >> 1) & 1));
            if (__any_sync(kFull, !ok)) {
                failed = true;
                break;
            }
            halo_done = i + 1;
            const T* src = halo_f + slot * (Lay::kHaloSlot / sizeof(T)) + 2 * lane + 2;
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                const float2 v = *reinterpret_cast<const float2*>(src + c * kPairHaloW);
                rn[0].v[c] = v.x;
                rn[1].v[c] = v.y;
                if constexpr (STAGE == 2) { // U* hi = fl(hi(U^n) + delta)
                    const float2 d = *reinterpret_cast<const float2*>(
                        src + Lay::kHaloBoxSlot / sizeof(T) + c * kPairHaloW);
                    rn[0].v[c] = __fadd_rn(rn[0].v[c], d.x);
                    rn[1].v[c] = __fadd_rn(rn[1].v[c], d.y);
                }
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (!in_x[j]) {
                    load(j, y + 2, rn[j]);
                }
            }
            __syncwarp();
            if (i + 2 < nrows) {
                if (lane == 0) {
                    issue_halo(i + 2);
                }
                halo_issued = i + 3;
            }
        }
        T W2[2][9];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            prim(j, y + 2, rn[j], W2[j]);
        }
        // x sweep of row y: dF = F(x + 1/2) - F(x - 1/2) for both columns
        T dF[2][9];
        {
            T An[9], sA[9], sB[9], sAn[9], FA[9], FB[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                An[c] = __shfl_down_sync(kFull, Wm[0][c], 1);
                const T Bp = __shfl_up_sync(kFull, Wm[1][c], 1);
                const T dAB = Wm[1][c] - Wm[0][c];
                sA[c] = limit_half_slope<L>(Wm[0][c] - Bp, dAB);
                sB[c] = limit_half_slope<L>(dAB, An[c] - Wm[1][c]);
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                sAn[c] = __shfl_down_sync(kFull, sA[c], 1);
            }
            face_flux_regs<T, false, true>(Wm[0], sA, Wm[1], sB, gamma, inv_gm1, c_h, FA);
            face_flux_regs<T, false, true>(Wm[1], sB, An, sAn, gamma, inv_gm1, c_h, FB);
            if constexpr (NI) {
                const T jx = __shfl_down_sync(kFull, Jc[0][0], 1);
                const T jy = __shfl_down_sync(kFull, Jc[0][1], 1);
                const T jz = __shfl_down_sync(kFull, Jc[0][2], 1);
                add_nonideal_face<T, false>(Jc[0][0], Jc[0][1], Jc[0][2], Jc[1][0], Jc[1][1],
                                            Jc[1][2], Wm[0][5], Wm[0][6], Wm[0][7], Wm[1][5],
                                            Wm[1][6], Wm[1][7], k.ni, FA);
                add_nonideal_face<T, false>(Jc[1][0], Jc[1][1], Jc[1][2], jx, jy, jz, Wm[1][5],
                                            Wm[1][6], Wm[1][7], An[5], An[6], An[7], k.ni, FB);
            }
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                dF[0][c] = FA[c] - __shfl_up_sync(kFull, FB[c], 1);
                dF[1][c] = FB[c] - FA[c];
            }
        }
        // y faces y + 1/2 of both columns
        T sYn[2][9], Gp[2][9];
        T Jn[2][NI ? 3 : 1];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                sYn[j][c] = limit_half_slope<L>(Wp[j][c] - Wm[j][c], W2[j][c] - Wp[j][c]);
            }
            face_flux_regs<T, true, true>(Wm[j], sYc[j], Wp[j], sYn[j], gamma, inv_gm1, c_h,
                                          Gp[j]);
        }
        if constexpr (NI) {
            pair_current(Wm, Wp, W2, inv_2dx, inv_2dy, Jn);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                march_nonideal_y(Jc[j], Wm[j], Jn[j], Wp[j], k.ni, Gp[j]);
            }
        }
        // own-cell operands of row y from the own stream (stage 2), then the stage updates
        {
            const uint32_t slot = static_cast<uint32_t>(i & 1);
            if constexpr (STAGE == 2) {
                const bool ok = mbar_wait(bar_s + 16 + 8 * slot,
                                          static_cast<uint32_t>((i >> 1) & 1));
                if (__any_sync(kFull, !ok)) {
                    failed = true;
                    break;
                }
                own_done = i + 1;
            }
            const T* osrc = own_f + slot * (Lay::kOwnSlot / sizeof(T)) + oc;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                if (own[j]) {
                    T Lc[9];
#pragma unroll
                    for (int c = 0; c < 9; ++c) {
                        Lc[c] = -dF[j][c] * inv_dx - (Gp[j][c] - Gm[j][c]) * inv_dy; // include/mhd/rhs.hpp:121
                    }
                    if (psi_damp != 0.0) {
                        Lc[8] -= static_cast<T>(psi_damp) * Wm[j][8]; // include/mhd/rhs.hpp:219-225
                    }
                    // own operand q: delta (q < 9), then U^n's hi and lo planes (q < 27)
                    P::template update_ops<STAGE>(a, g, gx[j], y, false, Lc, dt, k, smax,
                                                  [&](int q) {
                                                      return q < 9
                                                                 ? osrc[j + q * kPairOwnW]
                                                                 : osrc[Lay::kOwnBOff / sizeof(T) +
                                                                        j + (q - 9) * kPairOwnW];
                                                  });
                }
            }
            __syncwarp();
            if (i + 2 < nrows) {
                if (lane == 0) {
                    issue_own(i + 2);
                }
                if constexpr (STAGE == 2) {
                    own_issued = i + 3;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                Wm[j][c] = Wp[j][c];
                Wp[j][c] = W2[j][c];
                sYc[j][c] = sYn[j][c];
                Gm[j][c] = Gp[j][c];
            }
            if constexpr (NI) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    Jc[j][c] = Jn[j][c];
                }
            }
        }
    }
    if (failed) {
        // Record the failure and let every copy of this warp land before the CTA can exit.
        if (lane == 0) {
            atomicOr(&a.ctrl->status, static_cast<int>(kStatusWaitTimeout));
        }
        for (int j = halo_done; j < halo_issued; ++j) {
            mbar_wait(bar_s + 8 * (j & 1), static_cast<uint32_t>((j >> 1) & 1));
        }
        for (int j = own_done; j < own_issued; ++j) {
            mbar_wait(bar_s + 16 + 8 * (j & 1), static_cast<uint32_t>((j >> 1) & 1));
        }
        return 0.0;
    }
    __syncwarp();
    if (lane == 0) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            mbar_inval(bar_s + 8 * b);
        }
    }
    __syncwarp();
    return smax;
}

// One warp per block, one 60-column strip segment of LY rows per warp.
template <int L, int STAGE, int LY, int MINB, bool NI>
__global__ void __launch_bounds__(32, MINB) march_pair_kernel(const StageArgsDelta a,
                                                              const __grid_constant__ MarchTmaMaps m)
{
    if (a.ctrl->finished != 0) {
        return;
    }
    extern __shared__ unsigned char march_smem[];
    const int lane = threadIdx.x & 31;
    unsigned char* base = march_smem + ((128u - (smem_addr(march_smem) & 127u)) & 127u);
    const int x0 = static_cast<int>(blockIdx.x) * kPairOwned;
    double smax = 0.0;
    if (x0 < a.geom.nx) { // warp-uniform
        smax = march_pair_strip<L, STAGE, LY, NI>(a, m, x0, static_cast<int>(blockIdx.y) * LY,
                                                  lane, base);
    }
    if constexpr (STAGE == 2) {
        reduce_signal_speed_and_finish(smax, a.ctrl, a.k, gridDim.x * gridDim.y, true);
    }
}

} // namespace mhdb
