// Instantiation helpers shared by kernels_f64.cu and kernels_mixed.cu.
#pragma once

#include <type_traits>

#include "march_kernel.cuh"
#include "march_pair.cuh"
#include "march_tma.cuh"
#include "stage_kernel.cuh"
#include "stage_select.h"

namespace mhdb {

template <int TX_, int TY_, int NT_, int MINB_, bool MERGED_ = false>
struct TileCfg {
    static constexpr int TX = TX_, TY = TY_, NT = NT_, MINB = MINB_;
    static constexpr bool MERGED = MERGED_;
};

template <class Policy, class Cfg, int L, bool NI, bool MASK>
void fill_pair_tile(StageKernels& k)
{
    using T = typename Policy::T;
    auto s1 = stage_kernel<Policy, L, NI, MASK, 1, Cfg::TX, Cfg::TY, Cfg::NT, Cfg::MINB, Cfg::MERGED>;
    auto s2 = stage_kernel<Policy, L, NI, MASK, 2, Cfg::TX, Cfg::TY, Cfg::NT, Cfg::MINB, Cfg::MERGED>;
    if constexpr (sizeof(T) == 8) {
        k.f64_stage1 = s1;
        k.f64_stage2 = s2;
    } else {
        k.mx_stage1 = s1;
        k.mx_stage2 = s2;
    }
    k.tile_x = Cfg::TX;
    k.tile_y = Cfg::TY;
    k.threads = Cfg::NT;
    k.smem = stage_smem_bytes<T, Cfg::TX, Cfg::TY, NI, Cfg::MERGED>();
    k.smem2 = k.smem;
}

// Strip-march configuration: NW warps per block, LY rows per warp, MINB blocks per SM.
template <int NW_, int LY_, int MINB_>
struct MarchCfg {
    static constexpr int NW = NW_, LY = LY_, MINB = MINB_;
    static constexpr bool MARCH = true;
};

// TMA-fed strip-march configuration: NW warps per block, LY rows per warp, MINB blocks per SM.
template <int NW_, int LY_, int MINB_, bool HF_ = true, int ST1_ = 1, int ST2_ = 0,
          int DELTA_ = 0>
struct MarchTmaCfg {
    static constexpr int NW = NW_, LY = LY_, MINB = MINB_;
    static constexpr bool HF = HF_; // wait for the halo row before the x sweep
    static constexpr int ST1 = ST1_; // stage 1: 0 lane stores, 1 or 2 staging slots of TMA stores
    static constexpr int ST2 = ST2_; // the same for stage 2
    // FP32-mixed increment form (stage_delta.cuh): 0 no, 1 yes, 2 with stage 2's own-cell delta
    // taken from the halo stream (MarchTmaLayout kind 2)
    static constexpr int DELTA = DELTA_;
    static constexpr bool MARCH_TMA = true;
};

// Two-column TMA strip march of the increment form (march_pair.cuh): one warp per block, LY rows
// per warp, MINB blocks per SM.
template <int LY_, int MINB_>
struct MarchPairCfg {
    static constexpr int LY = LY_, MINB = MINB_;
    static constexpr bool MARCH_PAIR = true;
};

template <class Cfg, class = void>
struct is_march_pair : std::false_type {};
template <class Cfg>
struct is_march_pair<Cfg, std::void_t<decltype(Cfg::MARCH_PAIR)>> : std::true_type {};

template <class Cfg, class = void>
struct is_march_tma : std::false_type {};
template <class Cfg>
struct is_march_tma<Cfg, std::void_t<decltype(Cfg::MARCH_TMA)>> : std::true_type {};

template <class Cfg, class = void>
struct is_march : std::false_type {};
template <class Cfg>
struct is_march<Cfg, std::void_t<decltype(Cfg::MARCH)>> : std::true_type {};

template <class Policy, class Cfg, int L, bool NI, bool MASK>
void fill_pair(StageKernels& k)
{
    if constexpr (is_march_pair<Cfg>::value) {
        static_assert(!MASK, "the two-column strip march serves unmasked solves");
        static_assert(sizeof(typename Policy::T) == 4, "the two-column strip march is FP32-mixed");
        k.dx_tma1 = march_pair_kernel<L, 1, Cfg::LY, Cfg::MINB, NI>;
        k.dx_tma2 = march_pair_kernel<L, 2, Cfg::LY, Cfg::MINB, NI>;
        k.tile_x = kPairOwned;
        k.tile_y = Cfg::LY;
        k.threads = 32;
        k.smem = march_pair_smem_bytes<1>();
        k.smem2 = march_pair_smem_bytes<2>();
        k.halo_w = kPairHaloW;
        k.own_w = kPairOwnW;
        return;
    } else if constexpr (is_march_tma<Cfg>::value) {
        static_assert(!MASK || (Cfg::ST1 == 0 && Cfg::ST2 == 0),
                      "masked TMA strip marches store through the lanes");
        constexpr int E = static_cast<int>(sizeof(typename Policy::T));
        if constexpr (E == 8) {
            static_assert(Cfg::ST1 == 0 && Cfg::ST2 == 0,
                          "the FP64 TMA strip march stores through the lanes");
            k.f64_tma1 = march_tma_kernel<L, 1, Cfg::LY, Cfg::NW, Cfg::MINB, Cfg::HF, 0, NI, MASK,
                                          Policy>;
            k.f64_tma2 = march_tma_kernel<L, 2, Cfg::LY, Cfg::NW, Cfg::MINB, Cfg::HF, 0, NI, MASK,
                                          Policy>;
        } else if constexpr (Cfg::DELTA) {
            static_assert(Cfg::ST1 == 0 && Cfg::ST2 == 0, "the increment form stores through the lanes");
            k.dx_tma1 = march_tma_kernel<L, 1, Cfg::LY, Cfg::NW, Cfg::MINB, Cfg::HF, 0, NI, MASK,
                                         PolicyDelta<1>>;
            k.dx_tma2 = march_tma_kernel<L, 2, Cfg::LY, Cfg::NW, Cfg::MINB, Cfg::HF, 0, NI, MASK,
                                         PolicyDelta<2, Cfg::DELTA>>;
        } else {
            k.mx_tma1 = march_tma_kernel<L, 1, Cfg::LY, Cfg::NW, Cfg::MINB, Cfg::HF, Cfg::ST1, NI, MASK>;
            k.mx_tma2 = march_tma_kernel<L, 2, Cfg::LY, Cfg::NW, Cfg::MINB, Cfg::HF, Cfg::ST2, NI, MASK>;
        }
        constexpr int K = Cfg::DELTA;
        k.tile_x = Cfg::NW * kMarchOwned;
        k.tile_y = Cfg::LY;
        k.threads = Cfg::NW * 32;
        k.smem = march_tma_smem_bytes<1, Cfg::ST1, E, (K > 0 ? 1 : 0)>(Cfg::NW);
        k.smem2 = march_tma_smem_bytes<2, Cfg::ST2, E, K>(Cfg::NW);
        return;
    } else if constexpr (is_march<Cfg>::value) {
        static_assert(!MASK, "the strip-march kernel serves unmasked solves");
        using T = typename Policy::T;
        auto s1 = march_kernel<Policy, L, 1, Cfg::LY, Cfg::NW, Cfg::MINB, NI>;
        auto s2 = march_kernel<Policy, L, 2, Cfg::LY, Cfg::NW, Cfg::MINB, NI>;
        if constexpr (sizeof(T) == 8) {
            k.f64_stage1 = s1;
            k.f64_stage2 = s2;
        } else {
            k.mx_stage1 = s1;
            k.mx_stage2 = s2;
        }
        k.tile_x = Cfg::NW * kMarchOwned;
        k.tile_y = Cfg::LY;
        k.threads = Cfg::NW * 32;
        k.smem = 0;
        k.smem2 = 0;
        return;
    } else {
        fill_pair_tile<Policy, Cfg, L, NI, MASK>(k);
    }
}

// Every (limiter, non-ideal, mask) combination: the default configuration and the TMA strip
// march that stores through the lanes.
template <class Policy, class Cfg>
StageKernels select_full(int lim, bool ni, bool mask)
{
    StageKernels k;
#define MHDB_SEL(LL)                                                                               \
    if (ni) {                                                                                      \
        if (mask) fill_pair<Policy, Cfg, LL, true, true>(k);                                       \
        else fill_pair<Policy, Cfg, LL, true, false>(k);                                           \
    } else {                                                                                       \
        if (mask) fill_pair<Policy, Cfg, LL, false, true>(k);                                      \
        else fill_pair<Policy, Cfg, LL, false, false>(k);                                          \
    }
    if (lim == kMinmod) {
        MHDB_SEL(kMinmod)
    } else if (lim == kMC) {
        MHDB_SEL(kMC)
    } else {
        MHDB_SEL(kVanLeer)
    }
#undef MHDB_SEL
    return k;
}

// Tuning configurations: unmasked solves; the shared-memory tile configurations other than the
// default serve ideal solves only, the strip-march ones ideal and non-ideal solves.
template <class Policy, class Cfg>
StageKernels select_unmasked(int lim, bool ni, bool mask)
{
    StageKernels k;
    if (mask) {
        return k;
    }
    if constexpr (is_march<Cfg>::value || is_march_tma<Cfg>::value || is_march_pair<Cfg>::value) {
#define MHDB_SEL(LL)                                                                               \
    if (ni) fill_pair<Policy, Cfg, LL, true, false>(k);                                            \
    else fill_pair<Policy, Cfg, LL, false, false>(k);
        if (lim == kMinmod) {
            MHDB_SEL(kMinmod)
        } else if (lim == kMC) {
            MHDB_SEL(kMC)
        } else {
            MHDB_SEL(kVanLeer)
        }
#undef MHDB_SEL
        return k;
    } else {
        if (ni) {
            return k;
        }
        if (lim == kMinmod) {
            fill_pair<Policy, Cfg, kMinmod, false, false>(k);
        } else if (lim == kMC) {
            fill_pair<Policy, Cfg, kMC, false, false>(k);
        } else {
            fill_pair<Policy, Cfg, kVanLeer, false, false>(k);
        }
        return k;
    }
}

} // namespace mhdb
