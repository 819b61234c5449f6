// Stage-kernel instantiations of the plain FP64 form.
#include "kernel_table.cuh"

namespace mhdb {

namespace {
using Cfg0 = TileCfg<32, 8, 256, 2>; // default
using Cfg1 = TileCfg<32, 4, 128, 4>;
using Cfg2 = TileCfg<32, 8, 320, 2>;
using Cfg3 = TileCfg<32, 8, 320, 2, true>;
using Cfg4 = MarchCfg<4, 64, 2>;
using Cfg5 = MarchCfg<4, 64, 3>;
using Cfg6 = MarchTmaCfg<1, 32, 8, true, 0, 0>;
using Cfg7 = MarchTmaCfg<1, 32, 10, true, 0, 0>;
constexpr TileConfigInfo kInfo[] = {{32, 8, 256, 2, kKindTile},    {32, 4, 128, 4, kKindTile},
                                    {32, 8, 320, 2, kKindTile},    {32, 8, 320, 2, kKindTileMerged},
                                    {112, 64, 128, 2, kKindMarch}, {112, 64, 128, 3, kKindMarch},
                                    {28, 32, 32, 8, kKindMarchTma}, {28, 32, 32, 10, kKindMarchTma}};
constexpr int kCount = sizeof(kInfo) / sizeof(kInfo[0]);
} // namespace

int stage_config_count_f64() { return kCount; }

// Without a chosen configuration: FP64 grids of at least 2048^2 cells run the TMA strip march
// (configuration 7: 10 one-warp blocks per SM, masked grids included); smaller ones the 320-thread
// tile kernel (configuration 2; non-ideal solves then run configuration 0), smaller masked grids
// configuration 0.
int default_stage_config_f64(long long cells, bool mask)
{
    if (cells >= 2048LL * 2048) {
        return 7;
    }
    return mask ? 0 : 2;
}

TileConfigInfo stage_config_info_f64(int c) { return kInfo[c < 0 || c >= kCount ? 0 : c]; }

StageKernels select_stage_f64(int limiter, bool nonideal, bool mask, int config)
{
    switch (config) {
    case 1:
        return select_unmasked<PolicyF64, Cfg1>(limiter, nonideal, mask);
    case 2:
        return select_unmasked<PolicyF64, Cfg2>(limiter, nonideal, mask);
    case 3:
        return select_unmasked<PolicyF64, Cfg3>(limiter, nonideal, mask);
    case 4:
        return select_unmasked<PolicyF64, Cfg4>(limiter, nonideal, mask);
    case 5:
        return select_unmasked<PolicyF64, Cfg5>(limiter, nonideal, mask);
    case 6:
        return select_unmasked<PolicyF64, Cfg6>(limiter, nonideal, mask);
    case 7:
        return select_full<PolicyF64, Cfg7>(limiter, nonideal, mask);
    default:
        return select_full<PolicyF64, Cfg0>(limiter, nonideal, mask);
    }
}

} // namespace mhdb
