// Stage-kernel instantiations of the FP32-mixed form.
#include "kernel_table.cuh"

namespace mhdb {

namespace {
using Cfg0 = TileCfg<32, 16, 256, 2>; // default
using Cfg1 = TileCfg<32, 16, 256, 3>;
using Cfg2 = TileCfg<32, 8, 256, 3>;
using Cfg3 = TileCfg<32, 16, 384, 2, true>;
using Cfg4 = TileCfg<32, 16, 256, 2, true>;
using Cfg5 = TileCfg<32, 8, 320, 3, true>;
using Cfg6 = MarchCfg<4, 64, 3>;
using Cfg7 = MarchTmaCfg<4, 32, 4>;
using Cfg8 = MarchTmaCfg<2, 32, 8>;
using Cfg9 = MarchTmaCfg<1, 32, 16>;
using Cfg10 = MarchTmaCfg<4, 32, 4, true, 0>;
using Cfg11 = MarchTmaCfg<1, 32, 16, true, 0>;
using Cfg12 = MarchTmaCfg<1, 64, 16>;
using Cfg13 = MarchTmaCfg<1, 32, 16, true, 0, 0, 1>; // increment form (also masked)
using Cfg14 = MarchTmaCfg<1, 64, 16, true, 0, 0, 1>; // increment form, 64-row segments
using Cfg15 = MarchPairCfg<32, 8>;  // increment form, two columns per lane
using Cfg16 = MarchPairCfg<32, 10>; // the same, 10 blocks per SM requested (168 registers)
// increment form, stage 2's own-cell delta from the halo stream (also masked)
using Cfg17 = MarchTmaCfg<1, 32, 16, true, 0, 0, 2>;
constexpr TileConfigInfo kInfo[] = {
    {32, 16, 256, 2, kKindTile},       {32, 16, 256, 3, kKindTile},
    {32, 8, 256, 3, kKindTile},        {32, 16, 384, 2, kKindTileMerged},
    {32, 16, 256, 2, kKindTileMerged}, {32, 8, 320, 3, kKindTileMerged},
    {112, 64, 128, 3, kKindMarch},     {112, 32, 128, 4, kKindMarchTma},
    {56, 32, 64, 8, kKindMarchTma},    {28, 32, 32, 16, kKindMarchTma},
    {112, 32, 128, 4, kKindMarchTma},  {28, 32, 32, 16, kKindMarchTma},
    {28, 64, 32, 16, kKindMarchTma},   {28, 32, 32, 16, kKindMarchTmaDelta},
    {28, 64, 32, 16, kKindMarchTmaDelta}, {60, 32, 32, 8, kKindMarchTmaPair},
    {60, 32, 32, 10, kKindMarchTmaPair}, {28, 32, 32, 16, kKindMarchTmaDelta}};
constexpr int kCount = sizeof(kInfo) / sizeof(kInfo[0]);
} // namespace

int stage_config_count_mixed() { return kCount; }

// Without a chosen configuration: grids of at least 1024^2 cells run the TMA strip march with one
// warp per block, unmasked ones in the increment form with stage 2's own-cell increment taken
// from the halo stream (configuration 17), masked ones in the stored form that also serves masks
// (configuration 11); smaller grids have too few 28-column strips to fill the GPU with it and run
// the shared-memory tile kernel.
int default_stage_config_mixed(long long cells, bool mask)
{
    return cells >= 1024LL * 1024 ? (mask ? 11 : 17) : 0;
}

TileConfigInfo stage_config_info_mixed(int c) { return kInfo[c < 0 || c >= kCount ? 0 : c]; }

StageKernels select_stage_mixed(int limiter, bool nonideal, bool mask, int config)
{
    switch (config) {
    case 1:
        return select_unmasked<PolicyMixed, Cfg1>(limiter, nonideal, mask);
    case 2:
        return select_unmasked<PolicyMixed, Cfg2>(limiter, nonideal, mask);
    case 3:
        return select_unmasked<PolicyMixed, Cfg3>(limiter, nonideal, mask);
    case 4:
        return select_unmasked<PolicyMixed, Cfg4>(limiter, nonideal, mask);
    case 5:
        return select_unmasked<PolicyMixed, Cfg5>(limiter, nonideal, mask);
    case 6:
        return select_unmasked<PolicyMixed, Cfg6>(limiter, nonideal, mask);
    case 7:
        return select_unmasked<PolicyMixed, Cfg7>(limiter, nonideal, mask);
    case 8:
        return select_unmasked<PolicyMixed, Cfg8>(limiter, nonideal, mask);
    case 9:
        return select_unmasked<PolicyMixed, Cfg9>(limiter, nonideal, mask);
    case 10:
        return select_unmasked<PolicyMixed, Cfg10>(limiter, nonideal, mask);
    case 11:
        return select_full<PolicyMixed, Cfg11>(limiter, nonideal, mask);
    case 12:
        return select_unmasked<PolicyMixed, Cfg12>(limiter, nonideal, mask);
    case 13:
        return select_full<PolicyMixed, Cfg13>(limiter, nonideal, mask);
    case 14:
        return select_unmasked<PolicyMixed, Cfg14>(limiter, nonideal, mask);
    case 15:
        return select_unmasked<PolicyMixed, Cfg15>(limiter, nonideal, mask);
    case 16:
        return select_unmasked<PolicyMixed, Cfg16>(limiter, nonideal, mask);
    case 17:
        return select_full<PolicyMixed, Cfg17>(limiter, nonideal, mask);
    default:
        return select_full<PolicyMixed, Cfg0>(limiter, nonideal, mask);
    }
}

} // namespace mhdb
