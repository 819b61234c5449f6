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
constexpr TileConfigInfo kInfo[] = {{32, 8, 256, 2, kKindTile},    {32, 4, 128, 4, kKindTile},
                                    {32, 8, 320, 2, kKindTile},    {32, 8, 320, 2, kKindTileMerged},
                                    {112, 64, 128, 2, kKindMarch}, {112, 64, 128, 3, kKindMarch}};
constexpr int kCount = sizeof(kInfo) / sizeof(kInfo[0]);
} // namespace

int stage_config_count_f64() { return kCount; }

// Without a chosen configuration the FP64 form runs the shared-memory tile kernel.
int default_stage_config_f64(long long, bool) { return 0; }

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
    default:
        return select_full<PolicyF64, Cfg0>(limiter, nonideal, mask);
    }
}

} // namespace mhdb
