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
constexpr TileConfigInfo kInfo[] = {{32, 16, 256, 2, 0}, {32, 16, 256, 3, 0}, {32, 8, 256, 3, 0},
                                    {32, 16, 384, 2, 1}, {32, 16, 256, 2, 1}, {32, 8, 320, 3, 1}};
constexpr int kCount = sizeof(kInfo) / sizeof(kInfo[0]);
} // namespace

int stage_config_count_mixed() { return kCount; }

TileConfigInfo stage_config_info_mixed(int c) { return kInfo[c < 0 || c >= kCount ? 0 : c]; }

StageKernels select_stage_mixed(int limiter, bool nonideal, bool mask, int config)
{
    switch (config) {
    case 1:
        return select_ideal<PolicyMixed, Cfg1>(limiter, nonideal, mask);
    case 2:
        return select_ideal<PolicyMixed, Cfg2>(limiter, nonideal, mask);
    case 3:
        return select_ideal<PolicyMixed, Cfg3>(limiter, nonideal, mask);
    case 4:
        return select_ideal<PolicyMixed, Cfg4>(limiter, nonideal, mask);
    case 5:
        return select_ideal<PolicyMixed, Cfg5>(limiter, nonideal, mask);
    default:
        return select_full<PolicyMixed, Cfg0>(limiter, nonideal, mask);
    }
}

} // namespace mhdb
