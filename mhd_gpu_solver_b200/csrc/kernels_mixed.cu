// Stage-kernel instantiations of the FP32-mixed form.
#include "kernel_table.cuh"

namespace mhdb {

namespace {
using Cfg0 = TileCfg<32, 16, 256, 2>; // default
using Cfg1 = TileCfg<32, 16, 256, 3>;
using Cfg2 = TileCfg<32, 8, 256, 3>;
using Cfg3 = TileCfg<32, 16, 512, 1>;
constexpr TileConfigInfo kInfo[] = {
    {32, 16, 256, 2}, {32, 16, 256, 3}, {32, 8, 256, 3}, {32, 16, 512, 1}};
} // namespace

int stage_config_count_mixed() { return 4; }

TileConfigInfo stage_config_info_mixed(int c) { return kInfo[c < 0 || c > 3 ? 0 : c]; }

StageKernels select_stage_mixed(int limiter, bool nonideal, bool mask, int config)
{
    switch (config) {
    case 1:
        return select_ideal<PolicyMixed, Cfg1>(limiter, nonideal, mask);
    case 2:
        return select_ideal<PolicyMixed, Cfg2>(limiter, nonideal, mask);
    case 3:
        return select_ideal<PolicyMixed, Cfg3>(limiter, nonideal, mask);
    default:
        return select_full<PolicyMixed, Cfg0>(limiter, nonideal, mask);
    }
}

} // namespace mhdb
