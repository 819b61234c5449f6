// Host-side table of the compiled stage-kernel instantiations. Each precision form is compiled
// in its own translation unit (kernels_f64.cu, kernels_mixed.cu) for a few configurations of the
// shared-memory tile kernel (stage_kernel.cuh) and of the warp strip-march kernel
// (march_kernel.cuh); configuration 0 is the default tile kernel and the only one instantiated
// for every combination of limiter, non-ideal terms and mask. The other configurations exist for
// the ideal, unmasked case and are chosen by the autotuner per grid size class.
#pragma once

#include <cstddef>
#include <string>

#include "stage_f64.cuh"
#include "stage_delta.cuh"
#include "stage_mixed.cuh"
#include "tma.cuh"

namespace mhdb {

using StageFnF64 = void (*)(StageArgsF64);
using StageFnMx = void (*)(StageArgsMx);
using StageFnMxTma = void (*)(StageArgsMx, MarchTmaMaps); // TMA-fed kernels take tensor maps
using StageFnF64Tma = void (*)(StageArgsF64, MarchTmaMaps);
using StageFnDeltaTma = void (*)(StageArgsDelta, MarchTmaMaps); // increment form

struct StageKernels {
    StageFnF64 f64_stage1 = nullptr, f64_stage2 = nullptr;
    StageFnMx mx_stage1 = nullptr, mx_stage2 = nullptr;
    StageFnMxTma mx_tma1 = nullptr, mx_tma2 = nullptr;
    StageFnF64Tma f64_tma1 = nullptr, f64_tma2 = nullptr;
    StageFnDeltaTma dx_tma1 = nullptr, dx_tma2 = nullptr; // FP32-mixed increment form
    int tile_x = 0, tile_y = 0, threads = 0; // threads == 0: no such configuration
    size_t smem = 0, smem2 = 0;               // dynamic shared memory per block, stage 1 and 2
    int halo_w = kTmaHaloW, own_w = kTmaOwnW; // TMA box widths of the increment form's maps
};

enum StageKernelKind : int {
    kKindTile = 0,
    kKindTileMerged = 1,
    kKindMarch = 2,
    kKindMarchTma = 3,
    kKindMarchTmaDelta = 4, // TMA strip march of the increment form (stage_delta.cuh)
    kKindMarchTmaPair = 5   // its two-column form (march_pair.cuh)
};

// tile_x x tile_y: interior cells one block covers (strip march: warps x 28 columns, or 60 for
// the two-column form, by the rows of a warp's segment).
struct TileConfigInfo {
    int tile_x, tile_y, threads, min_blocks, kind;
};

// Number of tile configurations compiled per precision form, and their shapes.
int stage_config_count_f64();
int stage_config_count_mixed();
// Configuration used when none is chosen (mhdb_set_tile_config(h, -1), the default).
int default_stage_config_f64(long long cells, bool mask);
int default_stage_config_mixed(long long cells, bool mask);
TileConfigInfo stage_config_info_f64(int config);
TileConfigInfo stage_config_info_mixed(int config);

// Kernels of one configuration; threads == 0 when the configuration does not serve the
// combination (configurations other than 0 serve unmasked solves, and masked ones where they
// store through the lanes).
// Tensor maps of one TMA strip-march stage reading `in` and writing `out` (tma_maps.cu); false
// with a message when the driver cannot encode them.
bool encode_march_maps(const MixedState& in, const MixedState& out, const Geometry& g,
                       MarchTmaMaps* maps, std::string* err);
// The same for the FP64 state (9 double planes).
bool encode_march_maps_f64(const double* in, const double* out, const Geometry& g,
                           MarchTmaMaps* maps, std::string* err);
// Both stages' tensor maps of the increment form: U^n (18 float planes) and the increment
// (9 float planes).
bool encode_march_maps_delta(const MixedState& un, float* delta, const Geometry& g,
                             MarchTmaMaps* stage1, MarchTmaMaps* stage2, std::string* err,
                             unsigned halo_w = kTmaHaloW, unsigned own_w = kTmaOwnW);

StageKernels select_stage_f64(int limiter, bool nonideal, bool mask, int config);
StageKernels select_stage_mixed(int limiter, bool nonideal, bool mask, int config);

} // namespace mhdb
