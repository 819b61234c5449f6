// Host side of the TMA strip march: tensor maps of a state, encoded with the driver's
// cuTensorMapEncodeTiled (looked up through the runtime, so the library does not link libcuda).
#include "stage_select.h"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <string>

namespace mhdb {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        const cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000,
                                                               cudaEnableDefault, &q);
        return (e == cudaSuccess && q == cudaDriverEntryPointSuccess)
                   ? reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p)
                   : nullptr;
    }();
    return fn;
}

// 3D tensor map (x, y, plane) over `planes` planes of a state at `base`: extent nx x ny x planes,
// row stride pitch elements, plane stride g.plane elements; elements outside the extent read as
// 0 and are not written. FP32-mixed state: 18 float planes (hi, then lo); FP64: 9 double planes.
bool state_tensor_map(void* base, bool fp64, unsigned planes, const Geometry& g, unsigned box_x,
                      unsigned box_planes, CUtensorMap* map, std::string* err)
{
    auto encode = tensor_map_encoder();
    if (encode == nullptr) {
        *err = "CUDA: cuTensorMapEncodeTiled is not available";
        return false;
    }
    const cuuint64_t elem_bytes = fp64 ? 8 : 4;
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(g.nx), static_cast<cuuint64_t>(g.ny),
                                planes};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(g.pitch) * elem_bytes,
                                   static_cast<cuuint64_t>(g.plane) * elem_bytes};
    const cuuint32_t box[3] = {box_x, 1, box_planes};
    const cuuint32_t elem[3] = {1, 1, 1};
    const CUresult r = encode(map, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                        : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                              3, base, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        *err = "CUDA: cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")";
        return false;
    }
    return true;
}

} // namespace

bool encode_march_maps(const MixedState& in, const MixedState& out, const Geometry& g,
                       MarchTmaMaps* maps, std::string* err)
{
    return state_tensor_map(in.hi, false, 18, g, kTmaHaloW, 9, &maps->in_halo, err) &&
           state_tensor_map(in.hi, false, 18, g, kTmaOwnW, 18, &maps->in_own, err) &&
           state_tensor_map(out.hi, false, 18, g, kTmaOwnW, 18, &maps->out_own, err);
}

bool encode_march_maps_f64(const double* in, const double* out, const Geometry& g,
                           MarchTmaMaps* maps, std::string* err)
{
    void* i = const_cast<double*>(in);
    void* o = const_cast<double*>(out);
    return state_tensor_map(i, true, 9, g, kTmaHaloW, 9, &maps->in_halo, err) &&
           state_tensor_map(i, true, 9, g, kTmaOwnW, 9, &maps->in_own, err) &&
           state_tensor_map(o, true, 9, g, kTmaOwnW, 9, &maps->out_own, err);
}

bool encode_march_maps_delta(const MixedState& un, float* delta, const Geometry& g,
                             MarchTmaMaps* stage1, MarchTmaMaps* stage2, std::string* err,
                             unsigned halo_w, unsigned own_w)
{
    *stage1 = MarchTmaMaps{};
    *stage2 = MarchTmaMaps{};
    return state_tensor_map(un.hi, false, 18, g, halo_w, 9, &stage1->in_halo, err) &&
           state_tensor_map(un.hi, false, 18, g, halo_w, 9, &stage2->in_halo, err) &&
           state_tensor_map(delta, false, 9, g, halo_w, 9, &stage2->delta_halo, err) &&
           state_tensor_map(delta, false, 9, g, own_w, 9, &stage2->in_own, err) &&
           state_tensor_map(un.hi, false, 18, g, own_w, 18, &stage2->out_own, err);
}

} // namespace mhdb
