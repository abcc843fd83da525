// TMA tensor-map encoding through the driver entry point (no link-time
// dependency on libcuda).
#include <cudaTypedefs.h>

#include "fc_internal.cuh"
#include "tmap.cuh"

namespace fc {

static fc_status make_tmap_2d(CUtensorMap* map, CUtensorMapDataType type, const void* base, uint64_t inner,
                              uint64_t outer, uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer,
                              CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B) {
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return fail(FC_ERR_DRIVER, "cuTensorMapEncodeTiled is not available from the driver");
        enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_bytes & 15))
        return fail(FC_ERR_LAYOUT, "TMA operand base/stride not 16-byte aligned");
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, type, 2, const_cast<void*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(FC_ERR_LAYOUT, "cuTensorMapEncodeTiled failed with CUresult " + std::to_string((int)r));
    return FC_OK;
}

fc_status make_tmap_bf16_2d(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                            uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer) {
    return make_tmap_2d(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, inner, outer, row_bytes, box_inner, box_outer);
}

fc_status make_tmap_i8_2d(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint64_t row_bytes,
                          uint32_t box_inner, uint32_t box_outer) {
    return make_tmap_2d(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, base, inner, outer, row_bytes, box_inner, box_outer);
}

fc_status make_tmap_i8_2d_sw64(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                               uint64_t row_bytes, uint32_t box_outer) {
    return make_tmap_2d(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, base, inner, outer, row_bytes, 64, box_outer,
                        CU_TENSOR_MAP_SWIZZLE_64B);
}

fc_status make_tmap_i8_3d(CUtensorMap* map, const void* base, uint64_t inner, uint64_t mid, uint64_t outer,
                          uint64_t row_bytes, uint64_t plane_bytes, uint32_t box_inner, uint32_t box_outer) {
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return fail(FC_ERR_DRIVER, "cuTensorMapEncodeTiled is not available from the driver");
        enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_bytes & 15) || (plane_bytes & 15))
        return fail(FC_ERR_LAYOUT, "TMA operand base/stride not 16-byte aligned");
    cuuint64_t dims[3] = {inner, mid, outer};
    cuuint64_t strides[2] = {row_bytes, plane_bytes};
    cuuint32_t box[3] = {box_inner, 1, box_outer};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(FC_ERR_LAYOUT, "cuTensorMapEncodeTiled (3-D) failed with CUresult " + std::to_string((int)r));
    return FC_OK;
}

}  // namespace fc
