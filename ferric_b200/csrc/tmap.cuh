#pragma once
#include <cuda.h>

#include "fc_internal.cuh"

namespace fc {
// 2-D bf16 tensor map, 128-byte swizzle: `inner` contiguous elements per row,
// `outer` rows `row_bytes` apart, boxes of box_inner x box_outer.
fc_status make_tmap_bf16_2d(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                            uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer);
// The same for 8-bit elements (the int8 integer slices).
fc_status make_tmap_i8_2d(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint64_t row_bytes,
                          uint32_t box_inner, uint32_t box_outer);
// 8-bit elements in boxes of 64 B x box_outer rows with 64-byte swizzle (the
// RI-MP2 pair operands: four int8 slices per stage fit shared memory).
fc_status make_tmap_i8_2d_sw64(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                               uint64_t row_bytes, uint32_t box_outer);
}  // namespace fc
