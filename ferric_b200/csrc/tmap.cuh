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
// 3-D 8-bit map, 128-byte swizzle: `inner` contiguous elements, `mid` rows
// row_bytes apart, `outer` planes plane_bytes apart; boxes of box_inner x 1 x
// box_outer (one row of each of box_outer planes: rows strided by a plane).
fc_status make_tmap_i8_3d(CUtensorMap* map, const void* base, uint64_t inner, uint64_t mid, uint64_t outer,
                          uint64_t row_bytes, uint64_t plane_bytes, uint32_t box_inner, uint32_t box_outer);
}  // namespace fc
