// Exact integer-slice split shared by the split-BF16 kernels: every operand
// row r gets a power of two s_r with max|x| / s_r in [64, 128) and three
// bf16 slices holding integers in [-128, 128],
//     x / s_r = c1 + c2 / 256 + c3 / 65536 + eps,   |eps| <= 2^-17,
// so tensor-core sums of slice products are exact integers in FP32 while
// they stay below 2^24.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace fc {

// Power-of-two scale with max / s in [64, 128).
__device__ __forceinline__ double pow2_scale(double mx) {
    if (!(mx > 0.0) || !(mx <= 1.0e300)) return 1.0;
    int k;
    frexp(mx, &k);           // mx = m 2^k, m in [0.5, 1)
    return ldexp(1.0, k - 7);
}

__device__ __forceinline__ void fx_slices(double x, double inv_s, __nv_bfloat16& c1, __nv_bfloat16& c2,
                                          __nv_bfloat16& c3) {
    const double y = x * inv_s;
    const double a = rint(y);
    const double y2 = (y - a) * 256.0;
    const double b = rint(y2);
    const double c = rint((y2 - b) * 256.0);
    c1 = __double2bfloat16(a);
    c2 = __double2bfloat16(b);
    c3 = __double2bfloat16(c);
}

// Row q of B_ov -> Bq[s][q][j*tpad + b] (row pitch K) at the row's scale qs[q].
__device__ __forceinline__ void split_fx_qrows_body(const double* __restrict__ B, int64_t nocc, int64_t nvir,
                                                    int64_t tpad, int64_t K, int64_t q_rows,
                                                    double* __restrict__ qs, __nv_bfloat16* __restrict__ Bq,
                                                    int64_t q) {
    __shared__ double red[32];
    const int64_t nov = nocc * nvir;
    const double* row = B + q * nov;
    double m = 0.0;
    for (int64_t k = threadIdx.x; k < nov; k += 256) m = fmax(m, fabs(row[k]));
    // block max (fixed order)
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double s = pow2_scale(red[0]);
    if (threadIdx.x == 0) qs[q] = s;
    const double inv = 1.0 / s;
    const int64_t ss = q_rows * K;
    __nv_bfloat16* o0 = Bq + q * K;
    for (int64_t k = threadIdx.x; k < nov; k += 256) {
        const int64_t j = k / nvir, b = k % nvir;
        __nv_bfloat16 c1, c2, c3;
        fx_slices(row[k], inv, c1, c2, c3);
        const int64_t d = j * tpad + b;
        o0[d] = c1;
        o0[ss + d] = c2;
        o0[2 * ss + d] = c3;
    }
}

// Per-row split of the FP32 amplitude chunk T[rows][pitch] (first Kv columns)
// -> Ts[s][rows][pitch], ts[row].  One CTA per row; the row is read twice
// (max, then slices).  Kv and pitch are multiples of 4.
__device__ __forceinline__ void split_fx_rows_f32_body(const float* __restrict__ T, int64_t Kv, int64_t K,
                                                       int64_t slice_rows, double* __restrict__ ts,
                                                       __nv_bfloat16* __restrict__ Ts, int64_t r) {
    __shared__ double red[32];
    const float4* row = reinterpret_cast<const float4*>(T + r * K);
    const int64_t K4 = Kv / 4;
    float m = 0.f;
    for (int64_t k = threadIdx.x; k < K4; k += 256) {
        const float4 v = row[k];
        m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double s = pow2_scale(red[0]);
    if (threadIdx.x == 0) ts[r] = s;
    const double inv = 1.0 / s;
    const int64_t ss = slice_rows * K;
    __nv_bfloat16* o0 = Ts + r * K;
    for (int64_t k = threadIdx.x; k < K4; k += 256) {
        const float4 v = row[k];
        __nv_bfloat16 a[4], b[4], c[4];
        fx_slices(v.x, inv, a[0], b[0], c[0]);
        fx_slices(v.y, inv, a[1], b[1], c[1]);
        fx_slices(v.z, inv, a[2], b[2], c[2]);
        fx_slices(v.w, inv, a[3], b[3], c[3]);
        uint2 pa, pb, pc;
        __nv_bfloat162 t0 = __halves2bfloat162(a[0], a[1]), t1 = __halves2bfloat162(a[2], a[3]);
        pa.x = *reinterpret_cast<uint32_t*>(&t0);
        pa.y = *reinterpret_cast<uint32_t*>(&t1);
        t0 = __halves2bfloat162(b[0], b[1]);
        t1 = __halves2bfloat162(b[2], b[3]);
        pb.x = *reinterpret_cast<uint32_t*>(&t0);
        pb.y = *reinterpret_cast<uint32_t*>(&t1);
        t0 = __halves2bfloat162(c[0], c[1]);
        t1 = __halves2bfloat162(c[2], c[3]);
        pc.x = *reinterpret_cast<uint32_t*>(&t0);
        pc.y = *reinterpret_cast<uint32_t*>(&t1);
        reinterpret_cast<uint2*>(o0)[k] = pa;
        reinterpret_cast<uint2*>(o0 + ss)[k] = pb;
        reinterpret_cast<uint2*>(o0 + 2 * ss)[k] = pc;
    }
}

}  // namespace fc
