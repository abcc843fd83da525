// Exact integer-slice splits.  Every operand row r gets a power of two s_r
// and three (or four) integer slices,
//     x / s_r = c1 + c2 / W + c3 / W^2 [+ c4 / W^3] + eps,
//     |eps| <= 1 / (2 W^2)  [1 / (2 W^3) with four slices],
// so tensor-core sums of slice products are exact integers.  Two formats:
//   SliceBf16  bf16 integers in [-128, 128], W = 256, max|x| / s in [64, 128);
//              FP32 accumulation, exact while sums stay below 2^24 (the
//              DF-K, dressing and Imat GEMMs, which drain to FP64 in panels);
//   SliceI8    int8 integers in [-127, 127], W = 254, max|x| / s in (63.5, 127];
//              int32 accumulation (tcgen05.mma kind::i8).  Three slices (the
//              adjoint contraction, up to three products per level): exact for
//              K <= (2^31 - 1) / (3 127^2) = 44381.  Four slices (the RI-MP2 pair
//              kernel, up to four products per level): K <= (2^31 - 1) / (4 127^2)
//              = 33286.
// Three slices carry about 23 significant bits of each element relative to
// its row maximum, four about 31.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace fc {

struct SliceBf16 {
    using T = __nv_bfloat16;
    static constexpr double W = 256.0;
    // power of two with max / s in [64, 128)
    __device__ static double scale(double mx) {
        if (!(mx > 0.0) || !(mx <= 1.0e300)) return 1.0;
        int k;
        frexp(mx, &k);  // mx = m 2^k, m in [0.5, 1)
        return ldexp(1.0, k - 7);
    }
    __device__ static T cast(double v) { return __double2bfloat16(v); }
};

struct SliceI8 {
    using T = int8_t;
    static constexpr double W = 254.0;
    // power of two with max / s in (63.5, 127]
    __device__ static double scale(double mx) {
        const double s = SliceBf16::scale(mx);
        return mx > 127.0 * s ? 2.0 * s : s;
    }
    __device__ static T cast(double v) { return (int8_t)(int)v; }
};

// Power-of-two scale of the BF16 format (DF-K, dressing, Imat).
__device__ __forceinline__ double pow2_scale(double mx) { return SliceBf16::scale(mx); }

template <class SL = SliceBf16>
__device__ __forceinline__ void fx_slices(double x, double inv_s, typename SL::T& c1, typename SL::T& c2,
                                          typename SL::T& c3) {
    const double y = x * inv_s;
    const double a = rint(y);
    const double y2 = (y - a) * SL::W;
    const double b = rint(y2);
    const double c = rint((y2 - b) * SL::W);
    c1 = SL::cast(a);
    c2 = SL::cast(b);
    c3 = SL::cast(c);
}

// Four slices (the pair operands of the RI-MP2 pair kernel).
template <class SL = SliceI8>
__device__ __forceinline__ void fx_slices4(double x, double inv_s, typename SL::T& c1, typename SL::T& c2,
                                           typename SL::T& c3, typename SL::T& c4) {
    const double y = x * inv_s;
    const double a = rint(y);
    const double y2 = (y - a) * SL::W;
    const double b = rint(y2);
    const double y3 = (y2 - b) * SL::W;
    const double c = rint(y3);
    const double d = rint((y3 - c) * SL::W);
    c1 = SL::cast(a);
    c2 = SL::cast(b);
    c3 = SL::cast(c);
    c4 = SL::cast(d);
}

// Row q of B_ov -> Bq[s][q][j*tpad + b] (row pitch K) at the row's scale qs[q],
// over the columns k = j*nvir + b in [k0, k1) (k1 < 0: all).
template <class SL = SliceBf16>
__device__ __forceinline__ void split_fx_qrows_body(const double* __restrict__ B, int64_t nocc, int64_t nvir,
                                                    int64_t tpad, int64_t K, int64_t q_rows,
                                                    double* __restrict__ qs, typename SL::T* __restrict__ Bq,
                                                    int64_t q, int64_t k0 = 0, int64_t k1 = -1) {
    __shared__ double red[32];
    const int64_t nov = nocc * nvir;
    const int64_t kend = k1 < 0 ? nov : k1;
    const double* row = B + q * nov;
    double m = 0.0;
    for (int64_t k = k0 + threadIdx.x; k < kend; k += 256) m = fmax(m, fabs(row[k]));
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
    const double s = SL::scale(red[0]);
    if (threadIdx.x == 0) qs[q] = s;
    const double inv = 1.0 / s;
    const int64_t ss = q_rows * K;
    typename SL::T* o0 = Bq + q * K;
    for (int64_t k = k0 + threadIdx.x; k < kend; k += 256) {
        const int64_t j = k / nvir, b = k % nvir;
        typename SL::T c1, c2, c3;
        fx_slices<SL>(row[k], inv, c1, c2, c3);
        const int64_t d = j * tpad + b;
        o0[d] = c1;
        o0[ss + d] = c2;
        o0[2 * ss + d] = c3;
    }
}

// Per-row split of the FP32 amplitude chunk T[rows][pitch] (first Kv columns)
// -> Ts[s][rows][pitch], ts[row].  One CTA per row; the row is read twice
// (max, then slices), or once when its max |T| is given (rmax: bits of the
// non-negative FP32 maximum per row).  Kv and pitch are multiples of 4.
template <class SL = SliceBf16>
__device__ __forceinline__ void split_fx_rows_f32_body(const float* __restrict__ T, int64_t Kv, int64_t K,
                                                       int64_t slice_rows, double* __restrict__ ts,
                                                       typename SL::T* __restrict__ Ts, int64_t r,
                                                       const unsigned* __restrict__ rmax = nullptr) {
    using E = typename SL::T;
    __shared__ double red[32];
    const float4* row = reinterpret_cast<const float4*>(T + r * K);
    const int64_t K4 = Kv / 4;
    if (rmax) {
        if (threadIdx.x == 0) red[0] = (double)__uint_as_float(rmax[r]);
    } else {
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
    }
    __syncthreads();
    const double s = SL::scale(red[0]);
    if (threadIdx.x == 0) ts[r] = s;
    const double inv = 1.0 / s;
    const int64_t ss = slice_rows * K;
    E* o0 = Ts + r * K;
    for (int64_t k = threadIdx.x; k < K4; k += 256) {
        const float4 v = row[k];
        E a[4], b[4], c[4];
        fx_slices<SL>(v.x, inv, a[0], b[0], c[0]);
        fx_slices<SL>(v.y, inv, a[1], b[1], c[1]);
        fx_slices<SL>(v.z, inv, a[2], b[2], c[2]);
        fx_slices<SL>(v.w, inv, a[3], b[3], c[3]);
        // four elements of each slice in one store (8 B for bf16, 4 B for int8)
        struct alignas(4 * sizeof(E)) Q4 { E e[4]; };
        Q4 pa, pb, pc;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            pa.e[u] = a[u];
            pb.e[u] = b[u];
            pc.e[u] = c[u];
        }
        reinterpret_cast<Q4*>(o0)[k] = pa;
        reinterpret_cast<Q4*>(o0 + ss)[k] = pb;
        reinterpret_cast<Q4*>(o0 + 2 * ss)[k] = pc;
    }
}

}  // namespace fc
