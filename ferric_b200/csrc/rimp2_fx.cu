// Exact integer-slice RI-MP2 on the int8 tensor cores (FC_PREC_MIXED).
//
// Why: the tcgen05 FP32 accumulator does not round to nearest -- measured on
// B200, every accumulation step loses about 2^-24 of the running sum toward
// zero, so a floating hi/lo split accumulated over naux = 4800 is biased by
// ~1e-5 relative in E (the effect the reference measured for its f32 path,
// ferric-core/src/gpu/mixed.rs:18-21).  Here the operands are split into
// integer slices and multiplied on tcgen05.mma kind::i8 with int32
// accumulation, exact whatever the magnitudes.
//
// Split (SliceI8).  Each operand row r (an (i, a) column of B_ov over Q for
// the pair products, a Q row over (j, b) for the adjoint contraction) gets a
// power of two s_r with max|x| / s_r in (63.5, 127], and int8 slices holding
// integers in [-127, 127]:
//     x / s_r = c1 + c2 / 254 + c3 / 254^2 [+ c4 / 254^3] + eps.
// Pair kernel: four slices (|eps| <= 1/(2 254^3)) and the ten products of
// level k + m <= 3 in four TMEM accumulators, exact in int32 while
// 4 * 127^2 * naux < 2^31 (naux <= 33286):
//     L0 = c1 c1',  L1 = c1 c2' + c2 c1',  L2 = c1 c3' + c2 c2' + c3 c1',
//     L3 = c1 c4' + c2 c3' + c3 c2' + c4 c1',
//     g = s_r s_r' (((L0 254 + L1) 254 + L2) 254 + L3) / 254^3   (exact FP64 integer).
// The dropped level-4 products are 254^-4 of the row scales and of random
// sign, except where a row meets itself: (ia|ia) in the i == j blocks, whose
// c3 c3' term is one-signed; those values are taken exactly in FP64 from
// sum_Q B_Q,ia^2 (colsq_kernel).  Emulated at the config-3 shapes (naux 4800,
// nocc 120, nvir 1100, sampled pairs), E is within ~3e-8 Eh of FP64; three
// slices were 5e-5 Eh off.
// Adjoint contraction: three slices, six products in three accumulators
// (L0, L1, L2 above), exact while 3 * 127^2 * K < 2^31 (K segments of 32768).
//
// Pair kernel (this file): item = (pair, a-tile 128, b-tile 128); the X phase
// accumulates (ia|jb) into the four level accumulators (all 512 TMEM
// columns; the ten products go as six MMAs, four of them over two stacked B
// slices, or as ten narrower ones on a last virtual tile of <= 64 columns);
// the epilogue drains them into the CTA's column-major FP64 X tile in global
// scratch (L2-resident) and hands TMEM back; the Y phase accumulates
// (ib|ja) = G_ji[a, b] and is drained into the Y tile; the FP64 terms then
// run from the tiles in two halves, under the next item's two phases.  16
// epilogue warps, each thread one row and 32 columns of the tile.  Energy
// mode: unordered pairs,
// E_OS += (X^2 + Y^2)/D, E_SS += (X - Y)^2/D (i == j: X phase only, E_SS = 0),
// the reference pair loop of ferric-mp2/src/rimp2.rs:1399-1544 over both
// orderings.  Gradient mode: unordered pairs of an occupied chunk pair
// (I, J); the item writes Tt_ij = (2X - Y)/D (FP32) into the rows of i and
// (where the density terms need it, or I == J) Tt_ji = Tt_ij^T into the
// rows of j, and the dE/deps partials of both orderings; the adjoint
// contraction Gamma[:, I] += 4 Bq[:, J] Tt_IJ^T runs in gemm_fx_kernel, its
// J-side operand sliced from Tt_IJ by a tiled transpose when Tt_JI is not
// stored.  Diagonal tiles (ta == tb, i != j) run in one phase,
// Y = X^T read back transposed from the X tile (the exchange schedule).
#include <algorithm>
#include <cstdlib>

#include "batch.cuh"
#include "fc_internal.cuh"
#include "fx_split.cuh"
#include "rimp2.cuh"
#include "tc.cuh"
#include "tmap.cuh"
#include "xgemm.cuh"

namespace fc {

namespace fx {

constexpr int BM = 128, BN = 128;
constexpr int KT = 128;       // int8 elements (128 B) of K per pipeline stage (adjoint contraction)
constexpr int KT_BF16 = 64;   // bf16 elements per stage of the exact-slice xgemm (opposite-spin UMP2)
constexpr int64_t KMAX = 32768;  // K per int32 accumulation of the adjoint (3 * 127^2 * K < 2^31)
constexpr int A_BYTES = BM * KT;  // 16 KiB of int8
constexpr int B_BYTES = BN * KT;  // 16 KiB of int8
constexpr int NSL = 3;
// Pair kernel: four int8 slices per operand row, 64 B of K per stage (a
// 64-byte-swizzled box), three stages; four level accumulators fill TMEM.
constexpr int PKT = 64;
constexpr int PSL = 4;
constexpr int PA_BYTES = BM * PKT;                       // 8 KiB
constexpr int PB_BYTES = BN * PKT;                       // 8 KiB
constexpr int PSTAGE_BYTES = PSL * (PA_BYTES + PB_BYTES);  // 64 KiB
constexpr int PSTAGES = 3;
constexpr int COL_BYTES = 3 * BN * 8;             // a tile's virtual energies and column scales
// Pair-kernel epilogue: EPI_WARPS warps, EPI_WARPS / 4 per TMEM lane quadrant;
// each thread owns one row of the tile and HC of its columns.  The FP64
// epilogue is latency-bound (few independent FP64 instructions in flight per
// warp): 16 warps (4 per scheduler) at 32 columns each hide more of that
// latency than 8 at 64.
constexpr int EPI_WARPS = 16;
constexpr int NCG = EPI_WARPS / 4;                // column groups per row
constexpr int HC = BN / NCG;                      // columns per thread
constexpr int EPI_THREADS = 32 * EPI_WARPS;
constexpr int PAIR_THREADS = 64 + EPI_THREADS;    // + TMA producer warp + MMA warp
// epilogue scratch after the barriers ((2 PSTAGES + 4) x 8 B): per-warp partials
// [2][EPI_WARPS][3], row sums of column groups 1.. [NCG - 1][BM], column sums
// [4][NCG][HC] (doubles)
constexpr int SCR_BYTES = 8192;
static_assert((2 * PSTAGES + 4) * 8 + 8 * (2 * EPI_WARPS * 3 + (NCG - 1) * BM + 4 * NCG * HC) <= SCR_BYTES,
              "pair scratch");
static_assert(HC % 32 == 0 && 4 * NCG == EPI_WARPS, "pair epilogue layout");
constexpr int SMEM = PSTAGES * PSTAGE_BYTES + 1024 + SCR_BYTES + 2 * COL_BYTES;  // two column sets
constexpr uint32_t IDESC = tc::idesc_i8_s32(128, 128);
constexpr uint32_t IDESC2 = tc::idesc_i8_s32(128, 256);  // two stacked B slices
constexpr double LW = 254.0, LW2INV = 1.0 / (254.0 * 254.0), LW3INV = 1.0 / (254.0 * 254.0 * 254.0);

// s (L0 + L1 / 254 + L2 / 254^2) from the three int32 TMEM words of a level
// set: the integer combination (L0 254 + L1) 254 + L2 is exact in FP64.
__device__ __forceinline__ double level_value(float w0, float w1, float w2, double s) {
    const double v = (tc::i32_to_f64(w0) * LW + tc::i32_to_f64(w1)) * LW + tc::i32_to_f64(w2);
    return v * (s * LW2INV);
}

// 1 / d in FP64 by the Newton-Raphson iteration for the reciprocal, taken
// to third order from an FP32 seed: with rf = (1 / d)(1 + delta) and
// e = 1 - d rf = -delta (one FMA), rf (1 + e + e^2) = (1 / d)(1 - delta^3).
// |delta| <= 2^-23 (the FP32 roundings of d and of the seed), so the result
// is 1 / d to within the final FP64 rounding.  For normal FP32 magnitudes of
// d (the orbital-energy denominators are far inside them).
__device__ __forceinline__ double recip_nr(double d) {
    const double rf = (double)__frcp_rn(__double2float_rn(d));
    const double e = fma(-d, rf, 1.0);
    return fma(fma(e, e, e), rf, rf);
}

// s (L0 + L1 / 254 + L2 / 254^2 + L3 / 254^3) = s3 (((L0 254 + L1) 254 + L2)
// 254 + L3) for s3 = s / 254^3, from the four int32 TMEM words of the pair
// kernel's level set; the integer combination is below 2^53 while
// K <= 33286, so it is exact in FP64.
__device__ __forceinline__ double level_value4(float w0, float w1, float w2, float w3, double s3) {
    const double v =
        ((tc::i32_to_f64(w0) * LW + tc::i32_to_f64(w1)) * LW + tc::i32_to_f64(w2)) * LW + tc::i32_to_f64(w3);
    return v * s3;
}

}  // namespace fx

// ---------------------------------------------------------- split kernels --

// cmax[c] = max over rows of |B[r, c]| (as ordered uint64 bits of a double),
// for the columns c0 .. c0 + cols - 1 of rows of pitch ld (0: cols).
__device__ __forceinline__ void colmax_body(const double* __restrict__ B, int64_t rows, int64_t cols,
                                            int64_t rows_per_split, unsigned long long* cmax, int* bad, int64_t bx,
                                            int64_t by, int64_t ld = 0, int64_t c0 = 0) {
    const int64_t c = c0 + bx * 256 + threadIdx.x;
    if (c >= c0 + cols) return;
    const int64_t pitch = ld ? ld : cols;
    const int64_t r0 = by * rows_per_split;
    const int64_t r1 = r0 + rows_per_split < rows ? r0 + rows_per_split : rows;
    double m = 0.0;
    bool nf = false;
    for (int64_t r = r0; r < r1; ++r) {
        const double v = fabs(B[r * pitch + c]);
        nf |= !(v <= 1.0e300);
        m = v > m ? v : m;
    }
    if (nf) atomicOr(bad, 1);
    atomicMax(cmax + c, (unsigned long long)__double_as_longlong(m));
}

__global__ void __launch_bounds__(256) colmax_kernel(const double* __restrict__ B, int64_t rows, int64_t cols,
                                                     int64_t rows_per_split, unsigned long long* cmax, int* bad,
                                                     int64_t ld = 0, int64_t c0 = 0) {
    colmax_body(B, rows, cols, rows_per_split, cmax, bad, blockIdx.x, blockIdx.y, ld, c0);
}


// scl[i*a_pad + a] from the column maxima of B_ov (1 for padding rows), for
// the rows i*a_pad + a in [r0, r1) (r1 < 0: all).
template <class SL>
__global__ void row_scale_kernel(const unsigned long long* __restrict__ cmax, int64_t nocc, int64_t nvir,
                                 int64_t a_pad, double* __restrict__ scl, int64_t r0 = 0, int64_t r1 = -1) {
    const int64_t r = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= (r1 < 0 ? nocc * a_pad : r1)) return;
    const int64_t i = r / a_pad, a = r % a_pad;
    scl[r] = a < nvir ? SL::scale(__longlong_as_double((long long)cmax[i * nvir + a])) : 1.0;
}


// B[q, ia] -> Bt[s][i][a][q] (q < q_pad) integer slices at scale scl[i*a_pad+a],
// for the columns ia in [c0, c1) (c1 < 0: all).
template <class SL>
__device__ __forceinline__ void split_fx_transpose_body(const double* __restrict__ B, int64_t naux, int64_t nocc,
                                                        int64_t nvir, int64_t a_pad, int64_t q_pad,
                                                        const double* __restrict__ scl,
                                                        typename SL::T* __restrict__ Bt, int64_t bx, int64_t by,
                                                        int64_t c0 = 0, int64_t c1 = -1) {
    using E = typename SL::T;
    struct alignas(2 * sizeof(E)) P2 { E e[2]; };
    __shared__ double tile[64][65];
    const int64_t nov = nocc * nvir;
    const int64_t cend = c1 < 0 ? nov : c1;
    const int64_t q0 = by * 64, ia0 = c0 + bx * 64;
    const int tid = threadIdx.x;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const int idx = tid + 256 * e, r = idx >> 6, c = idx & 63;
        const int64_t q = q0 + r, ia = ia0 + c;
        tile[r][c] = (q < naux && ia < cend) ? B[q * nov + ia] : 0.0;
    }
    __syncthreads();
    const int64_t ss = nocc * a_pad * q_pad;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = tid + 256 * e, c = idx >> 5, qq = (idx & 31) * 2;
        const int64_t ia = ia0 + c;
        if (ia >= cend) continue;
        const int64_t i = ia / nvir, a = ia % nvir;
        const double inv = 1.0 / scl[i * a_pad + a];
        P2 pa, pb, pc;
        fx_slices<SL>(tile[qq][c], inv, pa.e[0], pb.e[0], pc.e[0]);
        fx_slices<SL>(tile[qq + 1][c], inv, pa.e[1], pb.e[1], pc.e[1]);
        const int64_t off = (i * a_pad + a) * q_pad + q0 + qq;
        *reinterpret_cast<P2*>(Bt + off) = pa;
        *reinterpret_cast<P2*>(Bt + ss + off) = pb;
        *reinterpret_cast<P2*>(Bt + 2 * ss + off) = pc;
    }
}

template <class SL>
__global__ void __launch_bounds__(256) split_fx_transpose_kernel(const double* __restrict__ B, int64_t naux,
                                                                 int64_t nocc, int64_t nvir, int64_t a_pad,
                                                                 int64_t q_pad, const double* __restrict__ scl,
                                                                 typename SL::T* __restrict__ Bt, int64_t c0 = 0,
                                                                 int64_t c1 = -1) {
    split_fx_transpose_body<SL>(B, naux, nocc, nvir, a_pad, q_pad, scl, Bt, blockIdx.x, blockIdx.y, c0, c1);
}

// The pair operands: B[q, ia] -> Bt[s][i][a][q] (q < q_pad), four int8 slices
// at scale scl[i*a_pad+a], for the columns ia in [c0, c1) (c1 < 0: all).
__device__ __forceinline__ void split_pair4_body(const double* __restrict__ B, int64_t naux, int64_t nocc,
                                                 int64_t nvir, int64_t a_pad, int64_t q_pad,
                                                 const double* __restrict__ scl, int8_t* __restrict__ Bt,
                                                 int64_t bx, int64_t by, int64_t c0 = 0, int64_t c1 = -1) {
    struct alignas(2) P2 { int8_t e[2]; };
    __shared__ double tile[64][65];
    const int64_t nov = nocc * nvir;
    const int64_t cend = c1 < 0 ? nov : c1;
    const int64_t q0 = by * 64, ia0 = c0 + bx * 64;
    const int tid = threadIdx.x;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const int idx = tid + 256 * e, r = idx >> 6, c = idx & 63;
        const int64_t q = q0 + r, ia = ia0 + c;
        tile[r][c] = (q < naux && ia < cend) ? B[q * nov + ia] : 0.0;
    }
    __syncthreads();
    const int64_t ss = nocc * a_pad * q_pad;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = tid + 256 * e, c = idx >> 5, qq = (idx & 31) * 2;
        const int64_t ia = ia0 + c;
        if (ia >= cend) continue;
        const int64_t i = ia / nvir, a = ia % nvir;
        const double inv = 1.0 / scl[i * a_pad + a];
        P2 p[4];
        fx_slices4<SliceI8>(tile[qq][c], inv, p[0].e[0], p[1].e[0], p[2].e[0], p[3].e[0]);
        fx_slices4<SliceI8>(tile[qq + 1][c], inv, p[0].e[1], p[1].e[1], p[2].e[1], p[3].e[1]);
        const int64_t off = (i * a_pad + a) * q_pad + q0 + qq;
#pragma unroll
        for (int s = 0; s < 4; ++s) *reinterpret_cast<P2*>(Bt + s * ss + off) = p[s];
    }
}

__global__ void __launch_bounds__(256) split_pair4_kernel(const double* __restrict__ B, int64_t naux, int64_t nocc,
                                                          int64_t nvir, int64_t a_pad, int64_t q_pad,
                                                          const double* __restrict__ scl, int8_t* __restrict__ Bt,
                                                          int64_t c0 = 0, int64_t c1 = -1) {
    split_pair4_body(B, naux, nocc, nvir, a_pad, q_pad, scl, Bt, blockIdx.x, blockIdx.y, c0, c1);
}

// gd[i*a_pad + a] = sum_q B[q, ia]^2 in FP64 (fixed order), the exact
// (ia|ia) of the pair kernel's i == j blocks, for the columns ia in [c0, c0+cols)
// of B (row pitch ld).  One thread per column; rows in one pass.
__device__ __forceinline__ void colsq_body(const double* __restrict__ B, int64_t rows, int64_t nvir, int64_t ld,
                                           int64_t a_pad, int64_t c, double* __restrict__ gd) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int64_t r = 0;
    for (; r + 4 <= rows; r += 4) {
        const double v0 = B[r * ld + c], v1 = B[(r + 1) * ld + c], v2 = B[(r + 2) * ld + c], v3 = B[(r + 3) * ld + c];
        s0 = fma(v0, v0, s0);
        s1 = fma(v1, v1, s1);
        s2 = fma(v2, v2, s2);
        s3 = fma(v3, v3, s3);
    }
    for (; r < rows; ++r) s0 = fma(B[r * ld + c], B[r * ld + c], s0);
    gd[(c / nvir) * a_pad + c % nvir] = (s0 + s1) + (s2 + s3);
}

__global__ void __launch_bounds__(256) colsq_kernel(const double* __restrict__ B, int64_t rows, int64_t nvir,
                                                    int64_t ld, int64_t a_pad, int64_t c0, int64_t c1,
                                                    double* __restrict__ gd) {
    const int64_t c = c0 + (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (c < c1) colsq_body(B, rows, nvir, ld, a_pad, c, gd);
}

__global__ void fill_kernel(double* __restrict__ x, int64_t n, double v) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) x[k] = v;
}

// Per-Q-row split of B_ov over (j, b) with b padded to a_pad:
// Bq[s][q][j*a_pad + b] (q < q_rows), scale qs[q].  One CTA per Q row.

__global__ void __launch_bounds__(256) split_fx_qrows_kernel(const double* __restrict__ B, int64_t nocc,
                                                             int64_t nvir, int64_t tpad, int64_t K,
                                                             int64_t q_rows, double* __restrict__ qs,
                                                             int8_t* __restrict__ Bq, int64_t k0 = 0,
                                                             int64_t k1 = -1) {
    split_fx_qrows_body<SliceI8>(B, nocc, nvir, tpad, K, q_rows, qs, Bq, blockIdx.x, k0, k1);
}


__global__ void __launch_bounds__(256) split_fx_rows_f32_kernel(const float* __restrict__ T, int64_t K,
                                                                int64_t slice_rows, double* __restrict__ ts,
                                                                int8_t* __restrict__ Ts) {
    split_fx_rows_f32_body<SliceI8>(T, K, K, slice_rows, ts, Ts, blockIdx.x);
}

// Column maxima of |T| over the rows [0, R) of the FP32 block T[R][ldt] for
// the columns [0, C) (C and ldt multiples of 4): cmax[c] takes the FP32 bits
// (ordered like the values for non-negative floats) by atomicMax and starts
// at 0.  A warp covers 128 columns (a float4 a lane); the eight warps and
// blockIdx.y split the rows.
__global__ void __launch_bounds__(256) colmax_f32_kernel(const float* __restrict__ T, int64_t R, int64_t C,
                                                         int64_t ldt, int64_t rows_per_split,
                                                         unsigned* __restrict__ cmax) {
    __shared__ float4 red[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t c = (int64_t)blockIdx.x * 128 + lane * 4;
    const int64_t r0 = (int64_t)blockIdx.y * rows_per_split;
    const int64_t r1 = r0 + rows_per_split < R ? r0 + rows_per_split : R;
    float4 m = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c < C) {
        for (int64_t r = r0 + w; r < r1; r += 8) {
            const float4 v = *reinterpret_cast<const float4*>(T + r * ldt + c);
            m.x = fmaxf(m.x, fabsf(v.x));
            m.y = fmaxf(m.y, fabsf(v.y));
            m.z = fmaxf(m.z, fabsf(v.z));
            m.w = fmaxf(m.w, fabsf(v.w));
        }
    }
    red[w][lane] = m;
    __syncthreads();
    if (w == 0 && c < C) {
#pragma unroll
        for (int k = 1; k < 8; ++k) {
            const float4 v = red[k][lane];
            m.x = fmaxf(m.x, v.x);
            m.y = fmaxf(m.y, v.y);
            m.z = fmaxf(m.z, v.z);
            m.w = fmaxf(m.w, v.w);
        }
        atomicMax(cmax + c, __float_as_uint(m.x));
        atomicMax(cmax + c + 1, __float_as_uint(m.y));
        atomicMax(cmax + c + 2, __float_as_uint(m.z));
        atomicMax(cmax + c + 3, __float_as_uint(m.w));
    }
}

// Three int8 slices of T^T: row c of the output is column c of T[R][ldt]
// (c < C) at the power-of-two scale of its maximum cmax[c]; Ts[s][c][r]
// (pitch R, slices slice_rows rows apart), ts[c] = the scale: the same
// values and scales as splitting the rows of a stored transpose.  64 x 64
// tiles of T pass through shared memory; R and C are multiples of 16.
__global__ void __launch_bounds__(256) split_cols_f32_kernel(const float* __restrict__ T, int64_t R, int64_t C,
                                                             int64_t ldt, const unsigned* __restrict__ cmax,
                                                             int64_t slice_rows, double* __restrict__ ts,
                                                             int8_t* __restrict__ Ts) {
    __shared__ float tile[64][65];
    const int t = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.y * 64, c0 = (int64_t)blockIdx.x * 64;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int rr = (t >> 4) + 16 * k, cc = (t & 15) * 4;
        const int64_t r = r0 + rr, c = c0 + cc;
        const float4 v = (r < R && c < C) ? *reinterpret_cast<const float4*>(T + r * ldt + c)
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
        tile[rr][cc] = v.x;
        tile[rr][cc + 1] = v.y;
        tile[rr][cc + 2] = v.z;
        tile[rr][cc + 3] = v.w;
    }
    __syncthreads();
    const int cc = t >> 2, rq = (t & 3) * 16;  // output row c0 + cc, its 16 columns from r0 + rq
    const int64_t c = c0 + cc, r = r0 + rq;
    if (c >= C || r >= R) return;
    const double s = SliceI8::scale((double)__uint_as_float(cmax[c]));
    if (blockIdx.y == 0 && rq == 0) ts[c] = s;
    const double inv = 1.0 / s;
    struct alignas(16) Q16 { int8_t e[16]; };
    Q16 p0, p1, p2;
#pragma unroll
    for (int k = 0; k < 16; ++k) fx_slices<SliceI8>(tile[rq + k][cc], inv, p0.e[k], p1.e[k], p2.e[k]);
    const int64_t ss = slice_rows * R;
    int8_t* o = Ts + c * R + r;
    *reinterpret_cast<Q16*>(o) = p0;
    *reinterpret_cast<Q16*>(o + ss) = p1;
    *reinterpret_cast<Q16*>(o + 2 * ss) = p2;
}

// The 6 products of one k-step (KT / 32 MMAs of K = 32 per product) from
// the stage whose A slice 0 has descriptor `da`; the three A slices are
// A_BYTES apart and the B slices start BOFS bytes after A slice 0 (adjacent,
// B_BYTES = 128 rows apart), and the level accumulators are adjacent in TMEM
// (BN columns apart).  Offsets are compile-time: the descriptor start-address
// field is linear in the address.  PART 1 issues the four products of slices
// 0 and 1 as two N = 256 MMAs of an A slice with the stacked rows [B0; B1]
// (A0 -> levels 0, 1; A1 -> levels 1, 2), except on the first K step of a
// segment, where level 2 starts (A1 B1 is its first product) while level 1
// accumulates, so A1 B0 and A1 B1 go as two N = 128 MMAs; PART 2 issues the
// two with a slice 2 (their operands may arrive later); PART 0 both.  The
// int32 sums are exact, so the order of the products does not change the
// result.
template <int BOFS, int PART = 0>
__device__ __forceinline__ void issue_products(uint64_t da, uint32_t tmem_base, int kt) {
    using namespace fx;
    auto a_of = [&](int sl, int kk) { return da + (uint64_t)((sl * A_BYTES + kk * 32) >> 4); };
    auto b_of = [&](int sl, int kk) { return da + (uint64_t)((BOFS + sl * B_BYTES + kk * 32) >> 4); };
    if (PART != 2) {
#pragma unroll
        for (int kk = 0; kk < KT / 32; ++kk) {
            const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
            tc::umma_i8(tmem_base, a_of(0, kk), b_of(0, kk), IDESC2, acc);
            if (acc) {
                tc::umma_i8(tmem_base + BN, a_of(1, kk), b_of(0, kk), IDESC2, 1u);
            } else {
                tc::umma_i8(tmem_base + BN, a_of(1, kk), b_of(0, kk), IDESC, 1u);
                tc::umma_i8(tmem_base + 2 * BN, a_of(1, kk), b_of(1, kk), IDESC, 0u);
            }
        }
    }
    if (PART != 1) {
#pragma unroll
        for (int kk = 0; kk < KT / 32; ++kk) {
            tc::umma_i8(tmem_base + 2 * BN, a_of(0, kk), b_of(2, kk), IDESC, 1u);
            tc::umma_i8(tmem_base + 2 * BN, a_of(2, kk), b_of(0, kk), IDESC, 1u);
        }
    }
}

// ------------------------------------------------------------ pair kernel --

// The 10 products of one k-step of the pair kernel (K = 32 per MMA, PKT / 32
// MMAs per product) from the stage whose A slice 0 has descriptor `da`; the
// four A slices are PA_BYTES apart and the B slices start BOFS bytes after A
// slice 0.  Level l = k + m collects the products c_k c'_m of slices k and m,
// l <= 3.  The B slices are adjacent in shared memory (PB_BYTES = 128 rows
// apart) and the level accumulators adjacent in TMEM (BN columns apart), so
// one N = 256 MMA of A slice k with the stacked rows [B_m; B_m+1] adds
// c_k c'_m to level k + m and c_k c'_m+1 to level k + m + 1: six MMAs (four
// of N = 256, two of N = 128) issue the ten products, and each A slice is
// read from shared memory once per 256 columns.  The ten 128 x 128 MMAs they
// replace were bound by shared-memory reads (8 KiB per 64-cycle MMA, with
// the TMA writes beside them).
template <int BOFS>
__device__ __forceinline__ void issue_products4(uint64_t da, uint32_t tmem_base, int kt) {
    using namespace fx;
    constexpr int PA[6] = {0, 0, 1, 1, 2, 3};  // A slice
    constexpr int PB[6] = {0, 2, 0, 2, 0, 0};  // first B slice; the MMA writes levels PA + PB (+ 1)
    constexpr int PW[6] = {1, 1, 0, 0, 0, 0};  // first write of its levels
    constexpr bool P2[6] = {true, true, true, false, true, false};  // two B slices (N = 256)
#pragma unroll
    for (int pr = 0; pr < 6; ++pr) {
#pragma unroll
        for (int kk = 0; kk < PKT / 32; ++kk)
            tc::umma_i8(tmem_base + (PA[pr] + PB[pr]) * BN, da + (uint64_t)((PA[pr] * PA_BYTES + kk * 32) >> 4),
                        da + (uint64_t)((BOFS + PB[pr] * PB_BYTES + kk * 32) >> 4), P2[pr] ? IDESC2 : IDESC,
                        (kt > 0 || kk > 0 || !PW[pr]) ? 1u : 0u);
    }
}

// The ten products one by one, N = n (a multiple of 16, idesc encodes it):
// the last virtual tile of a pair operand, whose columns past n are
// padding.  Ten MMAs of N = n issue n / 128 of the stacked form's work when
// n <= 64; the accumulator columns from n on keep stale integers, which the
// epilogue never reads as amplitudes (they are columns b >= nvir).
template <int BOFS>
__device__ __forceinline__ void issue_products4_n(uint64_t da, uint32_t tmem_base, int kt, uint32_t idesc) {
    using namespace fx;
    constexpr int PA[10] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};
    constexpr int PB[10] = {0, 1, 0, 2, 1, 0, 3, 2, 1, 0};
    constexpr int PL[10] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3};
    constexpr int PF[10] = {1, 1, 0, 1, 0, 0, 1, 0, 0, 0};  // first product of its level
#pragma unroll
    for (int pr = 0; pr < 10; ++pr) {
#pragma unroll
        for (int kk = 0; kk < PKT / 32; ++kk)
            tc::umma_i8(tmem_base + PL[pr] * BN, da + (uint64_t)((PA[pr] * PA_BYTES + kk * 32) >> 4),
                        da + (uint64_t)((BOFS + PB[pr] * PB_BYTES + kk * 32) >> 4), idesc,
                        (kt > 0 || kk > 0 || !PF[pr]) ? 1u : 0u);
    }
}

// One molecule of a batch (operand rows row0 .. row0 + 4*nocc*a_pad of the
// concatenated slice buffer, slice-major).
struct BatchMol {
    const double* eo;
    const double* ev;
    const double* scl;
    const double* gd;  // [nocc * a_pad] exact (ia|ia)
    int nocc, nvir, a_pad, nk;
    int row0, tpad;  // tpad: virtual pitch of the amplitude rows/columns (gradient)
    int xt, pad2_;   // exchange (one phase) on diagonal tiles
    float* T;        // amplitudes [nocc*tpad][ldt] (gradient)
    int64_t ldt;
};

struct PairFxArgs {
    // batch mode: item k is bitems[k] = (molecule, i, j, ta | tb << 16)
    const int4* bitems;
    const BatchMol* bmols;
    const double* eo;
    const double* ev;
    const double* scl;  // [nocc * a_pad] operand-row scales
    const double* gd;   // [nocc * a_pad] exact (ia|ia) = sum_Q B_Q,ia^2
    const int2* pairs;  // pairs of the launch
    const int2* tiles;  // (a-tile, b-tile) of each item of a pair
    int ntiles;         // tiles per pair
    int npairs;
    int nocc, nvir, a_pad, nTa, nTb, nk;
    int tpad;      // pitch of the amplitude rows and columns (>= nvir, multiple of 8)
    int xt;        // exchange (one phase) on diagonal tiles
    int64_t items;
    double* part;  // [item][2]
    double* scr;   // [grid][3][BM][BN] FP64 tiles of each CTA: X of two items, Y
    int* err;
    // failure-path test hook: the MMA warp's waits for operand stages give up
    // after wait_ns; with drop_load, CTA 0's producer issues no load for its
    // first stage, so that wait runs out with nothing in flight
    uint64_t wait_ns;
    int drop_load;
    // gradient mode: pairs (i, j), i in chunk I (from i0), j in chunk J (from j0)
    float* T;        // amplitude rows of I: [|I| a_pad][ldt = |J| a_pad]
    float* T2;       // amplitude rows of J: [|J| a_pad][ldt2 = |I| a_pad] (T when I == J; not
                     // written with no_t2)
    int64_t ldt, ldt2;
    int i0, j0;
    int no_t2;         // T2 (a buffer of its own) is not written: its slices come from T transposed
    double* occ_part;  // [item]
    double* vir_part;  // [item][2][128]: row-virtual and column-virtual sums
};

// Everything the roles need about item k.
struct ItemView {
    int i, j, ta, tb, nk, a_pad, nvir, row0, slice_rows, tpad, i0, j0;
    int xt;  // diagonal tile, i != j: Y = X^T read back transposed, no Y phase
    const double* eo;
    const double* ev;
    const double* scl;
    const double* gd;
    float* T;
    float* T2;
    int64_t ldt, ldt2;
};

template <int BATCH>
__device__ __forceinline__ ItemView item_view(const PairFxArgs& p, int64_t k) {
    ItemView v;
    if (BATCH) {
        const int4 it = p.bitems[k];
        const BatchMol& m = p.bmols[it.x];
        v.i = it.y;
        v.j = it.z;
        v.ta = it.w & 0xFFFF;
        v.tb = it.w >> 16;
        v.nk = m.nk;
        v.a_pad = m.a_pad;
        v.nvir = m.nvir;
        v.row0 = m.row0;
        v.slice_rows = m.nocc * m.a_pad;
        v.eo = m.eo;
        v.ev = m.ev;
        v.scl = m.scl;
        v.gd = m.gd;
        v.tpad = m.tpad;
        v.xt = m.xt && v.ta == v.tb && v.i != v.j;
        v.i0 = 0;
        v.j0 = 0;
        v.T = m.T;
        v.T2 = m.T;
        v.ldt = m.ldt;
        v.ldt2 = m.ldt;
    } else {
        const int2 ij = p.pairs[k / p.ntiles];
        const int2 tt = p.tiles[k % p.ntiles];
        v.i = ij.x;
        v.j = ij.y;
        v.ta = tt.x;
        v.tb = tt.y;
        v.nk = p.nk;
        v.a_pad = p.a_pad;
        v.nvir = p.nvir;
        v.row0 = 0;
        v.slice_rows = p.nocc * p.a_pad;
        v.eo = p.eo;
        v.ev = p.ev;
        v.scl = p.scl;
        v.gd = p.gd;
        v.tpad = p.tpad;
        v.xt = p.xt && v.ta == v.tb && v.i != v.j;
        v.i0 = p.i0;
        v.j0 = p.j0;
        v.T = p.T;
        v.T2 = p.T2;
        v.ldt = p.ldt;
        v.ldt2 = p.ldt2;
    }
    return v;
}

// This thread's HC columns of a phase's four level accumulators -> FP64
// values s_r s_c (L0 + L1/254 + L2/254^2 + L3/254^3), stored at dst + c BM
// for its column c (the CTA's column-major tile in global scratch, L2 only;
// dst is its row of the first of its columns).  gdv >= 0 is the column (of
// these HC) on the tile diagonal a == b of an i == j block: it takes the
// exact (ia|ia) instead, whose dropped level-4 products (the slice c3 c3' of
// a row with itself) are one-signed.
__device__ __forceinline__ void drain_levels(uint32_t tl, double sr, const double* __restrict__ sc, double* dst,
                                             int gdv, double gval) {
    using namespace fx;
    const double sr3 = sr * LW3INV;
#pragma unroll
    for (int c0 = 0; c0 < HC; c0 += 8) {
        float l0[8], l1[8], l2[8], l3[8];
        tc::tmem_ld8(tl + c0, l0);
        tc::tmem_ld8(tl + BN + c0, l1);
        tc::tmem_ld8(tl + 2 * BN + c0, l2);
        tc::tmem_ld8(tl + 3 * BN + c0, l3);
        tc::tmem_wait_ld();
        double x[8];
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
            x[cc] = level_value4(l0[cc], l1[cc], l2[cc], l3[cc], sr3 * sc[c0 + cc]);
            if (c0 + cc == gdv) x[cc] = gval;
        }
        // column-major tile: the warp's 32 rows of a column are one 256-byte run
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) __stcg(dst + (c0 + cc) * BM, x[cc]);
    }
}

template <int GRAD, int BATCH = 0>
__global__ void __launch_bounds__(fx::PAIR_THREADS, 1)
    pair_fx_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const PairFxArgs p) {
    using namespace fx;
    constexpr int S = PSTAGES;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_u32 = smem_u32(smem_raw);
    const uint32_t base_u32 = (raw_u32 + 1023u) & ~1023u;
    uint8_t* base = smem_raw + (base_u32 - raw_u32);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * PSTAGE_BYTES);
    uint64_t* full = bars;                // [S]
    uint64_t* empty = bars + S;           // [S]
    uint64_t* tfull = bars + 2 * S;       // [1] a phase's levels are complete in TMEM
    uint64_t* tempty = bars + 2 * S + 1;  // [1] the epilogue has read them out
    uint64_t* drain = bars + 2 * S + 2;   // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 3);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(bars + 2 * S + 4);  // [2][EPI_WARPS][3]
    double* rowsh = red + 2 * EPI_WARPS * 3;                     // [NCG - 1][BM] row sums of column groups 1..
    double* colsh = rowsh + (NCG - 1) * BM;                      // [4 quadrants][NCG][HC] column sums
    double* colb = reinterpret_cast<double*>(base + S * PSTAGE_BYTES + SCR_BYTES);  // [2 items][3][BN]

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(tfull, 1);
        tc::mbar_init(tempty, EPI_THREADS);
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) {
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 512);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    auto sa = [&](int s, int sl) { return base_u32 + s * PSTAGE_BYTES + sl * PA_BYTES; };
    auto sb = [&](int s, int sl) { return base_u32 + s * PSTAGE_BYTES + PSL * PA_BYTES + sl * PB_BYTES; };
    auto row_of = [&](const ItemView& v, int sl, int i, int r0) {
        return v.row0 + sl * v.slice_rows + i * v.a_pad + r0;
    };

    if (warp == 0) {
        // ------------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t g = 0;
            const bool drop = p.drop_load && blockIdx.x == 0;  // stage g == 0 gets no load
            for (int64_t k = blockIdx.x; k < p.items && !*abort_flag; k += gridDim.x) {
                const ItemView v = item_view<BATCH>(p, k);
                const int nph = (v.i == v.j || v.xt) ? 1 : 2;
                for (int ph = 0; ph < nph; ++ph) {
                    const int ia = ph == 0 ? v.i : v.j, ib = ph == 0 ? v.j : v.i;
                    for (int kt = 0; kt < v.nk; ++kt, ++g) {
                        const int s = g % S;
                        const uint32_t u = g / S;
                        if (!tc::mbar_wait(&empty[s], (u & 1) ^ 1, abort_flag, p.err)) goto prod_done;
                        if (drop && g == 0) continue;
                        tc::mbar_arrive_expect_tx(&full[s], PSTAGE_BYTES);
#pragma unroll
                        for (int sl = 0; sl < PSL; ++sl) {
                            tc::tma_load_2d(base + (sa(s, sl) - base_u32), &tmA, &full[s], kt * PKT,
                                            row_of(v, sl, ia, v.ta * BM));
                            tc::tma_load_2d(base + (sb(s, sl) - base_u32), &tmB, &full[s], kt * PKT,
                                            row_of(v, sl, ib, v.tb * BN));
                        }
                    }
                }
            }
        prod_done:
            // every load issued lands before the CTA leaves (a dropped stage has none)
            for (uint32_t q = 0; q < (uint32_t)S && q < g; ++q) {
                const uint32_t gg = g - 1 - q;
                if (drop && gg == 0) continue;
                int no_abort = 0;
                tc::mbar_wait(&full[gg % S], (gg / S) & 1, &no_abort, p.err);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------ UMMA issuer
        if (lane == 0) {
            // the operand descriptors of the stages, computed once: rebuilding
            // them every k-step delayed the MMA issue by ~9% (measured)
            uint64_t da[S];
#pragma unroll
            for (int s = 0; s < S; ++s) da[s] = tc::sdesc_k64(sa(s, 0));
            uint32_t g = 0, pc = 0;  // pc: phases issued (TMEM hand-overs)
            for (int64_t k = blockIdx.x; k < p.items && !*abort_flag; k += gridDim.x) {
                const ItemView v = item_view<BATCH>(p, k);
                const int nph = (v.i == v.j || v.xt) ? 1 : 2;
                // the last virtual tile of B: its first nt columns (rounded to 16) hold virtuals
                const int rem = v.nvir - v.tb * BN;
                const int nt = rem >= BN ? BN : (rem + 15) / 16 * 16;
                const bool trim = nt <= 64;
                const uint32_t idt = tc::idesc_i8_s32(128, nt);
                for (int ph = 0; ph < nph; ++ph, ++pc) {
                    if (!tc::mbar_wait(tempty, (pc & 1) ^ 1, abort_flag, p.err)) goto mma_done;
                    tc::fence_after_sync();
                    for (int kt = 0; kt < v.nk; ++kt, ++g) {
                        const int s = g % S;
                        const uint32_t u = g / S;
                        if (!tc::mbar_wait(&full[s], u & 1, abort_flag, p.err,
                                           p.wait_ns ? p.wait_ns : tc::WAIT_LIMIT_NS))
                            goto mma_done;
                        tc::fence_after_sync();
                        uint64_t d = da[0];
#pragma unroll
                        for (int t = 1; t < S; ++t)
                            if (s == t) d = da[t];
                        if (trim)
                            issue_products4_n<PSL * PA_BYTES>(d, tmem_base, kt, idt);
                        else
                            issue_products4<PSL * PA_BYTES>(d, tmem_base, kt);
                        tc::umma_commit(&empty[s]);
                    }
                    tc::umma_commit(tfull);
                }
            }
        mma_done:
            tc::umma_commit(drain);
            int no_abort = 0;
            tc::mbar_wait(drain, 0, &no_abort, p.err);
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- epilogue
        // EPI_WARPS warps: lane quadrant q = warp % 4 (TMEM lanes 32q..32q+31),
        // column group h = (warp - 2) / 4; each thread owns row `row`, columns
        // [HC h, HC h + HC).  A phase's four level accumulators fill TMEM, so
        // each phase is drained at once into the CTA's FP64 tiles in global
        // scratch (X, then Y), which hands TMEM back to the MMA warp.  The FP64
        // terms of an item run in two halves of its columns, software-pipelined
        // against the next item's phases:
        //     drain X_k | terms(k-1, 2nd half), finish(k-1) | drain Y_k | terms(k, 1st half)
        // so the first half runs under X_{k+1}'s MMAs and the second under
        // Y_{k+1}'s (the FP64 terms of a whole item outlast one MMA phase).  X
        // tiles alternate by item (X_k is drained while X_{k-1} is still read);
        // Y_k is drained after the last read of Y_{k-1}.
        const int q = warp & 3;
        const int h = (warp - 2) >> 2;
        const int row = q * 32 + lane;  // a within the tile
        const int et = tid - 64;        // 0 .. EPI_THREADS - 1
        const uint32_t tl = tmem_base + ((uint32_t)(q * 32) << 16) + h * HC;
        // X tiles [2][col][row], Y tile [col][row]: column-major, so a warp's
        // stores and loads of one column cover its 32 consecutive rows
        double* const scr0 = p.scr + (int64_t)blockIdx.x * (3 * BM * BN);
        double* const syt = scr0 + 2 * BM * BN;
        double* const ycol = syt + h * HC * BM + row;  // this thread's first column, its row
        constexpr int HH = HC / 2;  // columns per half
        // carried from an item's first half of terms to its second
        double os = 0.0, ss = 0.0, oc = 0.0, rowc = 0.0;

        // FP64 terms of columns [c_lo, c_lo + HH) of this thread's HC, item k
        // (li parity lk): energy sums, derivative sums, amplitude stores, and the
        // column terms of the mirrored tile reduced over the warp's 32 rows into
        // colsh[q][h][c_lo ..].
        auto terms = [&](int64_t k, uint32_t lk, int c_lo) {
            const ItemView v = item_view<BATCH>(p, k);
            const int i = v.i, j = v.j;
            const bool diag = i == j;
            const int ta = v.ta, tb = v.tb;
            const bool mir = GRAD && ta < tb;
            const bool both = GRAD && !diag;
            const int a = ta * BM + row;
            const bool va = a < v.nvir;
            const double dA = v.eo[i] + v.eo[j] - (va ? v.ev[a] : 0.0);
            const int b0 = tb * BN + h * HC;  // first column of this thread
            const double* evb = colb + (lk & 1) * 3 * BN + h * HC;
            const int bmax = v.nvir - b0;  // columns c < bmax are real virtuals
            const bool xt = v.xt;
            const bool two = !diag && !xt;
            double* const sxt = scr0 + (lk & 1) * BM * BN;
            const double* const xcol = sxt + h * HC * BM + row;
            constexpr int CW = 4;  // columns per step of the FP64 terms
            float ck[HH];          // column terms of this half's columns (gradient)
#pragma unroll
            for (int cs = 0; cs < HH; cs += CW) {
                const int c0 = c_lo + cs;
                double xv[CW] = {}, yv[CW] = {};
                // rows and columns past the last virtual read nothing (those tile
                // entries may not have been drained; their amplitudes are zeros)
                if (va && c0 < bmax) {
#pragma unroll
                    for (int cc = 0; cc < CW; ++cc) xv[cc] = __ldcg(xcol + (c0 + cc) * BM);
                    if (two) {
#pragma unroll
                        for (int cc = 0; cc < CW; ++cc) yv[cc] = __ldcg(ycol + (c0 + cc) * BM);
                    } else if (xt) {
                        // Y[a, b] = X[b, a]: column a of X, this thread's columns b as rows
                        const double2* x2 = reinterpret_cast<const double2*>(sxt + row * BM + h * HC + c0);
#pragma unroll
                        for (int u = 0; u < CW / 2; ++u) {
                            const double2 t = __ldcg(x2 + u);
                            yv[2 * u] = t.x;
                            yv[2 * u + 1] = t.y;
                        }
                    } else {
#pragma unroll
                        for (int cc = 0; cc < CW; ++cc) yv[cc] = xv[cc];  // i == j: Y = X
                    }
                }
                float tt8[CW], mv8[CW];
#pragma unroll
                for (int cc = 0; cc < CW; ++cc) {
                    const double x = xv[cc];
                    const double y = yv[cc];
                    float tval = 0.f, mval = 0.f, colv = 0.f;
                    if (va && c0 + cc < bmax) {
                        const double r = recip_nr(dA - evb[c0 + cc]);
                        const double xr = x * r;
                        const double yr = diag ? xr : y * r;
                        if (diag) {
                            os = fma(x, xr, os);
                        } else {
                            os = fma(y, yr, fma(x, xr, os));
                            ss = fma(x - y, xr - yr, ss);
                        }
                        if (GRAD) {
                            // t Tt summed over a pair's elements is the pair's share of
                            // dE/deps_occ; by virtual index, of dE/deps_vir.  Pair (i, j)
                            // puts its element (a, b) on the row virtual a, pair (j, i)
                            // on b (its row index); the mirrored tile the other way round.
                            // On an exchanged diagonal tile the thread of row a also
                            // holds (b, a)'s term and puts it on a directly.
                            const double tt = fma(2.0, xr, -yr);  // Tt_ij[a, b]
                            const double cd = xr * tt;            // t Tt at (a, b)
                            tval = (float)tt;
                            if (mir || xt) {
                                const double tm = fma(2.0, yr, -xr);  // Tt_ij[b, a]
                                const double cm = yr * tm;            // t Tt at (b, a)
                                const double cs = cd + cm;
                                if (mir) {
                                    mval = (float)tm;
                                    oc += cs;
                                } else {
                                    oc += cd;
                                }
                                rowc += (both || xt) ? cs : cd;
                                if (!xt) colv = (float)(both ? cs : cm);
                            } else {
                                oc += cd;
                                rowc += cd;
                                colv = both ? (float)cd : 0.f;
                            }
                        }
                    }
                    tt8[cc] = tval;
                    mv8[cc] = mval;
                    ck[cs + cc] = colv;
                }
                if (GRAD && a < v.tpad) {
                    // amplitude rows (i, a) and columns (j, b) at pitch tpad (>= nvir);
                    // elements with a or b >= tpad belong to no amplitude.  Rows of
                    // i go to T (columns of j from j0), rows of j to T2 (columns of i
                    // from i0); with one chunk for both, T2 is T.
                    const int bw = v.tpad - (b0 + c0);  // columns of this group inside the pitch
                    float* trow = v.T + ((int64_t)(i - v.i0) * v.tpad) * v.ldt + (int64_t)(j - v.j0) * v.tpad;
                    float* d = trow + (int64_t)a * v.ldt + b0 + c0;
                    if (bw >= CW) {
                        float4* dst = reinterpret_cast<float4*>(d);
#pragma unroll
                        for (int u = 0; u < CW / 4; ++u)
                            dst[u] = make_float4(tt8[4 * u], tt8[4 * u + 1], tt8[4 * u + 2], tt8[4 * u + 3]);
                    } else {
#pragma unroll
                        for (int cc = 0; cc < CW; ++cc)
                            if (cc < bw) d[cc] = tt8[cc];
                    }
                    if (mir) {
#pragma unroll
                        for (int cc = 0; cc < CW; ++cc)  // lanes hold consecutive a: coalesced
                            if (cc < bw) trow[(int64_t)(b0 + c0 + cc) * v.ldt + a] = mv8[cc];
                    }
                    if (both && (BATCH || !p.no_t2)) {
                        float* t2 = v.T2 + ((int64_t)(j - v.j0) * v.tpad) * v.ldt2 + (int64_t)(i - v.i0) * v.tpad;
#pragma unroll
                        for (int cc = 0; cc < CW; ++cc)  // Tt_ji[b, a] = Tt_ij[a, b]
                            if (cc < bw) t2[(int64_t)(b0 + c0 + cc) * v.ldt2 + a] = tt8[cc];
                        if (mir) {                      // Tt_ji[a, b] = Tt_ij[b, a]
                            float* d2 = t2 + (int64_t)a * v.ldt2 + b0 + c0;
                            if (bw >= CW) {
                                float4* dst = reinterpret_cast<float4*>(d2);
#pragma unroll
                                for (int u = 0; u < CW / 4; ++u)
                                    dst[u] = make_float4(mv8[4 * u], mv8[4 * u + 1], mv8[4 * u + 2], mv8[4 * u + 3]);
                            } else {
#pragma unroll
                                for (int cc = 0; cc < CW; ++cc)
                                    if (cc < bw) d2[cc] = mv8[cc];
                            }
                        }
                    }
                }
            }
            if ((mir || both) && !xt) {
                // column sums of the mirrored terms over this warp's 32 rows: a
                // reduce-scatter butterfly over offsets 16 .. 2 leaves column
                // lane / 2 of the half in ck[0] (lanes 2m and 2m + 1 hold the two
                // halves of the rows' sum), then lane pairs add
#pragma unroll
                for (int half = HH / 2, off = 16; off > 1; half >>= 1, off >>= 1) {
                    const bool up = (lane & off) != 0;
#pragma unroll
                    for (int c = 0; c < half; ++c) {
                        const float send = up ? ck[c] : ck[c + half];
                        const float recv = __shfl_xor_sync(0xffffffffu, send, off);
                        ck[c] = (up ? ck[c + half] : ck[c]) + recv;
                    }
                }
                const float tot = ck[0] + __shfl_xor_sync(0xffffffffu, ck[0], 1);
                if ((lane & 1) == 0) colsh[(q * NCG + h) * HC + c_lo + (lane >> 1)] = (double)tot;
            }
        };

        // the item's sums: partials of E_OS / E_SS / dE/deps (fixed order)
        auto finish = [&](int64_t k, uint32_t lk) {
            const ItemView v = item_view<BATCH>(p, k);
            const bool diag = v.i == v.j;
            const bool mir = GRAD && v.ta < v.tb;
            const bool both = GRAD && !diag;
            const bool xt = v.xt;
            const double wt = v.ta < v.tb ? 2.0 : 1.0;
            const double vo = warp_sum(os), vs = warp_sum(ss);
            const double vc = GRAD ? warp_sum(oc) : 0.0;
            double* rb = red + (lk & 1) * (EPI_WARPS * 3);
            if (lane == 0) {
                rb[(warp - 2) * 3 + 0] = vo;
                rb[(warp - 2) * 3 + 1] = vs;
                rb[(warp - 2) * 3 + 2] = vc;
            }
            if (GRAD && h > 0) rowsh[(h - 1) * BM + row] = rowc;
            asm volatile("bar.sync 1, %0;" ::"n"(EPI_THREADS) : "memory");
            if (GRAD && h == 0) {
                double rs = rowc;
#pragma unroll
                for (int hh = 1; hh < NCG; ++hh) rs += rowsh[(hh - 1) * BM + row];
                p.vir_part[k * 2 * BM + row] = rs;
            }
            if ((mir || both) && et < BM) {  // an exchanged tile put its column terms on the rows
                const int hh = et / HC, c = et % HC;
                double cs = 0.0;
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) cs += colsh[(qq * NCG + hh) * HC + c];
                p.vir_part[k * 2 * BM + BM + et] = xt ? 0.0 : cs;
            }
            if (et == 0) {
                KSum so, sn, sc;
#pragma unroll
                for (int w = 0; w < EPI_WARPS; ++w) {
                    so.add(rb[w * 3]);
                    sn.add(rb[w * 3 + 1]);
                    sc.add(rb[w * 3 + 2]);
                }
                p.part[2 * k] = wt * so.value();
                p.part[2 * k + 1] = wt * sn.value();
                if (GRAD) p.occ_part[k] = sc.value();
            }
            os = ss = oc = rowc = 0.0;
            // rowsh, colsh and the item's tiles are rewritten only after every
            // thread passed this barrier
            asm volatile("bar.sync 1, %0;" ::"n"(EPI_THREADS) : "memory");
        };

        uint32_t li = 0, pc = 0;
        int64_t kprev = -1;  // the item whose second half of terms is pending
        uint32_t lprev = 0;
        for (int64_t k = blockIdx.x;; k += gridDim.x, ++li) {
            const bool cur = k < p.items;
            bool two = false, xt = false;
            if (cur) {
                const ItemView v = item_view<BATCH>(p, k);
                const int i = v.i, j = v.j;
                const bool diag = i == j;
                const int ta = v.ta, tb = v.tb;
                const int a = ta * BM + row;
                const bool va = a < v.nvir;
                const double sxa = v.scl[(int64_t)i * v.a_pad + a];
                double* const cb_ = colb + (li & 1) * 3 * BN;
                // the tile's columns (virtual energies, scales of (j, b) and (i, b)) in
                // shared memory: every lane of a warp reads the same column (broadcast)
                {
                    const int cb = tb * BN + (et & (BN - 1));
                    if (et < BN) {
                        cb_[et] = cb < v.nvir ? v.ev[cb] : 0.0;
                        cb_[BN + et] = v.scl[(int64_t)j * v.a_pad + cb];
                    } else if (et < 2 * BN) {
                        cb_[2 * BN + (et - BN)] = v.scl[(int64_t)i * v.a_pad + cb];
                    }
                }
                asm volatile("bar.sync 1, %0;" ::"n"(EPI_THREADS) : "memory");
                const double* sxb = cb_ + BN + h * HC;
                const double* syb = cb_ + 2 * BN + h * HC;
                xt = v.xt;
                two = !diag && !xt;  // a Y phase follows in TMEM
                // X phase -> X tile.  One thread waits (bounded); the epilogue
                // threads leave together if it gave up, since named barriers follow.
                if (!tc::bar_and<1, EPI_THREADS>(et != 0 || tc::mbar_wait(tfull, pc & 1, abort_flag, p.err))) break;
                if (et != 0) tc::mbar_wait(tfull, pc & 1, abort_flag, p.err);  // phase complete: returns at once
                tc::fence_after_sync();
                {
                    // (ia|ia) on the diagonal of an i == j block's diagonal tile
                    const int gdv = (diag && ta == tb && va) ? row - h * HC : -1;
                    const double gval = gdv >= 0 ? v.gd[(int64_t)i * v.a_pad + a] : 0.0;
                    double* const xcol = scr0 + (li & 1) * BM * BN + h * HC * BM + row;
                    // a warp whose columns or rows lie wholly past the last virtual
                    // drains nothing: those tile entries are never read
                    if (h * HC < v.nvir - tb * BN && q * 32 < v.nvir - ta * BM)
                        drain_levels(tl, sxa, sxb, xcol, (gdv >= 0 && gdv < HC) ? gdv : -1, gval);
                }
                tc::fence_before_sync();
                tc::mbar_arrive(tempty);
                ++pc;
                (void)syb;
            }
            if (kprev >= 0) {
                terms(kprev, lprev, HH);
                finish(kprev, lprev);
                kprev = -1;
            }
            if (!cur) break;
            if (two) {
                const ItemView v = item_view<BATCH>(p, k);
                const double sya = v.scl[(int64_t)v.j * v.a_pad + v.ta * BM + row];
                const double* syb = colb + (li & 1) * 3 * BN + 2 * BN + h * HC;
                // Y phase: (ib|ja) = G_ji[a, b] -> Y tile
                if (!tc::bar_and<1, EPI_THREADS>(et != 0 || tc::mbar_wait(tfull, pc & 1, abort_flag, p.err))) break;
                if (et != 0) tc::mbar_wait(tfull, pc & 1, abort_flag, p.err);
                tc::fence_after_sync();
                if (h * HC < v.nvir - v.tb * BN && q * 32 < v.nvir - v.ta * BM)
                    drain_levels(tl, sya, syb, ycol, -1, 0.0);
                tc::fence_before_sync();
                tc::mbar_arrive(tempty);  // the level columns are free for the next item
                ++pc;
            }
            // an exchanged tile reads other threads' rows of X
            if (xt) asm volatile("bar.sync 1, %0;" ::"n"(EPI_THREADS) : "memory");
            terms(k, li, 0);
            kprev = (int64_t)k;
            lprev = li;
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 1) {
        __syncwarp();
        tc::tmem_dealloc(tmem_base, 512);
    }
}

// --------------------------------------------------- adjoint contraction --

// One molecule of a batched adjoint contraction: its own tensor maps (in
// global memory), scales, shape and output.
struct GemmMol {
    const CUtensorMap* tA;  // amplitude slices [3][M][K]
    const CUtensorMap* tB;  // Q-row slices [3][N][K]
    const double* rs;
    const double* cs;
    int M, N, nk, tpad, nvir, naux, rows, pad_;
    int64_t nov;
    double* out;
};

struct GemmFxArgs {
    const double* rs;  // [M] scales of the A rows (amplitude rows (i, a))
    const double* cs;  // [N] scales of the B rows (Q)
    int M, N, nk;      // padded to 128; nk = K / 64
    int nTm, nTn;
    int64_t tiles;
    int a_pad, nvir, naux, i0;  // a_pad: pitch of the amplitude rows (i, a)
    int rows;                   // real amplitude rows
    int64_t nov;
    double alpha;
    double* out;  // Gamma (naux, nov)
    int* err;
    int kofs;        // first K column of the B operand (Q-row slices)
    int aofs;        // first K column of the A operand (a K segment of the amplitude slices)
    int accumulate;  // out += instead of out =
    // batch mode: tile t is bitems[t] = (molecule, m-tile, n-tile, 0)
    const int4* bitems;
    const GemmMol* gmols;
};

struct GemmView {
    const CUtensorMap* tA;
    const CUtensorMap* tB;
    const double* rs;
    const double* cs;
    double* out;
    int64_t nov;
    int tm, tn, M, N, nk, tpad, nvir, naux, rows, i0;
};

template <int BATCH>
__device__ __forceinline__ GemmView gemm_view(const GemmFxArgs& p, const CUtensorMap* tmA, const CUtensorMap* tmB,
                                              int64_t t) {
    GemmView v;
    if (BATCH) {
        const int4 it = p.bitems[t];
        const GemmMol& g = p.gmols[it.x];
        v.tA = g.tA;
        v.tB = g.tB;
        v.rs = g.rs;
        v.cs = g.cs;
        v.out = g.out;
        v.nov = g.nov;
        v.tm = it.y;
        v.tn = it.z;
        v.M = g.M;
        v.N = g.N;
        v.nk = g.nk;
        v.tpad = g.tpad;
        v.nvir = g.nvir;
        v.naux = g.naux;
        v.rows = g.rows;
        v.i0 = 0;
    } else {
        v.tA = tmA;
        v.tB = tmB;
        v.rs = p.rs;
        v.cs = p.cs;
        v.out = p.out;
        v.nov = p.nov;
        // groups of GM m-tiles, n-major within a group: a wave of 148 CTAs
        // covers ~12 x 12 tiles, so each A and each B tile of the wave is read
        // by ~12 CTAs at about the same K (n-fastest order swept every B tile
        // in every wave and read ~2x the bytes from DRAM)
        constexpr int GM = 12;
        const int64_t g = t / ((int64_t)GM * p.nTn), r = t % ((int64_t)GM * p.nTn);
        const int gm = (int)(p.nTm - g * GM < GM ? p.nTm - g * GM : GM);
        v.tm = (int)(g * GM + r % gm);
        v.tn = (int)(r / gm);
        v.M = p.M;
        v.N = p.N;
        v.nk = p.nk;
        v.tpad = p.a_pad;
        v.nvir = p.nvir;
        v.naux = p.naux;
        v.rows = p.rows;
        v.i0 = p.i0;
    }
    return v;
}

constexpr int GF_STAGE = 3 * (16384 + 16384);  // 96 KiB
constexpr int GF_STAGES = 2;
constexpr int GF_SMEM = GF_STAGES * GF_STAGE + 1024 + 1024;
// TMA warp, MMA warp and 8 epilogue warps (two per TMEM lane quadrant, 64
// columns each: 64 FP64 values a thread, which 10 warps leave registers for)
constexpr int GF_THREADS = 320;

// out[Q, (i0 + il)*nvir + a] (+)= alpha * s_row s_Q (L0 + L1/254 + L2/254^2)
// for amplitude rows m = il*tpad + a (a < nvir).
template <int BATCH = 0>
__global__ void __launch_bounds__(GF_THREADS, 1)
    gemm_fx_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const GemmFxArgs p) {
    using namespace fx;
    constexpr int S = GF_STAGES;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_u32 = smem_u32(smem_raw);
    const uint32_t base_u32 = (raw_u32 + 1023u) & ~1023u;
    uint8_t* base = smem_raw + (base_u32 - raw_u32);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * GF_STAGE);
    uint64_t* full = bars;
    uint64_t* empty = bars + S;
    uint64_t* tfull = bars + 2 * S;
    uint64_t* tempty = bars + 2 * S + 1;
    uint64_t* drain = bars + 2 * S + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 3);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    // a stage arrives in two parts: slices 0 and 1 of A and B (full), then
    // slice 2 (full2); the four products of slices 0 and 1 start on the first
    uint64_t* full2 = bars + 2 * S + 4;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&full2[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(tfull, 1);
        tc::mbar_init(tempty, GF_THREADS - 64);
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::fence_barrier_init();
    }
    if (warp == 0 && lane == 0 && !BATCH) {
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 512);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;
    auto sa = [&](int s, int sl) { return base_u32 + s * GF_STAGE + sl * 16384; };
    auto sb = [&](int s, int sl) { return base_u32 + s * GF_STAGE + 3 * 16384 + sl * 16384; };

    if (warp == 0) {
        if (lane == 0) {
            uint32_t g = 0;
            for (int64_t t = blockIdx.x; t < p.tiles && !*abort_flag; t += gridDim.x) {
                const GemmView v = gemm_view<BATCH>(p, &tmA, &tmB, t);
                if (BATCH) {
                    tc::tmap_acquire(v.tA);
                    tc::tmap_acquire(v.tB);
                }
                for (int kt = 0; kt < v.nk; ++kt, ++g) {
                    const int s = g % S;
                    const uint32_t u = g / S;
                    if (!tc::mbar_wait(&empty[s], (u & 1) ^ 1, abort_flag, p.err)) goto prod_done;
                    tc::mbar_arrive_expect_tx(&full[s], GF_STAGE / 3 * 2);
                    tc::mbar_arrive_expect_tx(&full2[s], GF_STAGE / 3);
#pragma unroll
                    for (int sl = 0; sl < 3; ++sl) {
                        uint64_t* bar = sl < 2 ? &full[s] : &full2[s];
                        tc::tma_load_2d(base + (sa(s, sl) - base_u32), v.tA, bar, p.aofs + kt * KT,
                                        sl * v.M + v.tm * 128);
                        tc::tma_load_2d(base + (sb(s, sl) - base_u32), v.tB, bar, p.kofs + kt * KT,
                                        sl * v.N + v.tn * 128);
                    }
                }
            }
        prod_done:
            for (uint32_t q = 0; q < (uint32_t)S && q < g; ++q) {
                const uint32_t gg = g - 1 - q;
                int no_abort = 0;
                tc::mbar_wait(&full[gg % S], (gg / S) & 1, &no_abort, p.err);
                tc::mbar_wait(&full2[gg % S], (gg / S) & 1, &no_abort, p.err);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint64_t da0 = tc::sdesc_k128(sa(0, 0)), da1 = tc::sdesc_k128(sa(1, 0));
            uint32_t g = 0, li = 0;
            for (int64_t t = blockIdx.x; t < p.tiles && !*abort_flag; t += gridDim.x, ++li) {
                const int nk = BATCH ? p.gmols[p.bitems[t].x].nk : p.nk;
                if (!tc::mbar_wait(tempty, (li & 1) ^ 1, abort_flag, p.err)) break;
                tc::fence_after_sync();
                for (int kt = 0; kt < nk; ++kt, ++g) {
                    const int s = g % S;
                    const uint32_t u = g / S;
                    if (!tc::mbar_wait(&full[s], u & 1, abort_flag, p.err)) goto mma_done;
                    tc::fence_after_sync();
                    issue_products<3 * 16384, 1>(s ? da1 : da0, tmem_base, kt);
                    if (!tc::mbar_wait(&full2[s], u & 1, abort_flag, p.err)) goto mma_done;
                    tc::fence_after_sync();
                    issue_products<3 * 16384, 2>(s ? da1 : da0, tmem_base, kt);
                    tc::umma_commit(&empty[s]);
                }
                tc::umma_commit(tfull);
            }
        mma_done:
            tc::umma_commit(drain);
            int no_abort = 0;
            tc::mbar_wait(drain, 0, &no_abort, p.err);
        }
        __syncwarp();
    } else {
        // Epilogue: lane quadrant q = warp % 4, column half h; each thread owns
        // amplitude row `row` of the tile and aux columns [64h, 64h + 64).  It
        // combines its three level accumulators into FP64 registers and
        // releases TMEM before touching Gamma, so the read-modify-write of
        // Gamma runs under the next tile's MMAs (with one thread per row
        // holding TMEM through it, the MMAs waited ~8% of the time).
        const int q = warp & 3;
        const int h = (warp - 2) >> 2;
        const int row = q * 32 + lane;
        uint32_t li = 0;
        for (int64_t t = blockIdx.x; t < p.tiles; t += gridDim.x, ++li) {
            const GemmView v = gemm_view<BATCH>(p, &tmA, &tmB, t);
            if (!tc::mbar_wait(tfull, li & 1, abort_flag, p.err)) break;
            tc::fence_after_sync();
            const int m = v.tm * 128 + row;         // amplitude row (i - i0, a)
            const int il = m / v.tpad, a = m % v.tpad;
            const bool vm = a < v.nvir && m < v.rows;
            const double sr = vm ? p.alpha * v.rs[m] : 0.0;
            double* orow = v.out + (int64_t)(v.i0 + il) * v.nvir + a;
            const uint32_t tl = tmem_base + ((uint32_t)(q * 32) << 16) + h * 64;
            const int q0 = v.tn * 128 + h * 64;     // first aux row Q of this thread's columns
            double gv[64];
#pragma unroll
            for (int c0 = 0; c0 < 64; c0 += 16) {
                float l0[16], l1[16], l2[16];
                tc::tmem_ld16(tl + c0, l0);
                tc::tmem_ld16(tl + 128 + c0, l1);
                tc::tmem_ld16(tl + 256 + c0, l2);
                tc::tmem_wait_ld();
#pragma unroll
                for (int cc = 0; cc < 16; ++cc) {
                    const int Q = q0 + c0 + cc;
                    gv[c0 + cc] = level_value(l0[cc], l1[cc], l2[cc], Q < v.naux ? sr * v.cs[Q] : 0.0);
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(tempty);
            if (vm) {
                // the 16 old Gamma values of a column chunk (nov apart) are
                // loaded together, then updated
#pragma unroll
                for (int c0 = 0; c0 < 64; c0 += 16) {
                    double old[16];
#pragma unroll
                    for (int cc = 0; cc < 16; ++cc) {
                        const int Q = q0 + c0 + cc;
                        old[cc] = p.accumulate && Q < v.naux ? orow[(int64_t)Q * v.nov] : 0.0;
                    }
#pragma unroll
                    for (int cc = 0; cc < 16; ++cc) {
                        const int Q = q0 + c0 + cc;
                        if (Q < v.naux) orow[(int64_t)Q * v.nov] = p.accumulate ? old[cc] + gv[c0 + cc] : gv[c0 + cc];
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 1) {
        __syncwarp();
        tc::tmem_dealloc(tmem_base, 512);
    }
}

// ------------------------------------------------------------ reductions --

__global__ void __launch_bounds__(1024) fx_reduce_pairs_kernel(const double* __restrict__ part, int64_t n,
                                                               double* out) {
    __shared__ double so[1024], sss[1024];
    KSum a, b;
    for (int64_t k = threadIdx.x; k < n; k += 1024) {
        a.add(part[2 * k]);
        b.add(part[2 * k + 1]);
    }
    so[threadIdx.x] = a.value();
    sss[threadIdx.x] = b.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum x, y;
        for (int k = 0; k < 1024; ++k) {
            x.add(so[k]);
            y.add(sss[k]);
        }
        out[0] = x.value();
        out[1] = y.value();
    }
}

// acc_occ[o] += sum of the t Tt partials of every item whose pair holds o,
// for o in I (blocks 0 .. ni-1) and in J (the rest); fixed order.
__global__ void __launch_bounds__(256) fx_reduce_occ_kernel(const double* __restrict__ occ_part,
                                                            const int2* __restrict__ pairs, int64_t npairs,
                                                            int ntiles, int i0, int ni, int j0,
                                                            double* acc_occ) {
    __shared__ double sh[256];
    const int o = (int)blockIdx.x < ni ? i0 + (int)blockIdx.x : j0 + ((int)blockIdx.x - ni);
    KSum a;
    const int64_t n = npairs * ntiles;
    for (int64_t k = threadIdx.x; k < n; k += 256) {
        const int2 pr = pairs[k / ntiles];
        if (pr.x == o || pr.y == o) a.add(occ_part[k]);
    }
    sh[threadIdx.x] = a.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum x;
        for (int k = 0; k < 256; ++k) x.add(sh[k]);
        acc_occ[o] += x.value();
    }
}

__global__ void scale_copy_kernel(const double* __restrict__ x, int64_t n, double s, double* __restrict__ y) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) y[k] = s * x[k];
}

// acc_vir[v] += 2 * (sum over the launch's items of the row-virtual partials
// of v (v in the a-tile) and of the column-virtual partials (v in the b-tile;
// present for mirrored tiles and for pairs i < j)), in two coalesced
// fixed-order passes.  Pass 1: one block per (virtual
// tile tv, chunk of pairs), one thread per virtual of the tile; for each pair
// of the chunk in order it visits only the tile pairs that hold tv -- (tv, tb)
// for the row part, (ta, tv) for the column part -- and reads their 128
// partials as one 1 KB row.  Tile pairs are numbered ta-major with tb >= ta.
// Pass 2 folds the chunks in order.
__global__ void __launch_bounds__(128) fx_reduce_vir_part_kernel(const double* __restrict__ vir_part,
                                                                 const int2* __restrict__ pairs, int64_t npairs,
                                                                 int nT, int ntiles, int64_t pairs_per_chunk,
                                                                 double* __restrict__ out) {
    const int tv = blockIdx.x, rv = threadIdx.x;
    const int64_t p0 = (int64_t)blockIdx.y * pairs_per_chunk;
    const int64_t p1 = p0 + pairs_per_chunk < npairs ? p0 + pairs_per_chunk : npairs;
    auto tidx = [&](int ta, int tb) { return ta * nT - ta * (ta - 1) / 2 + (tb - ta); };
    KSum s;
    for (int64_t p = p0; p < p1; ++p) {
        const int2 pr = pairs[p];
        const double* base = vir_part + p * ntiles * 2 * fx::BM;
        for (int tb = tv; tb < nT; ++tb) s.add(base[(int64_t)tidx(tv, tb) * 2 * fx::BM + rv]);
        for (int ta = 0; ta <= tv; ++ta)
            if (ta < tv || pr.x != pr.y) s.add(base[(int64_t)tidx(ta, tv) * 2 * fx::BM + fx::BM + rv]);
    }
    out[((int64_t)blockIdx.y * nT + tv) * fx::BM + rv] = s.value();
}

__global__ void fx_reduce_vir_fold_kernel(const double* __restrict__ part, int nchunk, int nT, int nvir,
                                          double* acc_vir) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvir) return;
    KSum s;
    for (int c = 0; c < nchunk; ++c) s.add(part[(int64_t)c * nT * fx::BM + v]);
    acc_vir[v] += 2.0 * s.value();
}

// ------------------------------------------------------- batch kernels --
//
// One launch covers every molecule of a batch (or of one group of it): the
// flat block (or thread, or warp) index is mapped to its molecule by a binary
// search over a per-molecule prefix of that launch's work units.

// Everything the batched split / reduce kernels need about one molecule.
struct BatchPrep {
    const double* b;   // B_ov (naux, nocc*nvir)
    int64_t naux, nocc, nvir, a_pad, q_pad, tpad, ldt, q_rows, M;
    unsigned long long* cmax;  // [nocc*nvir]
    double* scl;               // [nocc*a_pad] pair-operand row scales
    double* gd;                // [nocc*a_pad] exact (ia|ia)
    int8_t* bt;                // pair-operand slices (rows of this molecule)
    double* qs;                // [q_rows] Q-row scales (gradient)
    int8_t* bq;                // Q-row slices [3][q_rows][ldt]
    float* T;                  // amplitudes [nocc*tpad][ldt]
    double* ts;                // [M] amplitude-row scales
    int8_t* Ts;                // amplitude slices [3][M][ldt]
    double* de_docc;           // [nocc]
    double* de_dvir;           // [nvir]
    int64_t seg0;              // first item of this molecule
    int64_t ntp;               // tile pairs (ta <= tb) per occupied pair
};

// Largest m in [lo, hi) with pre[m] <= x.
__device__ __forceinline__ int seg_find(const int64_t* __restrict__ pre, int lo, int hi, int64_t x) {
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

enum BatchPre { PRE_COLMAX, PRE_ROWSCALE, PRE_TRANSPOSE, PRE_QROWS, PRE_TROWS, PRE_OCC, PRE_VIR, PRE_COLSQ, PRE_COUNT };

__global__ void __launch_bounds__(256) batch_colmax_kernel(const BatchPrep* __restrict__ mp,
                                                           const int64_t* __restrict__ pre, int nmol, int* bad) {
    const int64_t x = blockIdx.x;
    const int m = seg_find(pre, 0, nmol, x);
    const BatchPrep& d = mp[m];
    const int64_t nov = d.nocc * d.nvir, nbx = (nov + 255) / 256, loc = x - pre[m];
    colmax_body(d.b, d.naux, nov, 64, d.cmax, bad, loc % nbx, loc / nbx);
}

__global__ void __launch_bounds__(256) batch_row_scale_kernel(const BatchPrep* __restrict__ mp,
                                                              const int64_t* __restrict__ pre, int nmol) {
    const int64_t x = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (x >= pre[nmol]) return;
    const int m = seg_find(pre, 0, nmol, x);
    const BatchPrep& d = mp[m];
    const int64_t r = x - pre[m], i = r / d.a_pad, a = r % d.a_pad;
    d.scl[r] = a < d.nvir ? SliceI8::scale(__longlong_as_double((long long)d.cmax[i * d.nvir + a])) : 1.0;
}

__global__ void __launch_bounds__(256) batch_transpose_kernel(const BatchPrep* __restrict__ mp,
                                                              const int64_t* __restrict__ pre, int nmol) {
    const int64_t x = blockIdx.x;
    const int m = seg_find(pre, 0, nmol, x);
    const BatchPrep& d = mp[m];
    const int64_t nbx = (d.nocc * d.nvir + 63) / 64, loc = x - pre[m];
    split_pair4_body(d.b, d.naux, d.nocc, d.nvir, d.a_pad, d.q_pad, d.scl, d.bt, loc % nbx, loc / nbx);
}

__global__ void __launch_bounds__(256) batch_colsq_kernel(const BatchPrep* __restrict__ mp,
                                                          const int64_t* __restrict__ pre, int nmol) {
    const int64_t x = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (x >= pre[nmol]) return;
    const int m = seg_find(pre, 0, nmol, x);
    const BatchPrep& d = mp[m];
    colsq_body(d.b, d.naux, d.nvir, d.nocc * d.nvir, d.a_pad, x - pre[m], d.gd);
}

__global__ void __launch_bounds__(256) batch_qrows_kernel(const BatchPrep* __restrict__ mp,
                                                          const int64_t* __restrict__ pre, int nmol) {
    const int64_t x = blockIdx.x;
    const int m = seg_find(pre, 0, nmol, x);
    const BatchPrep& d = mp[m];
    split_fx_qrows_body<SliceI8>(d.b, d.nocc, d.nvir, d.tpad, d.ldt, d.q_rows, d.qs, d.bq, x - pre[m]);
}

// Amplitude rows of the molecules [m0, m1).
__global__ void __launch_bounds__(256) batch_trows_kernel(const BatchPrep* __restrict__ mp,
                                                          const int64_t* __restrict__ pre, int m0, int m1) {
    const int64_t x = pre[m0] + blockIdx.x;
    const int m = seg_find(pre, m0, m1, x);
    const BatchPrep& d = mp[m];
    split_fx_rows_f32_body<SliceI8>(d.T, d.nocc * d.tpad, d.ldt, d.M, d.ts, d.Ts, x - pre[m]);
}

// dE/deps_o = -2 sum of the t Tt partials of the items of every pair holding o.
// Pairs i <= j are numbered row-major (pidx); partner s gives the pair
// (min(s, o), max(s, o)).
__global__ void __launch_bounds__(256) batch_occ_kernel(const BatchPrep* __restrict__ mp,
                                                        const int64_t* __restrict__ pre, int m0, int m1,
                                                        const double* __restrict__ occ_part) {
    __shared__ double sh[256];
    const int64_t x = pre[m0] + blockIdx.x;
    const int m = seg_find(pre, m0, m1, x);
    const BatchPrep& d = mp[m];
    const int64_t o = x - pre[m], n = d.nocc;
    KSum a;
    for (int64_t u = threadIdx.x; u < n * d.ntp; u += 256) {
        const int64_t sp = u / d.ntp, t = u % d.ntp;
        const int64_t i = sp < o ? sp : o, j = sp < o ? o : sp;
        const int64_t pidx = i * n - i * (i - 1) / 2 + (j - i);
        a.add(occ_part[d.seg0 + pidx * d.ntp + t]);
    }
    sh[threadIdx.x] = a.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum t;
        for (int k = 0; k < 256; ++k) t.add(sh[k]);
        d.de_docc[o] = -2.0 * t.value();
    }
}

// dE/deps_v = 2 sum of the row-virtual partials of v (v in the a-tile) and
// the column-virtual partials (v in the b-tile; mirrored tiles and pairs
// i < j); one warp per v.  vir_part is indexed from the group's first item g0.
__global__ void __launch_bounds__(256) batch_vir_kernel(const BatchPrep* __restrict__ mp,
                                                        const int64_t* __restrict__ pre, int m0, int m1,
                                                        const int4* __restrict__ items, int64_t g0,
                                                        const double* __restrict__ vir_part) {
    const int64_t x = pre[m0] + (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (x >= pre[m1]) return;
    const int m = seg_find(pre, m0, m1, x);
    const BatchPrep& d = mp[m];
    const int v = (int)(x - pre[m]);
    const int tv = v / fx::BM, rv = v % fx::BM;
    const int64_t k1 = d.seg0 + d.nocc * (d.nocc + 1) / 2 * d.ntp;
    KSum s;
    for (int64_t k = d.seg0 + lane; k < k1; k += 32) {
        const int4 it = items[k];
        const int ta = it.w & 0xFFFF, tb = it.w >> 16;
        const double* vp = vir_part + (k - g0) * 2 * fx::BM;
        if (ta == tv) s.add(vp[rv]);
        if (tb == tv && (ta < tb || it.y != it.z)) s.add(vp[fx::BM + rv]);
    }
    const double r = warp_sum(s.value());
    if (lane == 0) d.de_dvir[v] = 2.0 * r;
}

// Per-molecule (e_os, e_ss) of the molecules [m0, m1): items [seg[m], seg[m+1]).
__global__ void __launch_bounds__(256) batch_energy_kernel(const double* __restrict__ part,
                                                           const int64_t* __restrict__ seg, int m0,
                                                           double* out) {
    __shared__ double so[256], sn[256];
    const int m = m0 + blockIdx.x;
    KSum a, b;
    for (int64_t k = seg[m] + threadIdx.x; k < seg[m + 1]; k += 256) {
        a.add(part[2 * k]);
        b.add(part[2 * k + 1]);
    }
    so[threadIdx.x] = a.value();
    sn[threadIdx.x] = b.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum x, y;
        for (int t = 0; t < 256; ++t) {
            x.add(so[t]);
            y.add(sn[t]);
        }
        out[2 * m] = x.value();
        out[2 * m + 1] = y.value();
    }
}

// ------------------------------------------------------------------ host --

namespace {

// naux up to which the int32 level sums of the pair kernel are exact: up to
// four int8 products per level, 4 * 127^2 * naux <= 2^31 - 1 (and the FP64
// combination of the four levels stays an integer below 2^53).
constexpr int64_t PAIR_KMAX = 33286;

struct FxSplit {
    int8_t* bt;
    double* scl;
    double* gd;  // exact (ia|ia) per operand row
    unsigned long long* cmax;
    int64_t a_pad, q_pad;
    CUtensorMap tmA, tmB;
};

// The pair operands: buffers (zeroed: padding rows and columns stay 0) and
// tensor maps; fx_split_range fills the slices of occupied orbitals [o0, o1).
fc_status fx_split_alloc(const Rimp2Dev& d, cudaStream_t st, FxSplit* o) {
    const int64_t a_pad = (d.nvir + fx::BM - 1) / fx::BM * fx::BM;
    const int64_t q_pad = (d.naux + fx::PKT - 1) / fx::PKT * fx::PKT;
    const int64_t nov = d.nocc * d.nvir;
    const int64_t rows = (int64_t)fx::PSL * d.nocc * a_pad;
    if (d.naux > PAIR_KMAX)
        return fail(FC_ERR_LAYOUT, "mixed RI-MP2: naux > 33286 exceeds the exact int32 level sums (use FP64)");
    if ((d.naux + 63) / 64 > 65535) return fail(FC_ERR_LAYOUT, "split: naux too large");
    if (rows > (int64_t)INT32_MAX) return fail(FC_ERR_LAYOUT, "split: too many operand rows");
    void *vbt, *vscl;
    FC_TRY(ws_get(WS_SPLIT, (size_t)rows * q_pad, &vbt));
    FC_TRY(ws_get(WS_SCALE, (size_t)(nov + 2 * d.nocc * a_pad) * 8 + 256, &vscl));
    o->cmax = (unsigned long long*)vscl;
    o->scl = (double*)vscl + nov;
    o->gd = o->scl + d.nocc * a_pad;
    FC_CUDA(cudaMemsetAsync(o->cmax, 0, nov * 8, st));
    FC_CUDA(cudaMemsetAsync(vbt, 0, (size_t)rows * q_pad, st));
    FC_TRY(make_tmap_i8_2d_sw64(&o->tmA, vbt, q_pad, rows, q_pad, fx::BM));
    FC_TRY(make_tmap_i8_2d_sw64(&o->tmB, vbt, q_pad, rows, q_pad, fx::BN));
    o->bt = (int8_t*)vbt;
    o->a_pad = a_pad;
    o->q_pad = q_pad;
    return FC_OK;
}

fc_status fx_split_range(const Rimp2Dev& d, cudaStream_t st, int* bad, const FxSplit& o, int64_t o0, int64_t o1) {
    const int64_t nov = d.nocc * d.nvir;
    const int64_t c0 = o0 * d.nvir, nc = (o1 - o0) * d.nvir;
    {
        const int64_t rps = 64;
        dim3 g((unsigned)((nc + 255) / 256), (unsigned)((d.naux + rps - 1) / rps));
        colmax_kernel<<<g, 256, 0, st>>>(d.b_ov, d.naux, nc, rps, o.cmax, bad, nov, c0);
    }
    colsq_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(d.b_ov, d.naux, d.nvir, nov, o.a_pad, c0, c0 + nc,
                                                               o.gd);
    const int64_t r0 = o0 * o.a_pad, r1 = o1 * o.a_pad;
    row_scale_kernel<SliceI8><<<(unsigned)((r1 - r0 + 255) / 256), 256, 0, st>>>(o.cmax, d.nocc, d.nvir, o.a_pad,
                                                                                 o.scl, r0, r1);
    {
        dim3 g((unsigned)((nc + 63) / 64), (unsigned)((d.naux + 63) / 64));
        split_pair4_kernel<<<g, 256, 0, st>>>(d.b_ov, d.naux, d.nocc, d.nvir, o.a_pad, o.q_pad, o.scl, o.bt, c0,
                                              c0 + nc);
    }
    return check_launch("fixed-point split kernels");
}

fc_status fx_split_pairs(const Rimp2Dev& d, cudaStream_t st, int* bad, FxSplit* o) {
    FC_TRY(fx_split_alloc(d, st, o));
    return fx_split_range(d, st, bad, *o, 0, d.nocc);
}

fc_status fx_attrs() {
    static std::atomic<uint64_t> done{0};
    uint64_t bit = 0;
    if (!attrs_needed(done, &bit)) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(pair_fx_kernel<0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx::SMEM));
    FC_CUDA(cudaFuncSetAttribute(pair_fx_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx::SMEM));
    FC_CUDA(cudaFuncSetAttribute(pair_fx_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx::SMEM));
    FC_CUDA(cudaFuncSetAttribute(gemm_fx_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, GF_SMEM));
    FC_CUDA(cudaFuncSetAttribute(gemm_fx_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, GF_SMEM));
    FC_CUDA(cudaFuncSetAttribute(pair_fx_kernel<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx::SMEM));
    done.fetch_or(bit);
    return FC_OK;
}

}  // namespace

// Diagonal tiles (ta == tb, i != j) in one tensor-core phase with the
// transpose read back from the CTA's X tile (1), or in two phases (0).  The
// exchange saves a phase of MMAs for the price of strided (coalesced) reads
// of the X tile, so it is the default; FERRIC_CUDA_XT=0/1 forces it.
int fx_ksteps(int64_t naux) { return (int)((naux + fx::PKT - 1) / fx::PKT); }

int fx_exchange_choice(int nk, int grad) {
    (void)nk;
    (void)grad;
    const char* e = std::getenv("FERRIC_CUDA_XT");
    if (e && (e[0] == '0' || e[0] == '1')) return e[0] == '1';
    return 1;
}

// Failure-path test hook of the pair kernel.  FERRIC_CUDA_WAIT_MS bounds the
// MMA warp's waits for operand stages (default 4 s); with
// FERRIC_CUDA_TEST_DROP_LOAD=1 CTA 0's producer issues no load for its first
// stage, so that bounded wait runs out (nothing in flight, FC_ERR_TIMEOUT)
// while every other wait of the kernel keeps its 4 s limit.
static void fx_test_hooks(PairFxArgs* a) {
    a->wait_ns = tc::WAIT_LIMIT_NS;
    if (const char* e = std::getenv("FERRIC_CUDA_WAIT_MS")) {
        const long long v = std::atoll(e);
        if (v > 0 && v <= 60000) a->wait_ns = (uint64_t)v * 1000000ull;
    }
    const char* d = std::getenv("FERRIC_CUDA_TEST_DROP_LOAD");
    a->drop_load = (d && d[0] == '1') ? 1 : 0;
}

// FP64 X / Y tiles of the pair kernel's CTAs (global scratch, L2-resident).
fc_status pair_scratch(int grid, double** out) {
    void* v;
    FC_TRY(ws_get(WS_PSCR, (size_t)grid * 3 * fx::BM * fx::BN * sizeof(double), &v));
    *out = (double*)v;
    return FC_OK;
}

fc_status rimp2_energy_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss, fc_stats* stats) {
    FC_TRY(fx_attrs());
    if (d.nocc > (1 << 15)) return fail(FC_ERR_LAYOUT, "mixed RI-MP2: nocc too large");
    void* vout;
    FC_TRY(ws_get(WS_OUT, 256, &vout));
    double* out = (double*)vout;
    int* flags = (int*)(out + 4);  // [0] range, [1] timeout
    FC_CUDA(cudaMemsetAsync(vout, 0, 256, st));
    Context& c = ctx();
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    FxSplit sp;
    FC_TRY(fx_split_pairs(d, st, flags, &sp));
    const int nocc = (int)d.nocc;
    const int nT = (int)(sp.a_pad / fx::BM);
    int64_t plo, phi;  // this shard's pairs (all of them unsharded)
    shard_pair_range(nocc, d.shard, d.nshards, &plo, &phi);
    std::vector<int2> pairs;
    for (int64_t i = 0, k = 0; i < nocc; ++i)
        for (int64_t j = i; j < nocc; ++j, ++k)
            if (k >= plo && k < phi) pairs.push_back(make_int2((int)i, (int)j));
    const size_t npairs = pairs.size();
    if (npairs == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        if (stats) stats->precision = FC_PREC_MIXED;
        return FC_OK;
    }
    for (int ta = 0; ta < nT; ++ta)
        for (int tb = ta; tb < nT; ++tb) pairs.push_back(make_int2(ta, tb));
    void* vtab;
    FC_TRY(ws_get(WS_PAIRS, pairs.size() * sizeof(int2), &vtab));
    FC_CUDA(cudaMemcpyAsync(vtab, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    PairFxArgs a{};
    fx_test_hooks(&a);
    a.eo = d.eps_occ;
    a.ev = d.eps_vir;
    a.scl = sp.scl;
    a.pairs = (const int2*)vtab;
    a.tiles = (const int2*)vtab + npairs;
    a.ntiles = nT * (nT + 1) / 2;
    a.npairs = (int)npairs;
    a.nocc = nocc;
    a.nvir = (int)d.nvir;
    a.a_pad = (int)sp.a_pad;
    a.nTa = (int)(sp.a_pad / fx::BM);
    a.nTb = (int)(sp.a_pad / fx::BN);
    a.nk = (int)(sp.q_pad / fx::PKT);
    a.tpad = a.a_pad;
    a.xt = fx_exchange_choice(a.nk, 0);
    a.items = (int64_t)a.npairs * a.ntiles;
    a.gd = sp.gd;
    void* vpart;
    FC_TRY(ws_get(WS_PART, a.items * 2 * sizeof(double), &vpart));
    a.part = (double*)vpart;
    a.err = flags + 1;
    const int grid = (int)(a.items < c.sm_count ? a.items : c.sm_count);
    FC_TRY(pair_scratch(grid, &a.scr));
    cudaEvent_t* ev = nullptr;
    if (stats) {
        FC_TRY(timing_events(1, &ev));
        FC_CUDA(cudaEventRecord(ev[0], st));
    }
    pair_fx_kernel<0><<<grid, fx::PAIR_THREADS, fx::SMEM, st>>>(sp.tmA, sp.tmB, a);
    FC_TRY(check_launch("pair_fx_kernel<energy>"));
    if (stats) FC_CUDA(cudaEventRecord(ev[1], st));
    fx_reduce_pairs_kernel<<<1, 1024, 0, st>>>((const double*)vpart, a.items, out);
    FC_TRY(check_launch("fx_reduce_pairs_kernel"));
    if (stats) FC_CUDA(cudaEventRecord(c.ev1, st));
    double h[2];
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "mixed RI-MP2: B_ov has a non-finite element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "mixed pair kernel: a pipeline wait ran out");
    *e_os = h[0];
    *e_ss = h[1];
    if (stats) {
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        const double P = (double)d.nocc * (d.nocc + 1) / 2.0;
        stats->flops = 2.0 * (double)d.naux * (double)d.nvir * (double)d.nvir * P;
        stats->precision = FC_PREC_MIXED;
        stats->launches += 6;
        stats->tile_m = fx::BM;
        stats->tile_n = fx::BN;
        stats->k_panel = 0;
        stats->main_launches = 1;
        FC_TRY(timing_sum(1, &stats->main_ms));
        stats->main_flops = stats->flops;
        stats->main_bytes = 8.0 * (double)d.naux * (double)(d.nocc * d.nvir);
        stats->h2d_bytes += pairs.size() * sizeof(int2);
        stats->d2h_bytes += sizeof(h) + sizeof(hf);
    }
    return FC_OK;
}

fc_status rimp2_grad_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss, double* gamma,
                        double* de_docc, double* de_dvir, fc_stats* stats, const GammaSink* sink,
                        const DensOut* dens) {
    FC_TRY(fx_attrs());
    if (d.nocc > (1 << 15)) return fail(FC_ERR_LAYOUT, "mixed RI-MP2: nocc too large");
    if (dens && d.nshards != 1) return fail(FC_ERR_INVALID, "RI-MP2 densities: no sharded form");
    const int64_t nocc = d.nocc, nvir = d.nvir, naux = d.naux, nov = nocc * nvir;
    Context& c = ctx();
    FxSplit sp;
    void* vout0;
    FC_TRY(ws_get(WS_OUT, 256, &vout0));
    int* flags = (int*)vout0;  // [0] range, [1] timeout
    FC_CUDA(cudaMemsetAsync(vout0, 0, 256, st));
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    FC_TRY(fx_split_alloc(d, st, &sp));
    const int64_t a_pad = sp.a_pad;
    const int64_t tp = (nvir + 15) / 16 * 16;  // amplitude pitch: rows (i, a) and columns (j, b), a, b < tp
                                               // (16: int8 slice columns of a chunk start 16-byte aligned)
    const int64_t K2 = nocc * tp;           // (j, b) columns of the Q-row slices
    const int64_t q_rows = (naux + 127) / 128 * 128;
    const int nTa = (int)(a_pad / fx::BM);
    const int ntiles = nTa * (nTa + 1) / 2;  // tiles ta <= tb

    // occupied chunks: a chunk pair (I, J), I <= J, holds the amplitude rows of
    // I (columns of J) and of J (columns of I) in FP32, plus the slices of one
    // of them; each unordered pair (i, j) is computed once and feeds both.
    // with densities the chunk is also bounded by the slab budget (four
    // chunk budgets: the slabs are the densities' whole working set)
    const int64_t cc = dens ? dens_chunk_fx(nocc, nvir, grad_chunk_fx(nocc, nvir, d.chunk_bytes, 1),
                                            4 * d.chunk_bytes)
                            : grad_chunk_fx(nocc, nvir, d.chunk_bytes, d.nshards);
    const int64_t nch = (nocc + cc - 1) / cc;
    struct CP {
        int64_t i0, ni, j0, nj, p0, np;
    };
    std::vector<CP> cps;
    std::vector<int2> pairs;
    std::vector<int64_t> cp_index((size_t)(nch * nch), -1);  // [I][J], I <= J
    for (int64_t I = 0; I < nch; ++I)
        for (int64_t J = I; J < nch; ++J) {
            cp_index[(size_t)(I * nch + J)] = (int64_t)cps.size();
            CP x;
            x.i0 = I * cc;
            x.ni = std::min(cc, nocc - x.i0);
            x.j0 = J * cc;
            x.nj = std::min(cc, nocc - x.j0);
            x.p0 = (int64_t)pairs.size();
            for (int64_t i = x.i0; i < x.i0 + x.ni; ++i)
                for (int64_t j = (I == J ? i : x.j0); j < x.j0 + x.nj; ++j) pairs.push_back(make_int2((int)i, (int)j));
            x.np = (int64_t)pairs.size() - x.p0;
            cps.push_back(x);
        }
    const int64_t npairs_all = (int64_t)pairs.size();
    for (int ta = 0; ta < nTa; ++ta)
        for (int tb = ta; tb < nTa; ++tb) pairs.push_back(make_int2(ta, tb));
    const int64_t ncp = (int64_t)cps.size();
    const std::vector<int> owner = chunk_pair_owner(nocc, cc, d.nshards);
    int64_t max_items = 0;
    for (const auto& x : cps) max_items = std::max(max_items, x.np * ntiles);
    // The run order.  Gradient: each chunk pair once, both of its amplitude
    // blocks.  Densities: by column chunk K, the block (I, K) of every I from
    // chunk pair (min, max) -- T (rows of its first chunk) when I <= K, T2
    // otherwise; the energy and dE/deps terms of a chunk pair are taken at
    // its I <= K visit.  The slab of K is complete after its last step.
    //
    // Densities kept without recomputation (the store form, when the blocks
    // above the diagonal fit 8 chunk budgets; FERRIC_CUDA_DENS_STORE=0 forces
    // the recomputing form): column chunk K runs chunk pairs (K, I), I >= K,
    // once each -- T2 = block (I, K) goes to K's slab, T = block (K, I), I > K,
    // is kept in FP32 until column I, whose slab takes it first (its Tt and t
    // slices; its adjoint ran when it was made).
    struct Step {
        int64_t x;
        int blk;    // 0: T, 1: T2, 2: both (store form: both, T2 to the slab, T to the store)
        bool sums;  // take the chunk pair's energy and dE/deps terms
        bool last;  // last block of the column chunk
        int64_t col = -1;  // store form: the column chunk (the pair's first chunk)
    };
    std::vector<Step> steps;
    std::vector<int64_t> store_off;  // [I][K], I < K: element offset of block (I, K) in the store
    size_t store_elems = 0;
    bool store = false;
    if (dens) {
        store_off.assign((size_t)(nch * nch), -1);
        for (int64_t I = 0; I < nch; ++I)
            for (int64_t K = I + 1; K < nch; ++K) {
                store_off[(size_t)(I * nch + K)] = (int64_t)store_elems;
                store_elems += (size_t)(std::min(cc, nocc - I * cc) * tp) * (size_t)(std::min(cc, nocc - K * cc) * tp);
            }
        const char* e = std::getenv("FERRIC_CUDA_DENS_STORE");
        store = !(e && e[0] == '0') && store_elems * 4 <= (size_t)(8 * d.chunk_bytes);
    }
    if (!dens) {
        for (int64_t x = 0; x < ncp; ++x) steps.push_back({x, 2, true, false});
    } else if (store) {
        for (int64_t K = 0; K < nch; ++K)
            for (int64_t I = K; I < nch; ++I)
                steps.push_back({cp_index[(size_t)(K * nch + I)], 2, true, I == nch - 1, K});
    } else {
        for (int64_t K = 0; K < nch; ++K)
            for (int64_t I = 0; I < nch; ++I)
                steps.push_back({cp_index[(size_t)(std::min(I, K) * nch + std::max(I, K))], I <= K ? 0 : 1, I <= K,
                                 I == nch - 1});
    }
    DensFx dx{};
    float* dstore = nullptr;
    if (dens) FC_TRY(dens_fx_alloc(nocc, nvir, tp, cc, st, &dx));
    if (store && store_elems) {
        void* vs;
        FC_TRY(ws_get(WS_DSTORE, store_elems * 4, &vs));
        dstore = (float*)vs;
    }

    void *vbq, *vtab, *vT, *vTs, *vpart;
    const size_t tab_bytes = ((pairs.size() * sizeof(int2) + 255) / 256) * 256;
    FC_TRY(ws_get(WS_SPLIT2, (size_t)3 * q_rows * K2, &vbq));
    FC_TRY(ws_get(WS_PAIRS, tab_bytes + (size_t)nch * q_rows * 8, &vtab));
    double* qs = (double*)((char*)vtab + tab_bytes);  // [nch][q_rows] Q-row scales per occupied chunk
    const size_t cbytes = (size_t)cc * tp * cc * tp;  // elements of one amplitude block
    const int64_t mp_max = (cc * tp + 127) / 128 * 128;
    FC_TRY(ws_get(WS_T, cbytes * 8 + (size_t)mp_max * 8, &vT));
    FC_TRY(ws_get(WS_TS, (size_t)3 * mp_max * cc * tp, &vTs));
    int64_t max_np = 1;
    for (const auto& x : cps) max_np = std::max(max_np, x.np);
    const int vir_chunks = (int)std::min<int64_t>(max_np, std::max<int64_t>(1, 4 * c.sm_count / nTa));
    FC_TRY(ws_get(WS_PART,
                  (size_t)max_items * (2 + 1 + 2 * fx::BM) * 8 + (size_t)(2 * ncp + nocc) * 8 +
                      (size_t)vir_chunks * nTa * fx::BM * 8,
                  &vpart));
    float* T1 = (float*)vT;
    float* T2 = T1 + cbytes;
    double* ts = (double*)(T2 + cbytes);
    double* part = (double*)vpart;
    double* occ_part = part + 2 * max_items;
    double* vir_part = occ_part + max_items;
    double* e_cp = vir_part + 2 * fx::BM * max_items;  // [ncp][2]
    double* acc_occ = e_cp + 2 * ncp;                  // [nocc]
    double* vir_fold = acc_occ + nocc;                 // [vir_chunks][nTa * 128]
    FC_CUDA(cudaMemcpyAsync(vtab, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemsetAsync(de_dvir, 0, nvir * 8, st));
    FC_CUDA(cudaMemsetAsync(acc_occ, 0, nocc * 8, st));
    FC_CUDA(cudaMemsetAsync(e_cp, 0, 2 * ncp * 8, st));  // chunk pairs of other shards add nothing
    FC_CUDA(cudaMemsetAsync(gamma, 0, (size_t)naux * nov * 8, st));
    // per-Q-row split of B_ov for the adjoint contraction, at one scale per
    // (Q row, occupied chunk): a chunk's slices need only its own columns
    FC_CUDA(cudaMemsetAsync(vbq, 0, (size_t)3 * q_rows * K2, st));
    int64_t nl = 0;  // kernels launched
    fill_kernel<<<(unsigned)((nch * q_rows + 255) / 256), 256, 0, st>>>(qs, nch * q_rows, 1.0);
    ++nl;
    // Occupied chunk J's operands (pair slices and Q-row slices) are made the
    // first time a chunk pair uses it -- after its columns of b_ov arrived,
    // when the caller uploads them chunk by chunk (d.arrive)
    const bool arrive_ok = d.arrive && d.arrive_cc == cc;
    if (d.arrive && !arrive_ok)
        for (int64_t J = 0; J < (nocc + d.arrive_cc - 1) / d.arrive_cc; ++J)
            FC_CUDA(cudaStreamWaitEvent(st, d.arrive[J], 0));
    std::vector<char> ready((size_t)nch, 0);
    auto prep = [&](int64_t J) -> fc_status {
        if (ready[(size_t)J]) return FC_OK;
        if (arrive_ok) FC_CUDA(cudaStreamWaitEvent(st, d.arrive[J], 0));
        const int64_t o0 = J * cc, o1 = std::min(nocc, o0 + cc);
        FC_TRY(fx_split_range(d, st, flags, sp, o0, o1));
        split_fx_qrows_kernel<<<(unsigned)naux, 256, 0, st>>>(d.b_ov, nocc, nvir, tp, K2, q_rows, qs + J * q_rows,
                                                              (int8_t*)vbq, o0 * nvir, o1 * nvir);
        FC_TRY(check_launch("split_fx_qrows_kernel"));
        nl += 4;  // column maxima, scales, pair slices, Q-row slices
        ready[(size_t)J] = 1;
        return FC_OK;
    };
    CUtensorMap tmBq;
    FC_TRY(make_tmap_i8_2d(&tmBq, vbq, K2, 3 * q_rows, K2, fx::KT, 128));
    const int2* dpairs = (const int2*)vtab;
    const int2* dtiles = dpairs + npairs_all;

    cudaEvent_t* ev = nullptr;
    const int64_t nsteps = (int64_t)steps.size();
    int64_t npair_launch = 0;
    double pair_flops = 0.0;
    if (stats) FC_TRY(timing_events((int)nsteps, &ev));
    // K segment of the adjoint contraction: fx::KMAX, or FERRIC_CUDA_KSEG (a
    // positive multiple of fx::KT up to fx::KMAX; tests use short segments)
    int64_t kseg = fx::KMAX;
    if (const char* e = std::getenv("FERRIC_CUDA_KSEG")) {
        const long long v = std::atoll(e);
        if (v > 0 && v % fx::KT == 0 && v <= fx::KMAX) kseg = v;
    }
    // timing of the adjoint launches: at most two blocks per chunk pair, each
    // in ceil(K / kseg) segments
    cudaEvent_t* ev2 = nullptr;
    int nadj = 0;
    double adj_flops = 0.0, adj_bytes = 0.0;
    if (stats) FC_TRY(timing_events2((int)(2 * nsteps * ((cc * tp + kseg - 1) / kseg)), &ev2));
    // Gamma[:, rows] += 4 Bq[:, cols] T^T for one amplitude block
    // (with densities the slices go to the block's rows of the column chunk's
    // slab, slices nocc tp rows apart, and stay there for the density terms)
    // (from_t: T holds the block transposed, [nk tp][nr tp], as T1 of the
    // chunk pair whose T2 was not written; its column maxima go to the T2
    // buffer and a tiled transpose writes the slices of its columns)
    auto adjoint = [&](float* T, int64_t r0, int64_t nr, int64_t k0, int64_t nk, bool to_slab,
                       bool from_t = false) -> fc_status {
        const int64_t ldk = nk * tp, rows = nr * tp, mp = (rows + 127) / 128 * 128;
        const int64_t sstride = to_slab ? dx.rows : mp;  // rows between slices
        int8_t* sl = to_slab ? dx.ts + r0 * tp * ldk : (int8_t*)vTs;
        double* rsc = to_slab ? dx.tsc + r0 * tp : ts;
        if (from_t) {
            unsigned* cmax = reinterpret_cast<unsigned*>(T2);
            constexpr int64_t kSplit = 8;  // row ranges of the column maxima
            FC_CUDA(cudaMemsetAsync(cmax, 0, (size_t)rows * sizeof(unsigned), st));
            colmax_f32_kernel<<<dim3((unsigned)((rows + 127) / 128), (unsigned)kSplit), 256, 0, st>>>(
                T, ldk, rows, rows, (ldk + kSplit - 1) / kSplit, cmax);
            split_cols_f32_kernel<<<dim3((unsigned)((rows + 63) / 64), (unsigned)((ldk + 63) / 64)), 256, 0, st>>>(
                T, ldk, rows, rows, cmax, sstride, rsc, sl);
            FC_TRY(check_launch("split_cols_f32_kernel"));
            nl += 2;
        } else {
            split_fx_rows_f32_kernel<<<(unsigned)rows, 256, 0, st>>>(T, ldk, sstride, rsc, sl);
            ++nl;
        }
        CUtensorMap tmTs;
        FC_TRY(make_tmap_i8_2d(&tmTs, sl, ldk, 3 * sstride - (to_slab ? r0 * tp : 0), ldk, fx::KT, 128));
        GemmFxArgs g{};
        g.rs = rsc;
        g.cs = qs + (k0 / cc) * q_rows;  // the Q-row scales of the column chunk
        g.M = (int)sstride;
        g.N = (int)q_rows;
        g.nTm = (int)(mp / 128);
        g.rows = (int)rows;
        g.nTn = (int)(q_rows / 128);
        g.tiles = (int64_t)g.nTm * g.nTn;
        g.a_pad = (int)tp;
        g.nvir = (int)nvir;
        g.naux = (int)naux;
        g.i0 = (int)r0;
        g.nov = nov;
        g.alpha = 4.0;
        g.out = gamma;
        g.err = flags + 1;
        g.accumulate = 1;
        const int g2 = (int)(g.tiles < c.sm_count ? g.tiles : c.sm_count);
        // K segments of at most kseg (a multiple of KT) keep the int32 level
        // sums exact; each segment adds its part into Gamma
        for (int64_t ks = 0; ks < ldk; ks += kseg) {
            const int64_t kl = std::min<int64_t>(kseg, ldk - ks);
            g.aofs = (int)ks;
            g.kofs = (int)(k0 * tp + ks);
            g.nk = (int)((kl + fx::KT - 1) / fx::KT);
            if (stats) FC_CUDA(cudaEventRecord(ev2[2 * nadj], st));
            gemm_fx_kernel<0><<<g2, GF_THREADS, GF_SMEM, st>>>(tmTs, tmBq, g);
            FC_TRY(check_launch("gemm_fx_kernel"));
            if (stats) FC_CUDA(cudaEventRecord(ev2[2 * nadj + 1], st));
            ++nadj;
            ++nl;
        }
        // algorithmic: Gamma[:, rows] += 4 B[:, cols] T^T, and the bytes of
        // the three Q-row and amplitude slices plus Gamma's read-modify-write
        adj_flops += 2.0 * (double)naux * (double)(nr * nvir) * (double)(nk * nvir);
        adj_bytes += 3.0 * (double)naux * (double)(nk * nvir) + 3.0 * (double)(nr * nvir) * (double)(nk * nvir) +
                     16.0 * (double)naux * (double)(nr * nvir);
        return FC_OK;
    };
    for (size_t sx = 0; sx < steps.size(); ++sx) {
        const Step& step = steps[sx];
        const int64_t x = step.x;
        const CP& cp = cps[x];
        const bool same = cp.i0 == cp.j0;
        if (store && same) {
            // column chunk K starts: its slab rows of chunks I < K come from the store
            const int64_t K = step.col, nk = std::min(cc, nocc - K * cc), ldk = nk * tp;
            for (int64_t I = 0; I < K; ++I) {
                float* blk = dstore + store_off[(size_t)(I * nch + K)];
                const int64_t nr = std::min(cc, nocc - I * cc), rows = nr * tp;
                split_fx_rows_f32_kernel<<<(unsigned)rows, 256, 0, st>>>(blk, ldk, dx.rows, dx.tsc + I * cc * tp,
                                                                       dx.ts + I * cc * tp * ldk);
                ++nl;
                FC_TRY(check_launch("split_fx_rows_f32_kernel<store>"));
                FC_TRY(dens_fx_block(dx, blk, I * cc * tp, nr, nk, st, &nl));
            }
        }
        if (owner[x] != d.shard) {
            if (stats) {
                FC_CUDA(cudaEventRecord(ev[2 * sx], st));
                FC_CUDA(cudaEventRecord(ev[2 * sx + 1], st));
            }
            continue;
        }
        FC_TRY(prep(cp.i0 / cc));
        FC_TRY(prep(cp.j0 / cc));
        PairFxArgs a{};
        fx_test_hooks(&a);
        a.eo = d.eps_occ;
        a.ev = d.eps_vir;
        a.scl = sp.scl;
        a.pairs = dpairs + cp.p0;
        a.tiles = dtiles;
        a.ntiles = ntiles;
        a.npairs = (int)cp.np;
        a.nocc = (int)nocc;
        a.nvir = (int)nvir;
        a.a_pad = (int)a_pad;
        a.nTa = nTa;
        a.nTb = nTa;
        a.nk = (int)(sp.q_pad / fx::PKT);
        a.tpad = (int)tp;
        a.xt = fx_exchange_choice(a.nk, 1);
        a.items = cp.np * ntiles;
        a.gd = sp.gd;
        a.part = part;
        a.err = flags + 1;
        a.T = T1;
        a.ldt = cp.nj * tp;
        a.T2 = same ? T1 : T2;
        a.ldt2 = same ? a.ldt : cp.ni * tp;
        // without densities T2 only feeds the J rows' adjoint, whose slices
        // come from T by a tiled transpose: the pair kernel skips its stores
        a.no_t2 = (!dens && !same) ? 1 : 0;
        a.i0 = (int)cp.i0;
        a.j0 = (int)cp.j0;
        a.occ_part = occ_part;
        a.vir_part = vir_part;
        const int grid = (int)(a.items < c.sm_count ? a.items : c.sm_count);
        FC_TRY(pair_scratch(grid, &a.scr));
        if (stats) FC_CUDA(cudaEventRecord(ev[2 * sx], st));
        pair_fx_kernel<1><<<grid, fx::PAIR_THREADS, fx::SMEM, st>>>(sp.tmA, sp.tmB, a);
        FC_TRY(check_launch("pair_fx_kernel<grad>"));
        if (stats) FC_CUDA(cudaEventRecord(ev[2 * sx + 1], st));
        ++npair_launch;
        pair_flops += 2.0 * naux * (double)nvir * nvir * (double)cp.np;
        if (step.sums) {
            fx_reduce_pairs_kernel<<<1, 1024, 0, st>>>(part, a.items, e_cp + 2 * x);
            fx_reduce_occ_kernel<<<(unsigned)(same ? cp.ni : cp.ni + cp.nj), 256, 0, st>>>(
                occ_part, dpairs + cp.p0, cp.np, ntiles, (int)cp.i0, (int)cp.ni, (int)cp.j0, acc_occ);
            {
                const int nchunk = (int)std::min<int64_t>(vir_chunks, cp.np);
                const int64_t ppc = (cp.np + nchunk - 1) / nchunk;
                fx_reduce_vir_part_kernel<<<dim3((unsigned)nTa, (unsigned)nchunk), 128, 0, st>>>(
                    vir_part, dpairs + cp.p0, cp.np, nTa, ntiles, ppc, vir_fold);
                fx_reduce_vir_fold_kernel<<<(unsigned)((nvir + 127) / 128), 128, 0, st>>>(vir_fold, nchunk, nTa,
                                                                                           (int)nvir, de_dvir);
            }
            FC_TRY(check_launch("gradient reductions"));
            nl += 4;  // the four reductions
        }
        ++nl;  // the pair kernel
        if (store) {
            // chunk pair (K, I), I >= K: T2 = block (I, K) of column K (the
            // slab); T = block (K, I) of column I (the store), or the
            // diagonal block (K, K) of column K
            if (same) {
                FC_TRY(adjoint(T1, cp.i0, cp.ni, cp.j0, cp.nj, true));
                FC_TRY(dens_fx_block(dx, T1, cp.i0 * tp, cp.ni, cp.nj, st, &nl));
            } else {
                FC_TRY(adjoint(T1, cp.i0, cp.ni, cp.j0, cp.nj, false));
                FC_CUDA(cudaMemcpyAsync(dstore + store_off[(size_t)((cp.i0 / cc) * nch + cp.j0 / cc)], T1,
                                        (size_t)(cp.ni * tp) * (size_t)(cp.nj * tp) * 4, cudaMemcpyDeviceToDevice,
                                        st));
                FC_TRY(adjoint(T2, cp.j0, cp.nj, cp.i0, cp.ni, true));
                FC_TRY(dens_fx_block(dx, T2, cp.j0 * tp, cp.nj, cp.ni, st, &nl));
            }
            if (step.last) FC_TRY(dens_fx_slab(dx, cp.ni, st, flags + 1, &nl));
        } else {
        if (step.blk != 1) FC_TRY(adjoint(T1, cp.i0, cp.ni, cp.j0, cp.nj, dens));
        if (step.blk != 0 && !same) {
            if (a.no_t2)
                FC_TRY(adjoint(T1, cp.j0, cp.nj, cp.i0, cp.ni, false, true));
            else
                FC_TRY(adjoint(T2, cp.j0, cp.nj, cp.i0, cp.ni, dens));
        }
        if (dens) {
            // the block (I, K) of the column chunk K: t and its slices, and
            // the slab's density terms once the column is complete
            const bool t2 = step.blk == 1;
            const int64_t r0 = t2 ? cp.j0 : cp.i0, nr = t2 ? cp.nj : cp.ni, nk = t2 ? cp.ni : cp.nj;
            FC_TRY(dens_fx_block(dx, t2 ? T2 : T1, r0 * tp, nr, nk, st, &nl));
            if (step.last) FC_TRY(dens_fx_slab(dx, nk, st, flags + 1, &nl));
        }
        }
        // row I of the chunk pairs is done: Gamma's columns of chunk I are final
        if (!dens && sink && cp.j0 + cp.nj == nocc)
            FC_TRY(gamma_sink_block(sink, gamma, naux, nov, nvir, cp.i0, cp.ni, st));
    }
    if (dens) {
        FC_TRY(dens_fx_finish(dx, *dens, st, &nl));
        if (sink) FC_TRY(gamma_sink_block(sink, gamma, naux, nov, nvir, 0, nocc, st));
    }
    scale_copy_kernel<<<(unsigned)((nocc + 255) / 256), 256, 0, st>>>(acc_occ, nocc, -2.0, de_docc);
    ++nl;
    FC_TRY(check_launch("scale_copy_kernel"));
    if (stats) FC_CUDA(cudaEventRecord(c.ev1, st));
    std::vector<double> h((size_t)(2 * ncp));
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(h.data(), e_cp, h.size() * 8, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "mixed RI-MP2: B_ov has a non-finite element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "mixed gradient kernels: a pipeline wait ran out");
    double eo = 0.0, co = 0.0, es = 0.0, cs2 = 0.0;  // Neumaier sums over the chunk pairs
    for (int64_t x = 0; x < ncp; ++x) {
        double v = h[2 * x], t = eo + v;
        co += fabs(eo) >= fabs(v) ? (eo - t) + v : (v - t) + eo;
        eo = t;
        v = h[2 * x + 1];
        t = es + v;
        cs2 += fabs(es) >= fabs(v) ? (es - t) + v : (v - t) + es;
        es = t;
    }
    *e_os = eo + co;
    *e_ss = es + cs2;
    if (stats) {
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        const double P = (double)nocc * (nocc + 1) / 2.0;
        stats->flops = 2.0 * naux * (double)nvir * nvir * P + 2.0 * naux * (double)nov * nov;
        stats->precision = FC_PREC_MIXED;
        stats->launches += (int)nl;
        stats->tile_m = fx::BM;
        stats->tile_n = fx::BN;
        stats->main_launches = (int)npair_launch;
        double tsum = 0.0;
        for (int64_t x = 0; x < nsteps; ++x) {
            float t = 0.f;
            FC_CUDA(cudaEventElapsedTime(&t, ev[2 * x], ev[2 * x + 1]));
            tsum += t;
        }
        stats->main_ms = tsum;
        // G_ij over unordered pairs (with densities: over the pairs launched,
        // off-diagonal chunk pairs twice)
        stats->main_flops = dens ? pair_flops : 2.0 * naux * (double)nvir * nvir * P;
        stats->main_bytes = 8.0 * naux * (double)nov * (double)nch * (dens ? (double)nsteps / ncp : 1.0);
        stats->aux_launches = nadj;
        FC_TRY(timing_sum2(nadj, &stats->aux_ms));
        stats->aux_flops = adj_flops;
        stats->aux_bytes = adj_bytes;
        stats->h2d_bytes += pairs.size() * sizeof(int2);
        stats->d2h_bytes += h.size() * 8 + sizeof(hf);
    }
    return FC_OK;
}

// ------------------------------------------------- unrestricted RI-MP2 --
//
// Opposite-spin energy E_ab = sum_{i a J B} (ia|JB)^2 / D on the exact-slice
// tensor-core GEMM: G = B_alpha^T B_beta over rows (i, a) and (J, B) with no
// padding per occupied orbital (no exchange partner is needed, so tiles need
// not hold whole (i, J) blocks); the epilogue forms g^2 / D and leaves one
// partial per warp and tile, summed in fixed order.

namespace {

struct EpiOS {
    const double* sa;  // [nov_a] row scales (rows (i, a))
    const double* sb;  // [nov_b] row scales (rows (J, B))
    const double* eoa;
    const double* eva;
    const double* eob;
    const double* evb;
    int nva, nvb;
    int64_t rows_a, rows_b;
    double* part;  // [tile][16] per epilogue warp
    __device__ void operator()(int64_t t, int4 it, int row, int col0, const double (&acc)[32]) const {
        const int64_t p = (int64_t)it.x * 128 + row;
        double s = 0.0;
        if (p < rows_a) {
            const int i = (int)(p / nva), a = (int)(p % nva);
            const double da = eoa[i] - eva[a];
            const double sp = sa[p];
            const int64_t w0 = (int64_t)it.y * 128 + col0;
            int J = (int)(w0 / nvb), B = (int)(w0 % nvb);
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const int64_t w = w0 + c;
                if (w < rows_b) {
                    const double g = sp * sb[w] * acc[c];
                    s += g * g / (da + eob[J] - evb[B]);
                }
                if (++B == nvb) {
                    B = 0;
                    ++J;
                }
            }
        }
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) part[t * 16 + ((threadIdx.x >> 5) - 2)] = s;
    }
};

// B_ov of one spin -> exact slices, rows (i, a) unpadded, K = q_pad.
fc_status ump2_split(const UmpSpin& x, int64_t naux, int64_t q_pad, cudaStream_t st, int* bad, int slot_split,
                     int slot_scale, __nv_bfloat16** bt, double** scl) {
    // consumed by the bf16 exact-slice xgemm (FP32 accumulation, panel drains)
    const int64_t nov = x.nocc * x.nvir;
    void *vbt, *vsc;
    FC_TRY(ws_get(slot_split, (size_t)3 * nov * q_pad * 2, &vbt));
    FC_TRY(ws_get(slot_scale, (size_t)nov * 16 + 256, &vsc));
    unsigned long long* cmax = (unsigned long long*)vsc;
    double* s = (double*)vsc + nov;
    FC_CUDA(cudaMemsetAsync(cmax, 0, nov * 8, st));
    dim3 g1((unsigned)((nov + 255) / 256), (unsigned)((naux + 63) / 64));
    colmax_kernel<<<g1, 256, 0, st>>>(x.b_ov, naux, nov, 64, cmax, bad);
    row_scale_kernel<SliceBf16><<<(unsigned)((nov + 255) / 256), 256, 0, st>>>(cmax, x.nocc, x.nvir, x.nvir, s);
    dim3 g3((unsigned)((nov + 63) / 64), (unsigned)((naux + 63) / 64));
    if (g3.y > 65535) return fail(FC_ERR_LAYOUT, "U-RI-MP2 split: naux too large");
    split_fx_transpose_kernel<SliceBf16><<<g3, 256, 0, st>>>(x.b_ov, naux, x.nocc, x.nvir, x.nvir, q_pad, s,
                                                             (__nv_bfloat16*)vbt);
    *bt = (__nv_bfloat16*)vbt;
    *scl = s;
    return check_launch("U-RI-MP2 split kernels");
}

bool g_os_attr = false;

}  // namespace

fc_status ump2_cross_fx(const UmpSpin& A, const UmpSpin& Bs, int64_t naux, cudaStream_t st, double* e_ab,
                        fc_stats* stats) {
    if (!g_os_attr) {
        FC_CUDA(cudaFuncSetAttribute(xgemm_kernel<128, EpiOS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     xg::Cfg<128>::SMEM));
        g_os_attr = true;
    }
    Context& c = ctx();
    const int64_t nova = A.nocc * A.nvir, novb = Bs.nocc * Bs.nvir;
    const int64_t q_pad = (naux + fx::KT_BF16 - 1) / fx::KT_BF16 * fx::KT_BF16;
    if (3 * nova > (int64_t)UINT32_MAX || 3 * novb > (int64_t)UINT32_MAX || nova > INT32_MAX)
        return fail(FC_ERR_LAYOUT, "U-RI-MP2: too many operand rows");
    void* vout;
    FC_TRY(ws_get(WS_OUT, 256, &vout));
    int* flags = (int*)vout;
    double* res = (double*)vout + 4;
    FC_CUDA(cudaMemsetAsync(vout, 0, 256, st));
    __nv_bfloat16 *bta, *btb;
    double *sa, *sb;
    FC_TRY(ump2_split(A, naux, q_pad, st, flags, WS_SPLIT, WS_SCALE, &bta, &sa));
    FC_TRY(ump2_split(Bs, naux, q_pad, st, flags, WS_SPLIT2, WS_MISC, &btb, &sb));
    std::vector<int4> items;
    const int ntm = (int)((nova + 127) / 128), ntn = (int)((novb + 127) / 128), nks = (int)(q_pad / fx::KT_BF16);
    for (int tn = 0; tn < ntn; ++tn)
        for (int tm = 0; tm < ntm; ++tm) items.push_back(make_int4(tm, tn, 0, nks));
    void *vtab, *vpart;
    FC_TRY(ws_get(WS_PAIRS, items.size() * sizeof(int4), &vtab));
    FC_TRY(ws_get(WS_PART, items.size() * 16 * 8, &vpart));
    FC_CUDA(cudaMemcpyAsync(vtab, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    CUtensorMap ta, tb;
    FC_TRY(make_tmap_bf16_2d(&ta, bta, q_pad, 3 * nova, q_pad * 2, fx::KT_BF16, 128));
    FC_TRY(make_tmap_bf16_2d(&tb, btb, q_pad, 3 * novb, q_pad * 2, fx::KT_BF16, 128));
    XArgs a{(const int4*)vtab, (int64_t)items.size(), (int)nova, (int)novb, flags + 1};
    EpiOS epi{sa, sb, A.eps_occ, A.eps_vir, Bs.eps_occ, Bs.eps_vir, (int)A.nvir, (int)Bs.nvir, nova, novb,
              (double*)vpart};
    cudaEvent_t* ev = nullptr;
    if (stats) {
        FC_TRY(timing_events(1, &ev));
        FC_CUDA(cudaEventRecord(ev[0], st));
    }
    const int grid = (int)std::min<int64_t>((int64_t)items.size(), c.sm_count);
    xgemm_kernel<128, EpiOS><<<grid, xg::Cfg<128>::THREADS, xg::Cfg<128>::SMEM, st>>>(ta, tb, a, epi);
    FC_TRY(check_launch("opposite-spin exact-slice GEMM"));
    if (stats) FC_CUDA(cudaEventRecord(ev[1], st));
    // the partials as (even, odd) pairs: out = (sum of even, sum of odd)
    fx_reduce_pairs_kernel<<<1, 1024, 0, st>>>((const double*)vpart, (int64_t)items.size() * 8, res);
    FC_TRY(check_launch("fx_reduce_pairs_kernel"));
    double h[2];
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "mixed RI-MP2: B_ov has a non-finite element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "opposite-spin GEMM: a pipeline wait ran out");
    *e_ab = h[0] + h[1];
    if (stats) {
        double ms = 0.0;
        FC_TRY(timing_sum(1, &ms));
        stats->main_ms += ms;
        stats->main_launches += 1;
        stats->main_flops += 2.0 * (double)naux * (double)nova * (double)novb;
        stats->launches += 8;
    }
    return FC_OK;
}

// ---------------------------------------------------------------- batch --
//
// Layout of a batch.  Pair operands: all molecules' integer slices in one
// buffer with a common row pitch (the largest padded aux range); molecule m
// owns rows row0_m .. row0_m + 3 nocc_m a_pad_m, slice-major.  Items
// (molecule, i, j, ta | tb << 16) are laid out molecule by molecule, i-major,
// so a molecule's partials (and one i's) are contiguous; the persistent pair
// kernel takes them round-robin, so every CTA mixes large and small
// molecules.  Gradient: amplitudes of a molecule are stored at virtual pitch
// tpad = nvir rounded up to 8 (not the 128-row tile pitch), and the adjoint
// contraction reads them and the Q-row slices through per-molecule tensor
// maps whose inner extent is the exact K = nocc tpad (the TMA zero-fills the
// K tail).  Molecules are grouped so one group's amplitudes fit group_bytes;
// groups run one after the other on the same workspace.
namespace {
int64_t rup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
}  // namespace

fc_status rimp2_batch_build_fx(fc_rimp2_batch* b, const std::vector<BatchMolIn>& mols, size_t group_bytes,
                               const int* plan) {
    FC_TRY(fx_attrs());
    const int nmol = (int)mols.size();
    const bool grad = b->grad != 0;
    Context& c = ctx();
    int64_t q_pad = fx::PKT;
    for (const auto& d : mols) q_pad = std::max(q_pad, rup(d.naux, fx::PKT));
    const int NP = nmol + 1;
    std::vector<BatchPrep> hp(nmol);
    std::vector<BatchMol> hm(nmol);
    std::vector<int64_t> pre((size_t)PRE_COUNT * NP, 0), seg(NP, 0);
    auto P = [&](int kind, int m) -> int64_t& { return pre[(size_t)kind * NP + m]; };
    std::vector<int64_t> scl_off(nmol), cmax_off(nmol), qs_off(nmol), bq_off(nmol), t_off(nmol), ntp(nmol);
    int64_t rows = 0, nscl = 0, ncmax = 0, nqs = 0, nbq = 0;
    for (int m = 0; m < nmol; ++m) {
        const auto& d = mols[m];
        BatchPrep& x = hp[m];
        const int64_t nov = d.nocc * d.nvir;
        x.b = d.b_ov;
        x.naux = d.naux;
        x.nocc = d.nocc;
        x.nvir = d.nvir;
        x.a_pad = rup(d.nvir, fx::BM);
        x.q_pad = q_pad;
        x.tpad = grad ? rup(d.nvir, 16) : x.a_pad;
        x.ldt = d.nocc * x.tpad;          // a multiple of 16 (16-byte int8 slice rows)
        x.q_rows = rup(d.naux, 128);
        x.M = rup(x.ldt, 128);
        x.de_docc = d.de_deps_occ;
        x.de_dvir = d.de_deps_vir;
        const int64_t nT = x.a_pad / fx::BM;
        ntp[m] = nT * (nT + 1) / 2;
        const int64_t npair = d.nocc * (d.nocc + 1) / 2;  // unordered pairs in both modes
        x.ntp = ntp[m];
        x.seg0 = seg[m];
        seg[m + 1] = seg[m] + npair * ntp[m];
        scl_off[m] = nscl;
        nscl += d.nocc * x.a_pad;
        cmax_off[m] = ncmax;
        ncmax += nov;
        hm[m].row0 = (int)rows;
        rows += fx::PSL * d.nocc * x.a_pad;
        qs_off[m] = nqs;
        nqs += x.q_rows;
        bq_off[m] = nbq;
        nbq += 3 * x.q_rows * x.ldt;
        P(PRE_COLMAX, m + 1) = P(PRE_COLMAX, m) + (nov + 255) / 256 * ((d.naux + 63) / 64);
        P(PRE_ROWSCALE, m + 1) = P(PRE_ROWSCALE, m) + d.nocc * x.a_pad;
        P(PRE_TRANSPOSE, m + 1) = P(PRE_TRANSPOSE, m) + (nov + 63) / 64 * ((d.naux + 63) / 64);
        P(PRE_QROWS, m + 1) = P(PRE_QROWS, m) + d.naux;
        P(PRE_TROWS, m + 1) = P(PRE_TROWS, m) + x.ldt;
        P(PRE_OCC, m + 1) = P(PRE_OCC, m) + d.nocc;
        P(PRE_VIR, m + 1) = P(PRE_VIR, m) + d.nvir;
        P(PRE_COLSQ, m + 1) = P(PRE_COLSQ, m) + nov;
        const double P2 = (double)d.nocc * (d.nocc + 1) / 2.0;
        b->flops += 2.0 * (double)d.naux * (double)d.nvir * (double)d.nvir * P2;
        if (grad) b->flops += 2.0 * (double)d.naux * (double)nov * (double)nov;
    }
    const int64_t items = seg[nmol];
    for (const auto& x : hp)
        if (x.naux > PAIR_KMAX || (grad && x.ldt > fx::KMAX))
            return fail(FC_ERR_LAYOUT, "RI-MP2 batch: a molecule exceeds the exact int32 level-sum range");
    if (rows >= INT32_MAX || items >= INT32_MAX || P(PRE_COLMAX, nmol) >= INT32_MAX ||
        P(PRE_TRANSPOSE, nmol) >= INT32_MAX || P(PRE_ROWSCALE, nmol) >= (int64_t)INT32_MAX * 256 ||
        P(PRE_QROWS, nmol) >= INT32_MAX || P(PRE_TROWS, nmol) >= INT32_MAX)
        return fail(FC_ERR_LAYOUT, "RI-MP2 batch too large for one graph");

    // ---- groups of molecules whose amplitudes share one workspace
    struct Group {
        int m0, m1;
        int64_t i0, i1, t0, t1;
    };
    std::vector<Group> groups;
    size_t gws = 0, gvir = 0;
    if (grad) {
        size_t cur = 0;
        int m0 = 0;
        for (int m = 0; m < nmol; ++m) {
            const BatchPrep& x = hp[m];
            const size_t tb = rup(x.ldt * x.ldt * 4, 256) + rup(x.M * 8, 256) + rup(3 * x.M * x.ldt, 256);
            if (m > m0 && cur + tb > group_bytes) {
                groups.push_back({m0, m, seg[m0], seg[m], 0, 0});
                m0 = m;
                cur = 0;
            }
            t_off[m] = (int64_t)cur;
            cur += tb;
            gws = std::max(gws, cur);
        }
        groups.push_back({m0, nmol, seg[m0], seg[nmol], 0, 0});
        for (const auto& g : groups) gvir = std::max(gvir, (size_t)(g.i1 - g.i0) * 2 * fx::BM * 8);
    }

    // ---- device buffers
    void *vbt, *vscl, *vgd, *vcmax, *vmols, *vprep, *vpre, *vseg, *vitems, *vpart, *vscr;
    FC_TRY(batch_alloc(b, (size_t)rows * q_pad, &vbt));
    FC_TRY(batch_alloc(b, (size_t)nscl * 8, &vscl));
    FC_TRY(batch_alloc(b, (size_t)nscl * 8, &vgd));
    FC_TRY(batch_alloc(b, (size_t)ncmax * 8, &vcmax));
    FC_TRY(batch_alloc(b, (size_t)nmol * sizeof(BatchMol), &vmols));
    FC_TRY(batch_alloc(b, (size_t)nmol * sizeof(BatchPrep), &vprep));
    FC_TRY(batch_alloc(b, pre.size() * 8, &vpre));
    FC_TRY(batch_alloc(b, seg.size() * 8, &vseg));
    FC_TRY(batch_alloc(b, (size_t)items * sizeof(int4), &vitems));
    FC_TRY(batch_alloc(b, (size_t)items * 16, &vpart));
    const int pgrid = (int)std::min<int64_t>(std::max<int64_t>(items, 1), c.sm_count);
    FC_TRY(batch_alloc(b, (size_t)pgrid * 3 * fx::BM * fx::BN * sizeof(double), &vscr));
    FC_CUDA(cudaMemset(vbt, 0, (size_t)rows * q_pad));
    void *vocc = nullptr, *vvir = nullptr, *vqs = nullptr, *vbq = nullptr, *vgws = nullptr;
    void *vgm = nullptr, *vmaps = nullptr, *vgit = nullptr;
    std::vector<int4> git;
    if (grad) {
        FC_TRY(batch_alloc(b, (size_t)items * 8, &vocc));
        FC_TRY(batch_alloc(b, gvir, &vvir));
        FC_TRY(batch_alloc(b, (size_t)nqs * 8, &vqs));
        FC_TRY(batch_alloc(b, (size_t)nbq, &vbq));
        FC_TRY(batch_alloc(b, gws, &vgws));
        FC_TRY(batch_alloc(b, (size_t)nmol * sizeof(GemmMol), &vgm));
        FC_TRY(batch_alloc(b, (size_t)nmol * 2 * sizeof(CUtensorMap), &vmaps));
        FC_CUDA(cudaMemset(vbq, 0, (size_t)nbq));
    }
    // per-molecule pointers
    std::vector<CUtensorMap> maps(grad ? 2 * nmol : 0);
    std::vector<GemmMol> gm(grad ? nmol : 0);
    for (int m = 0; m < nmol; ++m) {
        BatchPrep& x = hp[m];
        x.cmax = (unsigned long long*)vcmax + cmax_off[m];
        x.scl = (double*)vscl + scl_off[m];
        x.gd = (double*)vgd + scl_off[m];
        x.bt = (int8_t*)vbt + (int64_t)hm[m].row0 * q_pad;
        hm[m].eo = mols[m].eps_occ;
        hm[m].ev = mols[m].eps_vir;
        hm[m].scl = x.scl;
        hm[m].gd = x.gd;
        hm[m].nocc = (int)x.nocc;
        hm[m].nvir = (int)x.nvir;
        hm[m].a_pad = (int)x.a_pad;
        hm[m].nk = (int)(rup(x.naux, fx::PKT) / fx::PKT);
        hm[m].tpad = (int)x.tpad;
        hm[m].xt = plan ? plan[m] : fx_exchange_choice(hm[m].nk, grad);
        hm[m].T = nullptr;
        hm[m].ldt = x.ldt;
        if (grad) {
            char* g0 = (char*)vgws + t_off[m];
            x.T = (float*)g0;
            x.ts = (double*)(g0 + rup(x.ldt * x.ldt * 4, 256));
            x.Ts = (int8_t*)(g0 + rup(x.ldt * x.ldt * 4, 256) + rup(x.M * 8, 256));
            x.qs = (double*)vqs + qs_off[m];
            x.bq = (int8_t*)vbq + bq_off[m];
            hm[m].T = x.T;
            FC_TRY(make_tmap_i8_2d(&maps[2 * m], x.Ts, x.ldt, 3 * x.M, x.ldt, fx::KT, 128));
            FC_TRY(make_tmap_i8_2d(&maps[2 * m + 1], x.bq, x.ldt, 3 * x.q_rows, x.ldt, fx::KT, 128));
            GemmMol& g = gm[m];
            g.tA = (const CUtensorMap*)vmaps + 2 * m;
            g.tB = (const CUtensorMap*)vmaps + 2 * m + 1;
            g.rs = x.ts;
            g.cs = x.qs;
            g.M = (int)x.M;
            g.N = (int)x.q_rows;
            g.nk = (int)((x.ldt + fx::KT - 1) / fx::KT);
            g.tpad = (int)x.tpad;
            g.nvir = (int)x.nvir;
            g.naux = (int)x.naux;
            g.rows = (int)x.ldt;
            g.nov = x.nocc * x.nvir;
            g.out = mols[m].gamma;
        }
    }
    // work items
    std::vector<int4> hi;
    hi.reserve((size_t)items);
    for (int m = 0; m < nmol; ++m) {
        const int nocc = hm[m].nocc, nT = hm[m].a_pad / fx::BM;
        for (int i = 0; i < nocc; ++i)
            for (int j = i; j < nocc; ++j)
                for (int ta = 0; ta < nT; ++ta)
                    for (int tb = ta; tb < nT; ++tb) hi.push_back(make_int4(m, i, j, ta | (tb << 16)));
    }
    if (grad) {
        for (auto& g : groups) {
            g.t0 = (int64_t)git.size();
            for (int m = g.m0; m < g.m1; ++m) {
                const int ntm = (int)(hp[m].M / 128), ntn = (int)(hp[m].q_rows / 128);
                for (int tm = 0; tm < ntm; ++tm)
                    for (int tn = 0; tn < ntn; ++tn) git.push_back(make_int4(m, tm, tn, 0));
            }
            g.t1 = (int64_t)git.size();
        }
        FC_TRY(batch_alloc(b, git.size() * sizeof(int4), &vgit));
        FC_CUDA(cudaMemcpy(vgit, git.data(), git.size() * sizeof(int4), cudaMemcpyHostToDevice));
        FC_CUDA(cudaMemcpy(vgm, gm.data(), gm.size() * sizeof(GemmMol), cudaMemcpyHostToDevice));
        FC_CUDA(cudaMemcpy(vmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    }
    FC_CUDA(cudaMemcpy(vmols, hm.data(), hm.size() * sizeof(BatchMol), cudaMemcpyHostToDevice));
    FC_CUDA(cudaMemcpy(vprep, hp.data(), hp.size() * sizeof(BatchPrep), cudaMemcpyHostToDevice));
    FC_CUDA(cudaMemcpy(vpre, pre.data(), pre.size() * 8, cudaMemcpyHostToDevice));
    FC_CUDA(cudaMemcpy(vseg, seg.data(), seg.size() * 8, cudaMemcpyHostToDevice));
    FC_CUDA(cudaMemcpy(vitems, hi.data(), hi.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CUtensorMap tmA, tmB;
    FC_TRY(make_tmap_i8_2d_sw64(&tmA, vbt, q_pad, rows, q_pad, fx::BM));
    FC_TRY(make_tmap_i8_2d_sw64(&tmB, vbt, q_pad, rows, q_pad, fx::BN));
    FC_CUDA(cudaDeviceSynchronize());

    // ---- the recorded sequence
    cudaStream_t st = b->stream;
    const BatchPrep* dp = (const BatchPrep*)vprep;
    const int64_t* dpre = (const int64_t*)vpre;
    auto PD = [&](int kind) { return dpre + (size_t)kind * NP; };
    FC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    fc_status rc = [&]() -> fc_status {
        int launches = 0;
        FC_CUDA(cudaMemsetAsync(b->flags, 0, 2 * sizeof(int), st));
        FC_CUDA(cudaMemsetAsync(vcmax, 0, (size_t)ncmax * 8, st));
        batch_colmax_kernel<<<(unsigned)P(PRE_COLMAX, nmol), 256, 0, st>>>(dp, PD(PRE_COLMAX), nmol, b->flags);
        batch_row_scale_kernel<<<(unsigned)((P(PRE_ROWSCALE, nmol) + 255) / 256), 256, 0, st>>>(
            dp, PD(PRE_ROWSCALE), nmol);
        batch_transpose_kernel<<<(unsigned)P(PRE_TRANSPOSE, nmol), 256, 0, st>>>(dp, PD(PRE_TRANSPOSE), nmol);
        batch_colsq_kernel<<<(unsigned)((P(PRE_COLSQ, nmol) + 255) / 256), 256, 0, st>>>(dp, PD(PRE_COLSQ), nmol);
        launches += 4;
        if (grad) {
            batch_qrows_kernel<<<(unsigned)P(PRE_QROWS, nmol), 256, 0, st>>>(dp, PD(PRE_QROWS), nmol);
            ++launches;
        }
        FC_TRY(check_launch("batch split kernels"));
        PairFxArgs a{};
        a.wait_ns = tc::WAIT_LIMIT_NS;
        a.bitems = (const int4*)vitems;
        a.bmols = (const BatchMol*)vmols;
        a.err = b->flags + 1;
        a.scr = (double*)vscr;
        if (!grad) {
            a.items = items;
            a.part = (double*)vpart;
            const int grid = (int)std::min<int64_t>(items, c.sm_count);
            pair_fx_kernel<0, 1><<<grid, fx::PAIR_THREADS, fx::SMEM, st>>>(tmA, tmB, a);
            batch_energy_kernel<<<(unsigned)nmol, 256, 0, st>>>((const double*)vpart, (const int64_t*)vseg, 0,
                                                                  b->out);
            FC_TRY(check_launch("batched pair kernel"));
            launches += 2;
            b->pair_launches = 1;
        } else {
            for (const auto& g : groups) {
                const int64_t gi = g.i1 - g.i0;
                a.bitems = (const int4*)vitems + g.i0;
                a.items = gi;
                a.part = (double*)vpart + 2 * g.i0;
                a.occ_part = (double*)vocc + g.i0;
                a.vir_part = (double*)vvir;
                const int grid = (int)std::min<int64_t>(gi, c.sm_count);
                pair_fx_kernel<1, 1><<<grid, fx::PAIR_THREADS, fx::SMEM, st>>>(tmA, tmB, a);
                batch_energy_kernel<<<(unsigned)(g.m1 - g.m0), 256, 0, st>>>((const double*)vpart,
                                                                               (const int64_t*)vseg, g.m0, b->out);
                batch_occ_kernel<<<(unsigned)(P(PRE_OCC, g.m1) - P(PRE_OCC, g.m0)), 256, 0, st>>>(
                    dp, PD(PRE_OCC), g.m0, g.m1, (const double*)vocc);
                batch_vir_kernel<<<(unsigned)((P(PRE_VIR, g.m1) - P(PRE_VIR, g.m0) + 7) / 8), 256, 0, st>>>(
                    dp, PD(PRE_VIR), g.m0, g.m1, (const int4*)vitems, g.i0, (const double*)vvir);
                batch_trows_kernel<<<(unsigned)(P(PRE_TROWS, g.m1) - P(PRE_TROWS, g.m0)), 256, 0, st>>>(
                    dp, PD(PRE_TROWS), g.m0, g.m1);
                FC_TRY(check_launch("batched gradient reductions / split"));
                GemmFxArgs ga{};
                ga.bitems = (const int4*)vgit + g.t0;
                ga.gmols = (const GemmMol*)vgm;
                ga.tiles = g.t1 - g.t0;
                ga.alpha = 4.0;
                ga.err = b->flags + 1;
                const int g2 = (int)std::min<int64_t>(ga.tiles, c.sm_count);
                gemm_fx_kernel<1><<<g2, GF_THREADS, GF_SMEM, st>>>(tmA, tmB, ga);
                FC_TRY(check_launch("batched adjoint contraction"));
                launches += 6;
            }
            b->pair_launches = (int)groups.size();
        }
        b->launches = launches;
        return FC_OK;
    }();
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(st, &graph);
    if (rc != FC_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture");
    b->graph = graph;
    FC_CUDA(cudaGraphInstantiate(&b->exec, graph, 0));
    b->items = items;
    b->gemm_tiles = (int64_t)git.size();
    b->groups = grad ? (int)groups.size() : 0;
    return FC_OK;
}

}  // namespace fc

// ------------------------------------------------------------ self-check --

namespace fc {
namespace {
__global__ void recip_check_kernel(const double* __restrict__ d, int64_t n, double* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = fx::recip_nr(d[k]);
}
}  // namespace
}  // namespace fc

extern "C" fc_status fc_check_recip(const double* d, int64_t n, double* out) {
    using namespace fc;
    if (n < 0 || (n > 0 && (!d || !out))) return fail(FC_ERR_INVALID, "fc_check_recip: bad arguments");
    if (n == 0) return FC_OK;
    FC_TRY(require_init());
    double* dd = nullptr;
    FC_CUDA(cudaMalloc(&dd, 2 * (size_t)n * sizeof(double)));
    fc_status st = FC_OK;
    cudaError_t e = cudaMemcpy(dd, d, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        recip_check_kernel<<<(unsigned)((n + 255) / 256), 256>>>(dd, n, dd + n);
        st = check_launch("recip_check_kernel");
        if (st == FC_OK) e = cudaMemcpy(out, dd + n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    }
    cudaFree(dd);
    if (st != FC_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "fc_check_recip copy");
    return FC_OK;
}
