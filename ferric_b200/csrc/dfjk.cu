// DF-J and DF-K builders behind a device-resident handle.
//
// DF-J (ferric-scf/src/df_j.rs:1199-1245, 1459-1572) is two GEMV passes over
// the packed lower triangle of B, HBM-bound:
//   pass 1  d_P = sum_k Bp[P, k] w_k      (CTAs over row segments, fixed-order sums)
//   solve   c = V^-1 d                     (FP64 Cholesky solves, when a metric is set)
//   pass 2  J_k = sum_P Bp[P, k] c_P       (column-parallel over k, split over P,
//                                           fixed-order fold of the splits)
// DF-K occupied path (ferric-scf/src/df_k.rs:1409-1520, 1575-1660):
//   stage 1 M_Q = B_Q C_occ on the DMMA tile GEMM, written as W[mu, (Q, i)]
//   stage 2 K = W W^T, upper tiles only, split over (Q, i), fixed-order fold
//           that also symmetrises (the final J/K symmetrisation in FP64).
#include "fc_internal.cuh"
#include "dgemm_tn.cuh"
#include "dfjk.cuh"

#include <vector>

using namespace fc;

namespace fc {

// ------------------------------------------------------------- layout --

__global__ void pack_lower_kernel(const double* __restrict__ sq, int64_t n, int64_t pair,
                                  double* __restrict__ pk) {
    const int64_t mu = blockIdx.x, q = blockIdx.y;
    const double* src = sq + (q * n + mu) * n;
    double* dst = pk + q * pair + mu * (mu + 1) / 2;
    for (int64_t nu = threadIdx.x; nu <= mu; nu += blockDim.x) dst[nu] = src[nu];
}

// Packed density weights (ferric-scf/src/df_j.rs:1134-1150).
__global__ void density_weights_kernel(const double* __restrict__ d, int64_t n,
                                       double* __restrict__ w) {
    const int64_t mu = blockIdx.x;
    double* dst = w + mu * (mu + 1) / 2;
    for (int64_t nu = threadIdx.x; nu <= mu; nu += blockDim.x)
        dst[nu] = nu == mu ? d[mu * n + mu] : d[mu * n + nu] + d[nu * n + mu];
}

// ---------------------------------------------------------- DF-J passes --

// Pass 1 reads each aux row in segments of DFJ_SEG_BYTES, one CTA per
// (row, segment): a row per CTA left a near-empty last wave (2400 rows are
// 2.03 waves of 148 x 8 CTAs) that ran latency-bound.  Segment partials land
// in part[row * nseg + seg] and dfj_seg_sum_kernel adds them in fixed order.
constexpr int64_t DFJ_SEG_BYTES = 65536;

template <typename TB>
__global__ void __launch_bounds__(256) dfj_pass1_kernel(const TB* __restrict__ bp, int64_t pair, int64_t seg,
                                                        const double* __restrict__ w,
                                                        double* __restrict__ part) {
    __shared__ double red[32];
    const TB* row = bp + (int64_t)blockIdx.x * pair;
    const int64_t k0 = (int64_t)blockIdx.y * seg;
    const int64_t k1 = k0 + seg < pair ? k0 + seg : pair;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int64_t k = k0 + threadIdx.x;
    for (; k + 768 < k1; k += 1024) {
        s0 += (double)row[k] * w[k];
        s1 += (double)row[k + 256] * w[k + 256];
        s2 += (double)row[k + 512] * w[k + 512];
        s3 += (double)row[k + 768] * w[k + 768];
    }
    for (; k < k1; k += 256) s0 += (double)row[k] * w[k];
    const double v = block_sum((s0 + s1) + (s2 + s3), red);
    if (threadIdx.x == 0) part[(int64_t)blockIdx.x * gridDim.y + blockIdx.y] = v;
}

__global__ void dfj_seg_sum_kernel(const double* __restrict__ part, int nseg, int64_t naux,
                                   double* __restrict__ dp) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= naux) return;
    double s = 0.0;
    for (int g = 0; g < nseg; ++g) s += part[q * nseg + g];
    dp[q] = s;
}

template <typename TB>
__global__ void __launch_bounds__(256) dfj_pass2_kernel(const TB* __restrict__ bp, int64_t naux,
                                                        int64_t pair, const double* __restrict__ c,
                                                        int64_t rows_per_split,
                                                        double* __restrict__ part) {
    const int64_t k = (int64_t)blockIdx.x * 256 + threadIdx.x;
    const int64_t p0 = (int64_t)blockIdx.y * rows_per_split;
    const int64_t p1 = p0 + rows_per_split < naux ? p0 + rows_per_split : naux;
    if (k >= pair) return;
    double s0 = 0.0, s1 = 0.0;
    int64_t p = p0;
    for (; p + 1 < p1; p += 2) {
        s0 += (double)bp[p * pair + k] * c[p];
        s1 += (double)bp[(p + 1) * pair + k] * c[p + 1];
    }
    if (p < p1) s0 += (double)bp[p * pair + k] * c[p];
    part[(int64_t)blockIdx.y * pair + k] = s0 + s1;
}

// Exact FP32 -> FP64 widening.  The hardware conversion issues at a few per
// clock per SM, which alone held the FP32 passes to ~3.6 TB/s; widen_f32 does
// the same on the integer pipe, and the passes convert DFJ_HW_WIDEN of each
// float4's four elements in hardware and the rest here, so the two pipes
// share the load (measured best at 2 of 4).  widen_f32 is the IEEE 754 field
// mapping for normal numbers: an arithmetic shift by 3 moves sign, 8-bit
// exponent and the top 20 fraction bits into the high word (the sign lands
// in bits 31..28; the mask keeps bit 31), adding 896 << 20 rebiases the
// exponent (1023 - 127), and the low 3 fraction bits go to the top of the low
// word.  +-0 widen to +0 (a product's zero sign is all that differs).
// SUB = true also widens subnormals, through the hardware conversion; the
// FP32 copy records whether it holds any, so the usual tensor takes the
// branch-free form.  No Inf/NaN reaches here: the FP32 copy is refused when a
// value overflows.
constexpr int DFJ_HW_WIDEN = 2;

template <bool SUB>
__device__ __forceinline__ double widen_f32(float f) {
    const uint32_t u = __float_as_uint(f);
    if constexpr (SUB) {
        if ((u & 0x7f800000u) == 0u) return (double)f;
    }
    const uint32_t hi = ((uint32_t)((int32_t)u >> 3) & 0x8fffffffu) + 0x38000000u;
    return __hiloint2double((u << 1) ? (int)hi : 0, (int)(u << 29));
}

template <int I, bool SUB>
__device__ __forceinline__ double widen_at(float f) {
    if constexpr (I < DFJ_HW_WIDEN) return (double)f;
    else return widen_f32<SUB>(f);
}

template <bool SUB>
__device__ __forceinline__ double dot4(const float4& a, const double* w) {
    return widen_at<0, SUB>(a.x) * w[0] + widen_at<1, SUB>(a.y) * w[1] + widen_at<2, SUB>(a.z) * w[2] +
           widen_at<3, SUB>(a.w) * w[3];
}

// Pass 1 over the FP32 rows (pitch ld = pair rounded up to 4, zero padded):
// one CTA per (group of DFJ_ROWS rows, segment); each float4's FP64 weights
// (32 B of w, from L2) serve DFJ_ROWS rows, so L2 -> SM traffic is 1.25x the
// HBM stream instead of 3x it (one row per CTA), and the DFJ_ROWS loads per
// thread in flight cover HBM latency.  Rows past naux re-read the last row;
// their sums are dropped.
constexpr int DFJ_ROWS = 8;

template <bool SUB>
__global__ void __launch_bounds__(256, 3) dfj_pass1_f32v_kernel(const float* __restrict__ bp, int64_t naux,
                                                                int64_t ld, int64_t seg4,
                                                                const double* __restrict__ w,
                                                                double* __restrict__ part) {
    __shared__ double red[DFJ_ROWS][8];
    const int64_t r0 = (int64_t)blockIdx.x * DFJ_ROWS;
    const int64_t n4 = ld / 4;
    const float4* rows[DFJ_ROWS];
#pragma unroll
    for (int r = 0; r < DFJ_ROWS; ++r)
        rows[r] = reinterpret_cast<const float4*>(bp + (r0 + r < naux ? r0 + r : naux - 1) * ld);
    const int64_t k0 = (int64_t)blockIdx.y * seg4;
    const int64_t k1 = k0 + seg4 < n4 ? k0 + seg4 : n4;
    double s[DFJ_ROWS] = {};
    for (int64_t k = k0 + threadIdx.x; k < k1; k += 256) {
        float4 a[DFJ_ROWS];
#pragma unroll
        for (int r = 0; r < DFJ_ROWS; ++r) a[r] = rows[r][k];
        const double* wa = w + 4 * k;
#pragma unroll
        for (int r = 0; r < DFJ_ROWS; ++r) s[r] += dot4<SUB>(a[r], wa);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < DFJ_ROWS; ++r) {
        double v = s[r];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[r][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < DFJ_ROWS && r0 + threadIdx.x < naux) {
        double v = 0.0;
        for (int i = 0; i < 8; ++i) v += red[threadIdx.x][i];
        part[(r0 + threadIdx.x) * gridDim.y + blockIdx.y] = v;
    }
}

// Pass 2 over the FP32 rows: each thread owns four columns (one float4) and
// keeps four rows' loads in flight.
template <bool SUB>
__global__ void __launch_bounds__(256) dfj_pass2_f32v_kernel(const float* __restrict__ bp, int64_t naux, int64_t ld,
                                                             const double* __restrict__ c, int64_t rows_per_split,
                                                             double* __restrict__ part) {
    const int64_t k4 = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (k4 >= ld / 4) return;
    const int64_t p0 = (int64_t)blockIdx.y * rows_per_split;
    const int64_t p1 = p0 + rows_per_split < naux ? p0 + rows_per_split : naux;
    double s[4] = {0.0, 0.0, 0.0, 0.0}, t[4] = {0.0, 0.0, 0.0, 0.0};
    const float4* col = reinterpret_cast<const float4*>(bp) + k4;
    const int64_t l4 = ld / 4;
    int64_t p = p0;
    for (; p + 3 < p1; p += 4) {
        const float4 a = col[p * l4], b = col[(p + 1) * l4], e = col[(p + 2) * l4], f = col[(p + 3) * l4];
        const double ca = c[p], cb = c[p + 1], ce = c[p + 2], cf = c[p + 3];
        s[0] += widen_at<0, SUB>(a.x) * ca + widen_at<0, SUB>(b.x) * cb;
        s[1] += widen_at<1, SUB>(a.y) * ca + widen_at<1, SUB>(b.y) * cb;
        s[2] += widen_at<2, SUB>(a.z) * ca + widen_at<2, SUB>(b.z) * cb;
        s[3] += widen_at<3, SUB>(a.w) * ca + widen_at<3, SUB>(b.w) * cb;
        t[0] += widen_at<0, SUB>(e.x) * ce + widen_at<0, SUB>(f.x) * cf;
        t[1] += widen_at<1, SUB>(e.y) * ce + widen_at<1, SUB>(f.y) * cf;
        t[2] += widen_at<2, SUB>(e.z) * ce + widen_at<2, SUB>(f.z) * cf;
        t[3] += widen_at<3, SUB>(e.w) * ce + widen_at<3, SUB>(f.w) * cf;
    }
    for (; p < p1; ++p) {
        const float4 a = col[p * l4];
        const double ca = c[p];
        s[0] += widen_at<0, SUB>(a.x) * ca;
        s[1] += widen_at<1, SUB>(a.y) * ca;
        s[2] += widen_at<2, SUB>(a.z) * ca;
        s[3] += widen_at<3, SUB>(a.w) * ca;
    }
    double2* dst = reinterpret_cast<double2*>(part + (int64_t)blockIdx.y * ld + 4 * k4);
    dst[0] = make_double2(s[0] + t[0], s[1] + t[1]);
    dst[1] = make_double2(s[2] + t[2], s[3] + t[3]);
}

// FP64 -> FP32 (round to nearest) copy of the packed rows, row p of x (pitch
// pair) to row p of y (pitch ld); flags values outside the FP32 range (bit 0,
// the reference's F32Range check, ferric-core/src/gpu/kernels/round_f64_to_f32.cu
// semantics) and subnormal results, which are kept as the reference keeps
// them (bit 1).
__global__ void round_f32_kernel(const double* __restrict__ x, int64_t rows, int64_t pair, int64_t ld,
                                 float* __restrict__ y, int* bad) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * pair) return;
    const int64_t p = e / pair, k = e % pair;
    const double v = x[e];
    if (!(fabs(v) <= 3.4028234663852886e38)) atomicOr(bad, 1);
    const float f = __double2float_rn(v);
    if (f != 0.0f && fabsf(f) < 1.17549435e-38f) atomicOr(bad, 2);
    y[p * ld + k] = f;
}

// part: [nsplit][ld] pass-2 partials of the packed J (ld >= pair).
__global__ void dfj_unpack_kernel(const double* __restrict__ part, int nsplit, int64_t ld, int64_t n,
                                  double* __restrict__ j) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * n) return;
    const int64_t r = idx / n, c = idx % n;
    const int64_t hi = r > c ? r : c, lo = r > c ? c : r;
    const int64_t k = hi * (hi + 1) / 2 + lo;
    double s = 0.0;
    for (int sp = 0; sp < nsplit; ++sp) s += part[(int64_t)sp * ld + k];
    j[idx] = s;
}

// c = V^-1 d with V = L L^T, L lower row-major (naux x naux); in place on x.
// One CTA of 32 warps, blocked by 32 rows: left-looking forward solve, then
// the backward solve with L^T.  Fixed reduction order throughout.
__global__ void __launch_bounds__(1024) chol_solve_kernel(const double* __restrict__ L, int64_t naux,
                                                          double* __restrict__ x) {
    __shared__ double sh[32][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // forward: L y = d
    for (int64_t kb = 0; kb < naux; kb += 32) {
        const int nb = (int)(naux - kb < 32 ? naux - kb : 32);
        if (warp < nb) {
            const int64_t r = kb + warp;
            double s = 0.0;
            for (int64_t k = lane; k < kb; k += 32) s += L[r * naux + k] * x[k];
            s = warp_sum(s);
            if (lane == 0) x[r] -= s;
        }
        __syncthreads();
        if (warp == 0) {
            double yl = lane < nb ? x[kb + lane] : 0.0;
            for (int rr = 0; rr < nb; ++rr) {
                const double v = lane < rr ? L[(kb + rr) * naux + kb + lane] * yl : 0.0;
                const double s = warp_sum(v);
                if (lane == rr) yl = (yl - s) / L[(kb + rr) * naux + kb + rr];
            }
            if (lane < nb) x[kb + lane] = yl;
        }
        __syncthreads();
    }
    // backward: L^T c = y
    const int64_t nblk = (naux + 31) / 32;
    for (int64_t bi = nblk - 1; bi >= 0; --bi) {
        const int64_t kb = bi * 32;
        const int nb = (int)(naux - kb < 32 ? naux - kb : 32);
        double part = 0.0;
        if (lane < nb)
            for (int64_t k = kb + nb + warp; k < naux; k += 32) part += L[k * naux + kb + lane] * x[k];
        sh[warp][lane] = part;
        __syncthreads();
        if (warp == 0) {
            double s = 0.0;
            for (int w = 0; w < 32; ++w) s += sh[w][lane];
            double yl = lane < nb ? x[kb + lane] - s : 0.0;
            for (int rr = nb - 1; rr >= 0; --rr) {
                const double v = (lane > rr && lane < nb) ? L[(kb + lane) * naux + kb + rr] * yl : 0.0;
                const double s2 = warp_sum(v);
                if (lane == rr) yl = (yl - s2) / L[(kb + rr) * naux + kb + rr];
            }
            if (lane < nb) x[kb + lane] = yl;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- DF-K --

__global__ void transpose_kernel(const double* __restrict__ a, int64_t rows, int64_t cols,
                                 double* __restrict__ at) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= rows * cols) return;
    const int64_t r = idx / cols, c = idx % cols;
    at[c * rows + r] = a[idx];
}

// Stage-1 epilogue: row (Q, mu) of M = B C goes to W[mu, Q*nocc + i].
struct EpiScatterW {
    double* W;
    int64_t n, naux, nocc;
    __device__ __forceinline__ void operator()(int m, int i, double v, int) const {
        const int64_t q = m / n, mu = m % n;
        W[mu * (naux * nocc) + q * nocc + i] = v;
    }
};

__global__ void dfk_fold_kernel(const double* __restrict__ part, int nsplit, int64_t n,
                                double* __restrict__ k) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * n) return;
    const int64_t r = idx / n, c = idx % n;
    const int64_t lo = r < c ? r : c, hi = r < c ? c : r;
    double s = 0.0;
    for (int sp = 0; sp < nsplit; ++sp) s += part[(int64_t)sp * n * n + lo * n + hi];
    k[idx] = s;
}

static fc_status dfjk_smem_once() {
    static std::atomic<uint64_t> done{0};
    uint64_t bit = 0;
    if (!attrs_needed(done, &bit)) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiScatterW>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiSplit>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    done.fetch_or(bit);
    return FC_OK;
}

// c = V^-1 d in place (when a metric is set), pass 2 J_k = sum_P Bp[P, k] c_P
// in nsplit row splits (part: nsplit x ld doubles), fixed-order fold and unpack.
template <typename TB>
static fc_status dfj_solve_pass2(fc_dfjk* h, const TB* bp, double* dp, double* part, int nsplit, double* j,
                                 cudaStream_t st) {
    const int64_t naux = h->naux, n = h->n, pair = h->pair;
    constexpr bool F32 = sizeof(TB) == 4;
    const int64_t ld = F32 ? h->ld32 : pair;
    if (h->l_chol) chol_solve_kernel<<<1, 1024, 0, st>>>(h->l_chol, naux, dp);
    const int64_t rps = (naux + nsplit - 1) / nsplit;
    if constexpr (F32) {
        dim3 g2((unsigned)((ld / 4 + 255) / 256), nsplit);
        if (h->pk32_subnormal)
            dfj_pass2_f32v_kernel<true><<<g2, 256, 0, st>>>((const float*)bp, naux, ld, dp, rps, part);
        else
            dfj_pass2_f32v_kernel<false><<<g2, 256, 0, st>>>((const float*)bp, naux, ld, dp, rps, part);
    } else {
        dim3 g2((unsigned)((pair + 255) / 256), nsplit);
        dfj_pass2_kernel<TB><<<g2, 256, 0, st>>>(bp, naux, pair, dp, rps, part);
    }
    dfj_unpack_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, st>>>(part, nsplit, ld, n, j);
    return check_launch("DF-J pass 2");
}

template <typename TB>
static fc_status dfj_build_t(fc_dfjk* h, const TB* bp, int prec, const double* d, double* j, cudaStream_t st,
                             fc_stats* stats) {
    const int64_t naux = h->naux, n = h->n, pair = h->pair;
    constexpr bool F32 = sizeof(TB) == 4;
    const int64_t ld = F32 ? h->ld32 : pair;  // row pitch of bp
    void *vw, *vpart;
    const int nsplit = 4;
    const int64_t seg = F32 ? DFJ_SEG_BYTES / 2 / 16 : DFJ_SEG_BYTES / (int64_t)sizeof(TB);  // float4 or TB units
    const int64_t nseg = ((F32 ? ld / 4 : pair) + seg - 1) / seg;
    FC_TRY(ws_get(WS_MISC, (ld + naux * (nseg + 1) + 64) * 8, &vw));
    FC_TRY(ws_get(WS_PART, (int64_t)nsplit * ld * 8, &vpart));
    double* w = (double*)vw;
    double* dp = w + ld;
    double* segp = dp + naux;
    Context& c = ctx();
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    if (ld > pair) FC_CUDA(cudaMemsetAsync(w + pair, 0, (ld - pair) * 8, st));
    density_weights_kernel<<<(unsigned)n, 128, 0, st>>>(d, n, w);
    if constexpr (F32) {
        const dim3 g1((unsigned)((naux + DFJ_ROWS - 1) / DFJ_ROWS), (unsigned)nseg);
        if (h->pk32_subnormal)
            dfj_pass1_f32v_kernel<true><<<g1, 256, 0, st>>>((const float*)bp, naux, ld, seg, w, segp);
        else
            dfj_pass1_f32v_kernel<false><<<g1, 256, 0, st>>>((const float*)bp, naux, ld, seg, w, segp);
    } else {
        dfj_pass1_kernel<TB><<<dim3((unsigned)naux, (unsigned)nseg), 256, 0, st>>>(bp, pair, seg, w, segp);
    }
    dfj_seg_sum_kernel<<<(unsigned)((naux + 255) / 256), 256, 0, st>>>(segp, (int)nseg, naux, dp);
    FC_TRY(dfj_solve_pass2<TB>(h, bp, dp, (double*)vpart, nsplit, j, st));
    FC_TRY(check_launch("DF-J kernels"));
    if (stats) {
        FC_CUDA(cudaEventRecord(c.ev1, st));
        FC_CUDA(cudaEventSynchronize(c.ev1));
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        stats->flops = 4.0 * (double)naux * (double)pair;
        stats->precision = prec;
        stats->launches += 5 + (h->l_chol ? 1 : 0);
        stats->main_launches = 2;
        stats->main_ms = ms;
        stats->main_flops = stats->flops;
        stats->main_bytes = 2.0 * sizeof(TB) * (double)naux * (double)pair;
    }
    return FC_OK;
}

fc_status dfj_build_f64(fc_dfjk* h, const double* d, double* j, cudaStream_t st, fc_stats* stats) {
    return dfj_build_t<double>(h, h->b_pk, FC_PREC_F64, d, j, st, stats);
}

fc_status dfj_build_mixed(fc_dfjk* h, const double* d, double* j, cudaStream_t st, fc_stats* stats) {
    if (!h->pk32) return fail(FC_ERR_KERNEL, "DF-J: handle has no FP32 copy (created with FC_PREC_F64)");
    return dfj_build_t<float>(h, h->pk32, FC_PREC_MIXED, d, j, st, stats);
}

fc_status dfjk_prepare_mixed(fc_dfjk* h, cudaStream_t st) {
    h->ld32 = (h->pair + 3) / 4 * 4;
    const int64_t npk = h->naux * h->ld32;
    FC_TRY(pool_reserve((uint64_t)npk * 4));
    FC_CUDA(cudaMalloc(&h->pk32, (size_t)npk * 4));
    h->bytes += (uint64_t)npk * 4;
    if (h->ld32 != h->pair) FC_CUDA(cudaMemsetAsync(h->pk32, 0, (size_t)npk * 4, st));
    void* vf;
    FC_TRY(ws_get(WS_OUT, 256, &vf));
    FC_CUDA(cudaMemsetAsync(vf, 0, 256, st));
    round_f32_kernel<<<(unsigned)((h->naux * h->pair + 255) / 256), 256, 0, st>>>(h->b_pk, h->naux, h->pair, h->ld32,
                                                                                 h->pk32, (int*)vf);
    FC_TRY(check_launch("round_f32_kernel"));
    int bad = 0;
    FC_CUDA(cudaMemcpyAsync(&bad, vf, sizeof(int), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (bad & 1) return fail(FC_ERR_RANGE, "DF-JK: tensor element outside the FP32 range (mixed storage refused)");
    h->pk32_subnormal = (bad & 2) != 0;
    // square handles also keep the exact-slice split for the tensor-core DF-K
    if (h->b_sq) FC_TRY(dfk_prepare_split(h, st));
    return FC_OK;
}

void dfjk_free_mixed(fc_dfjk* h) {
    if (h->pk32) cudaFree(h->pk32);
    if (h->sq_split) cudaFree(h->sq_split);
    h->pk32 = nullptr;
    h->sq_split = nullptr;
    h->sq_scale = nullptr;
}

fc_status dfk_build_f64(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, cudaStream_t st,
                        fc_stats* stats, const JFork* jf) {
    FC_TRY(dfjk_smem_once());
    const int64_t naux = h->naux, n = h->n;
    const int64_t M1 = naux * n;
    if (M1 > INT32_MAX || (M1 + DG_BM - 1) / DG_BM > 65535)
        return fail(FC_ERR_LAYOUT, "DF-K: naux*n too large for one stage-1 launch");
    const int64_t kdim = naux * nocc;
    const int tm = (int)((n + DG_BM - 1) / DG_BM), tn = (int)((n + DG_BN - 1) / DG_BN);
    int upper = 0;
    for (int a = 0; a < tm; ++a)
        for (int b = 0; b < tn; ++b) upper += (a * DG_BM <= b * DG_BN + DG_BN - 1);
    int nsplit = (1200 + upper - 1) / upper;
    if (nsplit < 1) nsplit = 1;
    if (nsplit > 64) nsplit = 64;
    int64_t kps = (kdim + nsplit - 1) / nsplit;
    kps = (kps + DG_BK - 1) / DG_BK * DG_BK;
    nsplit = (int)((kdim + kps - 1) / kps);

    void *vct, *vw, *vpart;
    FC_TRY(ws_get(WS_MISC, nocc * n * 8, &vct));
    FC_TRY(ws_get(WS_T, n * kdim * 8, &vw));
    FC_TRY(ws_get(WS_PART, (int64_t)nsplit * n * n * 8, &vpart));
    Context& c = ctx();
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    transpose_kernel<<<(unsigned)((n * nocc + 255) / 256), 256, 0, st>>>(c_occ, n, nocc, (double*)vct);
    {
        dim3 g((unsigned)((nocc + DG_BN - 1) / DG_BN), (unsigned)((M1 + DG_BM - 1) / DG_BM), 1);
        EpiScatterW epi{(double*)vw, n, naux, nocc};
        dgemm_tn_kernel<EpiScatterW><<<g, 256, DG_SMEM, st>>>(h->b_sq, n, (const double*)vct, n, (int)M1,
                                                               (int)nocc, n, n, 0, epi);
    }
    if (jf) {  // J: pass-1 vector from W = B C, second pass forked off
        // W rows of nocc doubles: 16-byte vectors when nocc is even (and W's base is)
        if (nocc % 2 == 0) {
            const int64_t dq = dfj_d_rows(nocc, 2);
            dfj_d_from_w_kernel<double, 2><<<dim3((unsigned)((naux + dq - 1) / dq), DFJ_DY), 256, 0, st>>>(
                (const double*)vw, kdim, nocc, n, nocc, naux, dq, c_occ, jf->dpart);
        } else {
            const int64_t dq = dfj_d_rows(nocc, 1);
            dfj_d_from_w_kernel<double, 1><<<dim3((unsigned)((naux + dq - 1) / dq), DFJ_DY), 256, 0, st>>>(
                (const double*)vw, kdim, nocc, n, nocc, naux, dq, c_occ, jf->dpart);
        }
        dfj_d_sum_kernel<<<(unsigned)((naux + 255) / 256), 256, 0, st>>>(jf->dpart, naux, jf->dp);
        FC_TRY(dfj_fork_pass2(h, *jf, st));
    }
    {
        dim3 g(tn, tm, nsplit);
        EpiSplit epi{(double*)vpart, n * n, (int)n};
        dgemm_tn_kernel<EpiSplit><<<g, 256, DG_SMEM, st>>>((const double*)vw, kdim, (const double*)vw, kdim,
                                                            (int)n, (int)n, kdim, kps, 1, epi);
    }
    dfk_fold_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, st>>>((const double*)vpart, nsplit, n, k);
    FC_TRY(check_launch("DF-K kernels"));
    if (jf) {  // join J's second pass
        FC_CUDA(cudaEventRecord(c.join, c.side));
        FC_CUDA(cudaStreamWaitEvent(st, c.join, 0));
    }
    if (stats) {
        FC_CUDA(cudaEventRecord(c.ev1, st));
        FC_CUDA(cudaEventSynchronize(c.ev1));
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        stats->flops = 4.0 * (double)naux * (double)n * (double)n * (double)nocc;
        stats->precision = FC_PREC_F64;
        stats->launches += 4;
        stats->main_launches = 2;
        stats->main_ms = ms;
        stats->main_flops = stats->flops;
        stats->main_bytes = 8.0 * (double)naux * (double)n * (double)n;
        stats->tile_m = DG_BM;
        stats->tile_n = DG_BN;
    }
    return FC_OK;
}

// J's second pass on the side stream, after everything `st` holds so far.
fc_status dfj_fork_pass2(fc_dfjk* h, const JFork& f, cudaStream_t st) {
    Context& c = ctx();
    FC_CUDA(cudaEventRecord(c.fork, st));
    FC_CUDA(cudaStreamWaitEvent(c.side, c.fork, 0));
    if (f.ev[0]) FC_CUDA(cudaEventRecord(f.ev[0], c.side));
    if (h->active != FC_PREC_F64) FC_TRY(dfj_solve_pass2<float>(h, h->pk32, f.dp, f.part, f.nsplit, f.j, c.side));
    else FC_TRY(dfj_solve_pass2<double>(h, h->b_pk, f.dp, f.part, f.nsplit, f.j, c.side));
    if (f.ev[1]) FC_CUDA(cudaEventRecord(f.ev[1], c.side));
    return FC_OK;
}

// J and K of one occupied-orbital matrix: K as dfk_build_*, J = J(C C^T) from
// the pass-1 vector d_P = <B_P, C C^T> that the K stage's W = B C already
// holds (one kernel over W instead of a pass over B), then the metric solve
// and J's second pass over the packed rows (FP64, or the FP32 copy in mixed)
// on the side stream, where it overlaps the rest of DF-K (W's split and the
// tensor-core W W^T).
static fc_status dfjk_build_occ(fc_dfjk* h, const double* c_occ, int64_t nocc, double* j, double* k,
                                cudaStream_t st, fc_stats* stats) {
    const bool mixed = h->active != FC_PREC_F64;
    const int nsplit = 4;
    const int64_t ld = mixed ? h->ld32 : h->pair;
    // d, then the pass-2 partials at a 256-byte aligned offset (the FP32
    // pass stores them as double2)
    const int64_t dlen = (h->naux + 31) / 32 * 32;
    void* vd;
    FC_TRY(ws_get(WS_JD, (size_t)((1 + DFJ_DY) * dlen + (int64_t)nsplit * ld) * 8, &vd));
    JFork jf{(double*)vd, (double*)vd + dlen, (double*)vd + (1 + DFJ_DY) * dlen, nsplit, j, {nullptr, nullptr}};
    cudaEvent_t* ev = nullptr;
    if (stats) {
        FC_TRY(timing_events2(1, &ev));
        jf.ev[0] = ev[0];
        jf.ev[1] = ev[1];
    }
    fc_stats sk{};
    if (mixed) FC_TRY(dfk_build_mixed(h, c_occ, nocc, k, st, stats ? &sk : nullptr, &jf));
    else FC_TRY(dfk_build_f64(h, c_occ, nocc, k, st, stats ? &sk : nullptr, &jf));
    if (stats) {
        float jms = 0.f;
        FC_CUDA(cudaEventSynchronize(ev[1]));
        FC_CUDA(cudaEventElapsedTime(&jms, ev[0], ev[1]));
        *stats = sk;  // kernel_ms spans the whole call (the join comes before its last event)
        stats->flops = sk.flops + 2.0 * (double)h->naux * (double)h->pair;  // + J pass 2
        stats->launches = sk.launches + 3 + (h->l_chol ? 1 : 0);
        stats->aux_launches = 1;
        stats->aux_ms = jms;
        stats->aux_flops = 2.0 * (double)h->naux * (double)h->pair;
        stats->aux_bytes = (mixed ? 4.0 : 8.0) * (double)h->naux * (double)h->pair;
    }
    return FC_OK;
}

}  // namespace fc

// ------------------------------------------------------------------ ABI --

namespace {

fc_status create_common(const double* b, int64_t naux, int64_t n, int32_t layout, int32_t precision,
                        bool host, cudaStream_t st, fc_dfjk** out) {
    if (!out) return fail(FC_ERR_INVALID, "fc_dfjk_create: null out");
    *out = nullptr;
    if (naux <= 0 || n <= 0) return fail(FC_ERR_LAYOUT, "fc_dfjk_create: naux and n must be > 0");
    if (!b) return fail(FC_ERR_INVALID, "fc_dfjk_create: null tensor");
    if (layout != FC_LAYOUT_SQUARE && layout != FC_LAYOUT_PACKED_LOWER)
        return fail(FC_ERR_INVALID, "fc_dfjk_create: unknown layout");
    if (precision < FC_PREC_F64 || precision > FC_PREC_MIXED_FAST)
        return fail(FC_ERR_INVALID, "fc_dfjk_create: unknown precision");
    int64_t nn, pair = n * (n + 1) / 2, bytes_sq = 0, bytes_pk;
    if (!mul_ok(n, n, &nn) || !mul_ok(nn, naux, &bytes_sq) || !mul_ok(bytes_sq, 8, &bytes_sq))
        return fail(FC_ERR_LAYOUT, "fc_dfjk_create: size overflow");
    if (!mul_ok(pair, naux, &bytes_pk) || !mul_ok(bytes_pk, 8, &bytes_pk))
        return fail(FC_ERR_LAYOUT, "fc_dfjk_create: size overflow");
    if (layout == FC_LAYOUT_PACKED_LOWER) bytes_sq = 0;
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    const uint64_t need = (uint64_t)bytes_sq + (uint64_t)bytes_pk;
    FC_TRY(pool_reserve(need));
    fc_dfjk* h = new fc_dfjk{};
    h->naux = naux;
    h->n = n;
    h->pair = pair;
    h->layout = layout;
    h->precision = precision;
    h->active = precision;
    h->bytes = need;
    auto bail = [&](fc_status s) {
        if (h->b_sq) cudaFree(h->b_sq);
        if (h->b_pk) cudaFree(h->b_pk);
        dfjk_free_mixed(h);
        delete h;
        return s;
    };
    cudaError_t e;
    if (bytes_sq) {
        e = cudaMalloc(&h->b_sq, bytes_sq);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(B square)"));
    }
    e = cudaMalloc(&h->b_pk, bytes_pk);
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(B packed)"));
    const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (layout == FC_LAYOUT_SQUARE) {
        e = cudaMemcpyAsync(h->b_sq, b, bytes_sq, kind, st);
        if (e != cudaSuccess) return bail(cuda_fail(e, "upload B"));
        dim3 g((unsigned)n, (unsigned)naux);
        pack_lower_kernel<<<g, 128, 0, st>>>(h->b_sq, n, pair, h->b_pk);
        fc_status s = check_launch("pack_lower_kernel");
        if (s != FC_OK) return bail(s);
    } else {
        e = cudaMemcpyAsync(h->b_pk, b, bytes_pk, kind, st);
        if (e != cudaSuccess) return bail(cuda_fail(e, "upload B"));
    }
    if (precision != FC_PREC_F64) {
        fc_status s = dfjk_prepare_mixed(h, st);
        if (s != FC_OK) return bail(s);
    }
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return bail(cuda_fail(e, "fc_dfjk_create sync"));
    ctx().handle_bytes += h->bytes;
    *out = h;
    return FC_OK;
}

}  // namespace

extern "C" {

fc_status fc_dfjk_create(const double* b, int64_t naux, int64_t n, int32_t layout, int32_t precision,
                         fc_dfjk** out) {
    return create_common(b, naux, n, layout, precision, true, ctx().stream, out);
}

fc_status fc_dfjk_create_dev(const double* b, int64_t naux, int64_t n, int32_t layout, int32_t precision,
                             void* stream, fc_dfjk** out) {
    return create_common(b, naux, n, layout, precision, false, pick_stream(stream), out);
}

fc_status fc_dfj_set_metric_chol(fc_dfjk* h, const double* l) {
    if (!h || !l) return fail(FC_ERR_INVALID, "fc_dfj_set_metric_chol: null argument");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    const uint64_t bytes = (uint64_t)h->naux * h->naux * 8;
    if (!h->l_chol) {
        FC_TRY(pool_reserve(bytes));
        FC_CUDA(cudaMalloc(&h->l_chol, bytes));
        h->bytes += bytes;
        ctx().handle_bytes += bytes;
    }
    FC_CUDA(cudaMemcpy(h->l_chol, l, bytes, cudaMemcpyHostToDevice));
    return FC_OK;
}

fc_status fc_dfj_build_dev(fc_dfjk* h, const double* d, double* j, void* stream, fc_stats* stats) {
    if (!h || !d || !j) return fail(FC_ERR_INVALID, "fc_dfj_build: null argument");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = pick_stream(stream);
    if (h->active == FC_PREC_F64) return dfj_build_f64(h, d, j, st, stats);
    return dfj_build_mixed(h, d, j, st, stats);
}

fc_status fc_dfj_build(fc_dfjk* h, const double* d, double* j, fc_stats* stats) {
    if (!h || !d || !j) return fail(FC_ERR_INVALID, "fc_dfj_build: null argument");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = ctx().stream;
    const size_t nn = (size_t)h->n * h->n * 8;
    void* buf;
    FC_TRY(ws_get(WS_B, 2 * nn, &buf));
    double* dd = (double*)buf;
    double* dj = dd + h->n * h->n;
    FC_CUDA(cudaMemcpyAsync(dd, d, nn, cudaMemcpyHostToDevice, st));
    if (h->active == FC_PREC_F64) FC_TRY(dfj_build_f64(h, dd, dj, st, stats));
    else FC_TRY(dfj_build_mixed(h, dd, dj, st, stats));
    FC_CUDA(cudaMemcpyAsync(j, dj, nn, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes += nn;
        stats->d2h_bytes += nn;
    }
    return FC_OK;
}

fc_status fc_dfk_build_occ_dev(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, void* stream,
                               fc_stats* stats) {
    if (!h || !k || (nocc > 0 && !c_occ)) return fail(FC_ERR_INVALID, "fc_dfk_build_occ: null argument");
    if (nocc < 0) return fail(FC_ERR_LAYOUT, "fc_dfk_build_occ: nocc < 0");
    if (!h->b_sq) return fail(FC_ERR_LAYOUT, "fc_dfk_build_occ: needs an FC_LAYOUT_SQUARE handle");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = pick_stream(stream);
    if (nocc == 0) {  // empty channel: K is identically zero (df_k.rs:1428-1436)
        FC_CUDA(cudaMemsetAsync(k, 0, h->n * h->n * 8, st));
        return FC_OK;
    }
    if (h->active == FC_PREC_F64) return dfk_build_f64(h, c_occ, nocc, k, st, stats);
    return dfk_build_mixed(h, c_occ, nocc, k, st, stats);
}

fc_status fc_dfk_build_occ(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, fc_stats* stats) {
    if (!h || !k || (nocc > 0 && !c_occ)) return fail(FC_ERR_INVALID, "fc_dfk_build_occ: null argument");
    if (nocc < 0) return fail(FC_ERR_LAYOUT, "fc_dfk_build_occ: nocc < 0");
    if (!h->b_sq) return fail(FC_ERR_LAYOUT, "fc_dfk_build_occ: needs an FC_LAYOUT_SQUARE handle");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = ctx().stream;
    const size_t nn = (size_t)h->n * h->n * 8, nc = (size_t)h->n * nocc * 8;
    if (nocc == 0) {
        for (size_t q = 0; q < (size_t)h->n * h->n; ++q) k[q] = 0.0;
        return FC_OK;
    }
    void* buf;
    FC_TRY(ws_get(WS_B, nn + nc, &buf));
    double* dk = (double*)buf;
    double* dc = dk + h->n * h->n;
    FC_CUDA(cudaMemcpyAsync(dc, c_occ, nc, cudaMemcpyHostToDevice, st));
    if (h->active == FC_PREC_F64) FC_TRY(dfk_build_f64(h, dc, nocc, dk, st, stats));
    else FC_TRY(dfk_build_mixed(h, dc, nocc, dk, st, stats));
    FC_CUDA(cudaMemcpyAsync(k, dk, nn, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes += nc;
        stats->d2h_bytes += nn;
    }
    return FC_OK;
}

fc_status fc_dfjk_build_occ_dev(fc_dfjk* h, const double* c_occ, int64_t nocc, double* j, double* k, void* stream,
                               fc_stats* stats) {
    if (!h || !j || !k || (nocc > 0 && !c_occ)) return fail(FC_ERR_INVALID, "fc_dfjk_build_occ: null argument");
    if (nocc < 0) return fail(FC_ERR_LAYOUT, "fc_dfjk_build_occ: nocc < 0");
    if (!h->b_sq) return fail(FC_ERR_LAYOUT, "fc_dfjk_build_occ: needs an FC_LAYOUT_SQUARE handle");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = pick_stream(stream);
    if (nocc == 0) {  // empty channel: D = 0, J = K = 0
        FC_CUDA(cudaMemsetAsync(j, 0, h->n * h->n * 8, st));
        FC_CUDA(cudaMemsetAsync(k, 0, h->n * h->n * 8, st));
        return FC_OK;
    }
    return dfjk_build_occ(h, c_occ, nocc, j, k, st, stats);
}

fc_status fc_dfjk_build_occ(fc_dfjk* h, const double* c_occ, int64_t nocc, double* j, double* k, fc_stats* stats) {
    if (!h || !j || !k || (nocc > 0 && !c_occ)) return fail(FC_ERR_INVALID, "fc_dfjk_build_occ: null argument");
    if (nocc < 0) return fail(FC_ERR_LAYOUT, "fc_dfjk_build_occ: nocc < 0");
    if (!h->b_sq) return fail(FC_ERR_LAYOUT, "fc_dfjk_build_occ: needs an FC_LAYOUT_SQUARE handle");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    const size_t nn = (size_t)h->n * h->n * 8, nc = (size_t)h->n * nocc * 8;
    if (nocc == 0) {
        for (size_t q = 0; q < (size_t)h->n * h->n; ++q) j[q] = k[q] = 0.0;
        return FC_OK;
    }
    cudaStream_t st = ctx().stream;
    void* buf;
    FC_TRY(ws_get(WS_B, 2 * nn + nc, &buf));
    double* dj = (double*)buf;
    double* dk = dj + h->n * h->n;
    double* dc = dk + h->n * h->n;
    FC_CUDA(cudaMemcpyAsync(dc, c_occ, nc, cudaMemcpyHostToDevice, st));
    FC_TRY(dfjk_build_occ(h, dc, nocc, dj, dk, st, stats));
    FC_CUDA(cudaMemcpyAsync(j, dj, nn, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(k, dk, nn, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes += nc;
        stats->d2h_bytes += 2 * nn;
    }
    return FC_OK;
}

fc_status fc_dfjk_set_precision(fc_dfjk* h, int32_t precision) {
    if (!h) return fail(FC_ERR_INVALID, "fc_dfjk_set_precision: null handle");
    if (precision == FC_PREC_F64) {
        h->active = FC_PREC_F64;
        return FC_OK;
    }
    if (precision != h->precision || h->precision == FC_PREC_F64)
        return fail(FC_ERR_INVALID, "fc_dfjk_set_precision: the handle holds no copy for that precision");
    h->active = precision;
    return FC_OK;
}

fc_status fc_dfjk_destroy(fc_dfjk* h) {
    if (!h) return FC_OK;
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.device >= 0) cudaSetDevice(c.device);
    cudaDeviceSynchronize();
    if (h->b_sq) cudaFree(h->b_sq);
    if (h->b_pk) cudaFree(h->b_pk);
    if (h->l_chol) cudaFree(h->l_chol);
    dfjk_free_mixed(h);
    c.handle_bytes -= h->bytes < c.handle_bytes ? h->bytes : c.handle_bytes;
    delete h;
    return FC_OK;
}

}  // extern "C"
