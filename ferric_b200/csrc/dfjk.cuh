// Internal state of a DF-JK handle.
#pragma once
#include "fc_internal.cuh"

struct fc_dfjk {
    int64_t naux = 0, n = 0, pair = 0;
    int layout = 0, precision = 0;
    int active = 0;            // precision of the next build (FC_PREC_F64 or `precision`)
    double* b_sq = nullptr;    // (naux, n, n) dressed tensor (square handles)
    double* b_pk = nullptr;    // (naux, n(n+1)/2) packed lower rows
    double* l_chol = nullptr;  // metric Cholesky factor (raw-Bp form)
    // mixed handles
    float* pk32 = nullptr;     // packed rows, FP32 (DF-J reads 4 B per element), row pitch ld32
    int64_t ld32 = 0;          // pair rounded up to 4 (16-byte rows for float4 loads), zero padded
    bool pk32_subnormal = false;  // the FP32 copy holds subnormals: DF-J widens them exactly (slower)
    void* sq_split = nullptr;  // square tensor: three int8 slices per row (Q, mu) for DF-K
    double* sq_scale = nullptr;  // their power-of-two row scales (inside the sq_split block)
    uint64_t bytes = 0;        // device bytes owned by the handle
};

namespace fc {
fc_status dfj_build_f64(fc_dfjk* h, const double* d, double* j, cudaStream_t st, fc_stats* stats);
// d_out (optional, naux doubles): also the J pass-1 vector d_P = <B_P, C C^T>,
// taken from the stage-1 product W = B C (dfj_d_from_w_kernel)
fc_status dfk_build_f64(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, cudaStream_t st,
                        fc_stats* stats, double* d_out = nullptr);
fc_status dfjk_prepare_mixed(fc_dfjk* h, cudaStream_t st);
fc_status dfk_prepare_split(fc_dfjk* h, cudaStream_t st);
void dfjk_free_mixed(fc_dfjk* h);
fc_status dfj_build_mixed(fc_dfjk* h, const double* d, double* j, cudaStream_t st, fc_stats* stats);
fc_status dfk_build_mixed(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, cudaStream_t st,
                          fc_stats* stats, double* d_out = nullptr);

// d[Q] = sum_{mu, i < nocc} W[mu * ldw + Q * ldq + i] C[mu * nocc + i], in a
// fixed order: the J pass-1 vector d_Q = <B_Q, C C^T> = sum_mu (B_Q C)[mu, :] . C[mu, :]
// from the DF-K stage-1 product, one CTA per aux row.
template <typename T>
__global__ void __launch_bounds__(256) dfj_d_from_w_kernel(const T* __restrict__ W, int64_t ldw, int64_t ldq,
                                                           int64_t n, int64_t nocc, const double* __restrict__ c,
                                                           double* __restrict__ d) {
    __shared__ double sh[32];
    const int64_t q = blockIdx.x, tot = n * nocc;
    double s = 0.0;
    for (int64_t e = threadIdx.x; e < tot; e += 256) {
        const int64_t mu = e / nocc, i = e % nocc;
        s += (double)W[mu * ldw + q * ldq + i] * c[e];
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) d[q] = s;
}
}  // namespace fc
