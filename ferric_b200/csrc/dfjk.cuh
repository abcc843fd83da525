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
// J's second pass, forked onto the context's side stream once the DF-K stage
// has produced d (so it overlaps the rest of DF-K): J = Bp^T V^-1 d into j.
struct JFork {
    double* dp;    // [naux] d, solved in place
    double* dpart; // [DFJ_DY][naux] pass-1 partials over ranges of mu
    double* part;  // [nsplit][ld] pass-2 partials
    int nsplit;
    double* j;
    cudaEvent_t ev[2];  // timing of the pass on the side stream (or null)
};
fc_status dfj_fork_pass2(fc_dfjk* h, const JFork& f, cudaStream_t st);

// jf (optional): also J of C C^T.  The J pass-1 vector d_P = <B_P, C C^T> is
// taken from the stage-1 product W = B C (dfj_d_from_w_kernel) and J's second
// pass is forked off (dfj_fork_pass2); the call's stream joins it before
// returning.
fc_status dfk_build_f64(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, cudaStream_t st,
                        fc_stats* stats, const JFork* jf = nullptr);
fc_status dfjk_prepare_mixed(fc_dfjk* h, cudaStream_t st);
fc_status dfk_prepare_split(fc_dfjk* h, cudaStream_t st);
void dfjk_free_mixed(fc_dfjk* h);
fc_status dfj_build_mixed(fc_dfjk* h, const double* d, double* j, cudaStream_t st, fc_stats* stats);
fc_status dfk_build_mixed(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, cudaStream_t st,
                          fc_stats* stats, const JFork* jf = nullptr);

// d[Q] = sum_{mu, i < nocc} W[mu * ldw + Q * ldq + i] C[mu * nocc + i], in a
// fixed order: the J pass-1 vector d_Q = <B_Q, C C^T> = sum_mu (B_Q C)[mu, :] . C[mu, :]
// from the DF-K stage-1 product.  A CTA takes dq consecutive aux rows and one
// of DFJ_DY ranges of mu.  For every mu the dq rows' W values are one run of
// vectors of VE elements (16 bytes when VE > 1; a row's nv = ceil(nocc / VE)
// vectors, ldq a multiple of VE so every row starts on a vector): each thread
// owns fixed vectors of the run for every mu (coalesced), four mu in flight;
// elements past nocc are read but not used.  Per q the owning threads'
// partials are added in thread order into dpart[range][q]; dfj_d_sum_kernel
// adds the ranges in order.
constexpr int DFJ_DY = 8;  // ranges of mu
inline int64_t dfj_d_rows(int64_t nocc, int ve) {
    const int64_t nv = (nocc + ve - 1) / ve;
    return nv >= 256 ? 1 : 256 / nv;
}
template <typename T, int VE>
__global__ void __launch_bounds__(256) dfj_d_from_w_kernel(const T* __restrict__ W, int64_t ldw, int64_t ldq,
                                                           int64_t n, int64_t nocc, int64_t naux, int64_t dq,
                                                           const double* __restrict__ c,
                                                           double* __restrict__ dpart) {
    struct alignas(16) Vec { T e[VE]; };
    __shared__ double part[256];
    const int64_t nv = (nocc + VE - 1) / VE;
    const int64_t q0 = (int64_t)blockIdx.x * dq;
    const int64_t nq = naux - q0 < dq ? naux - q0 : dq;
    const int64_t per = (n + gridDim.y - 1) / gridDim.y;
    const int64_t m0 = (int64_t)blockIdx.y * per, m1 = m0 + per < n ? m0 + per : n;
    const int t = threadIdx.x;
    // nv <= 256: thread t owns vector t % nv of row t / nv; nv > 256 (dq = 1):
    // thread t owns vectors t, t + 256, ... of the one row
    const int64_t vstep = nv > 256 ? 256 : nv * dq;
    double s = 0.0;
    for (int64_t vt = t; vt < nq * nv; vt += vstep) {
        const int64_t ql = vt / nv, i0 = (vt % nv) * VE;
        const int64_t off = (q0 + ql) * ldq + i0;
        int64_t mu = m0;
        for (; mu + 3 < m1; mu += 4) {
            Vec v[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) v[r] = *reinterpret_cast<const Vec*>(W + (mu + r) * ldw + off);
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int e = 0; e < VE; ++e)
                    if (i0 + e < nocc) s += (double)v[r].e[e] * c[(mu + r) * nocc + i0 + e];
        }
        for (; mu < m1; ++mu) {
            const Vec v = *reinterpret_cast<const Vec*>(W + mu * ldw + off);
#pragma unroll
            for (int e = 0; e < VE; ++e)
                if (i0 + e < nocc) s += (double)v.e[e] * c[mu * nocc + i0 + e];
        }
        if (nv <= 256) break;
    }
    part[t] = s;
    __syncthreads();
    if (t < nq) {
        const int64_t k0 = nv > 256 ? 0 : t * nv, k1 = nv > 256 ? 256 : (t + 1) * nv;
        double r = 0.0;
        for (int64_t k = k0; k < k1; ++k) r += part[k];
        dpart[(int64_t)blockIdx.y * naux + q0 + t] = r;
    }
}

// d[q] = sum over the DFJ_DY ranges (in order) of dpart[range][q].
static __global__ void __launch_bounds__(256) dfj_d_sum_kernel(const double* __restrict__ dpart, int64_t naux,
                                                        double* __restrict__ d) {
    const int64_t q = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (q >= naux) return;
    double s = 0.0;
    for (int y = 0; y < DFJ_DY; ++y) s += dpart[(int64_t)y * naux + q];
    d[q] = s;
}
}  // namespace fc
