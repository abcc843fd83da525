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
    void* sq_split = nullptr;  // square tensor: three bf16 slices per row (Q, mu) for DF-K
    double* sq_scale = nullptr;  // their power-of-two row scales (inside the sq_split block)
    uint64_t bytes = 0;        // device bytes owned by the handle
};

namespace fc {
fc_status dfj_build_f64(fc_dfjk* h, const double* d, double* j, cudaStream_t st, fc_stats* stats);
fc_status dfk_build_f64(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, cudaStream_t st,
                        fc_stats* stats);
fc_status dfjk_prepare_mixed(fc_dfjk* h, cudaStream_t st);
fc_status dfk_prepare_split(fc_dfjk* h, cudaStream_t st);
void dfjk_free_mixed(fc_dfjk* h);
fc_status dfj_build_mixed(fc_dfjk* h, const double* d, double* j, cudaStream_t st, fc_stats* stats);
fc_status dfk_build_mixed(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k, cudaStream_t st,
                          fc_stats* stats);
}  // namespace fc
