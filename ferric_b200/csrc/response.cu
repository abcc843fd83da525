// The GEMM-shaped part of the RI 3c/2c integral response of the RI-MP2
// gradient (integral_response_gradient_3c2c and ri_response_gradient_channels,
// ferric-mp2/src/gradient.rs:559-887), for one channel of weight w (2 for
// closed-shell RI-MP2, 1 per spin for the unrestricted form):
//     y_ov     = V^{-1/2 T} x_ov                            (naux x nov)
//     gamma_2c = -w (V^{-1/2 T} b_ov) y_ov^T                 (naux x naux)
//     g3c[P]   = w (G_P + G_P^T),   G_P = C_occ Y_P C_vir^T  (nbf x nbf)
// with Y_P the row P of y_ov read as nocc x nvir.  These are the weights the
// derivative integrals d(P|mu nu)/dR and d(P|Q)/dR are contracted with; the
// integral derivatives themselves stay with the caller (libint2), which
// takes g3c one aux slab [p0, p0 + np) at a time, as the reference builds
// it per aux shell.
//
// FP64 on the DMMA tile GEMM (the reference runs these products in FP64
// BLAS): y_ov and the fitted C = V^{-1/2 T} b_ov read V and the ov tensors
// MN-major (K = Q is their row index); gamma_2c is K-major over nov; the
// back-transform runs as T = Y C_vir^T over all rows (P, i) of the slab, then
// one batched GEMM G_P = C_occ T_P, then the weighted symmetrisation.
#include <algorithm>

#include "dgemm_tn.cuh"
#include "fc_internal.cuh"

namespace fc {

namespace {

// v -> C[z stride + m ldc + n]
struct EpiBatchStore {
    double* C;
    int64_t ldc, stride;
    __device__ __forceinline__ void operator()(int m, int n, double v, int z) const {
        C[(int64_t)z * stride + (int64_t)m * ldc + n] = v;
    }
};

// out[P][mu][nu] = w (G[P][mu][nu] + G[P][nu][mu])
__global__ void __launch_bounds__(256) sym_slab_kernel(const double* __restrict__ g, int64_t np, int64_t n, double w,
                                                       double* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (e >= np * n * n) return;
    const int64_t p = e / (n * n), r = (e / n) % n, c = e % n;
    out[e] = w * (g[e] + g[p * n * n + c * n + r]);
}

bool g_resp_attr = false;

fc_status resp_attrs() {
    if (g_resp_attr) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiStore, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_batched_kernel<EpiBatchStore, false, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    g_resp_attr = true;
    return FC_OK;
}

dim3 tiles(int64_t m, int64_t n, int64_t z = 1) {
    return dim3((unsigned)((n + DG_BN - 1) / DG_BN), (unsigned)((m + DG_BM - 1) / DG_BM), (unsigned)z);
}

fc_status response_2c(const double* x_ov, const double* b_ov, const double* vis, int64_t naux, int64_t nov, double w,
                      double* y_ov, double* gamma_2c, cudaStream_t st, fc_stats* stats) {
    FC_TRY(resp_attrs());
    Context& c = ctx();
    void* vc;
    FC_TRY(ws_get(WS_PART, (size_t)naux * nov * 8, &vc));
    double* cfit = (double*)vc;
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    // y[P, ia] = sum_Q V[Q, P] x[Q, ia];  C[P, ia] = sum_Q V[Q, P] b[Q, ia]
    dgemm_tn_kernel<EpiStore, true, true><<<tiles(naux, nov), 256, DG_SMEM, st>>>(
        vis, naux, x_ov, nov, (int)naux, (int)nov, naux, naux, 0, EpiStore{y_ov, nov, 1.0, 0});
    dgemm_tn_kernel<EpiStore, true, true><<<tiles(naux, nov), 256, DG_SMEM, st>>>(
        vis, naux, b_ov, nov, (int)naux, (int)nov, naux, naux, 0, EpiStore{cfit, nov, 1.0, 0});
    // gamma_2c[P, Q] = -w sum_ia C[P, ia] y[Q, ia]
    dgemm_tn_kernel<EpiStore><<<tiles(naux, naux), 256, DG_SMEM, st>>>(
        cfit, nov, y_ov, nov, (int)naux, (int)naux, nov, nov, 0, EpiStore{gamma_2c, naux, -w, 0});
    FC_TRY(check_launch("RI response 2c GEMMs"));
    if (stats) {
        FC_CUDA(cudaEventRecord(c.ev1, st));
        FC_CUDA(cudaEventSynchronize(c.ev1));
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        stats->flops = 6.0 * (double)naux * naux * nov;
        stats->precision = FC_PREC_F64;
        stats->launches += 3;
        stats->main_launches = 3;
        stats->main_ms = ms;
        stats->main_flops = stats->flops;
    }
    return FC_OK;
}

fc_status response_3c(const double* y_ov, const double* c_occ, const double* c_vir, int64_t nocc, int64_t nvir,
                      int64_t nbf, int64_t np, double w, double* g3c, cudaStream_t st, fc_stats* stats) {
    FC_TRY(resp_attrs());
    Context& c = ctx();
    void *vt, *vg;
    FC_TRY(ws_get(WS_T, (size_t)np * nocc * nbf * 8, &vt));
    FC_TRY(ws_get(WS_PART, (size_t)np * nbf * nbf * 8, &vg));
    double* T = (double*)vt;
    double* G = (double*)vg;
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    // T[(P, i), nu] = sum_a y[P, i nvir + a] C_vir[nu, a]   (rows (P, i) are nvir apart)
    dgemm_tn_kernel<EpiStore><<<tiles(np * nocc, nbf), 256, DG_SMEM, st>>>(
        y_ov, nvir, c_vir, nvir, (int)(np * nocc), (int)nbf, nvir, nvir, 0, EpiStore{T, nbf, 1.0, 0});
    // G_P[mu, nu] = sum_i C_occ[mu, i] T[(P, i), nu]
    dgemm_batched_kernel<EpiBatchStore, false, true><<<tiles(nbf, nbf, np), 256, DG_SMEM, st>>>(
        c_occ, nocc, 0, T, nbf, nocc * nbf, (int)nbf, (int)nbf, nocc, EpiBatchStore{G, nbf, nbf * nbf});
    const int64_t ne = np * nbf * nbf;
    sym_slab_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(G, np, nbf, w, g3c);
    FC_TRY(check_launch("RI response 3c GEMMs"));
    if (stats) {
        FC_CUDA(cudaEventRecord(c.ev1, st));
        FC_CUDA(cudaEventSynchronize(c.ev1));
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        stats->flops = 2.0 * (double)np * nocc * nvir * nbf + 2.0 * (double)np * nbf * nbf * nocc;
        stats->precision = FC_PREC_F64;
        stats->launches += 3;
        stats->main_launches = 2;
        stats->main_ms = ms;
        stats->main_flops = stats->flops;
    }
    return FC_OK;
}

fc_status resp_2c_common(const double* x_ov, const double* b_ov, const double* vis, int64_t naux, int64_t nov,
                         double w, double* y_ov, double* gamma_2c, bool host, void* stream, fc_stats* stats) {
    if (!x_ov || !b_ov || !vis || !y_ov || !gamma_2c) return fail(FC_ERR_INVALID, "fc_rimp2_response_2c: null argument");
    if (naux <= 0 || nov <= 0 || naux > INT32_MAX || nov > INT32_MAX)
        return fail(FC_ERR_LAYOUT, "fc_rimp2_response_2c: need 0 < naux, nov < 2^31");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = pick_stream(stream);
    if (!host) {
        FC_TRY(response_2c(x_ov, b_ov, vis, naux, nov, w, y_ov, gamma_2c, st, stats));
        FC_CUDA(cudaStreamSynchronize(st));
        return FC_OK;
    }
    const size_t no = (size_t)naux * nov * 8, nq = (size_t)naux * naux * 8;
    void *dx, *db, *dv, *dout;
    FC_TRY(ws_get(WS_B, no, &dx));
    FC_TRY(ws_get(WS_GAMMA, no, &db));
    FC_TRY(ws_get(WS_EPS, nq, &dv));
    FC_TRY(ws_get(WS_HOSTOUT, no + nq, &dout));
    FC_CUDA(cudaMemcpyAsync(dx, x_ov, no, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync(db, b_ov, no, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync(dv, vis, nq, cudaMemcpyHostToDevice, st));
    double* dy = (double*)dout;
    double* dg = dy + (size_t)naux * nov;
    FC_TRY(response_2c((const double*)dx, (const double*)db, (const double*)dv, naux, nov, w, dy, dg, st, stats));
    FC_CUDA(cudaMemcpyAsync(y_ov, dy, no, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(gamma_2c, dg, nq, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes += 2 * no + nq;
        stats->d2h_bytes += no + nq;
    }
    return FC_OK;
}

fc_status resp_3c_common(const double* y_ov, const double* c_occ, const double* c_vir, int64_t naux, int64_t nocc,
                         int64_t nvir, int64_t nbf, int64_t p0, int64_t np, double w, double* g3c, bool host,
                         void* stream, fc_stats* stats) {
    if (!y_ov || !c_occ || !c_vir || !g3c) return fail(FC_ERR_INVALID, "fc_rimp2_response_3c: null argument");
    if (naux <= 0 || nocc <= 0 || nvir <= 0 || nbf <= 0 || p0 < 0 || np <= 0 || p0 + np > naux)
        return fail(FC_ERR_LAYOUT, "fc_rimp2_response_3c: need naux, nocc, nvir, nbf, np > 0, 0 <= p0, p0 + np <= naux");
    if (np * nocc > INT32_MAX || nbf > INT32_MAX || np > 65535)
        return fail(FC_ERR_LAYOUT, "fc_rimp2_response_3c: slab too large (np <= 65535)");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = pick_stream(stream);
    const int64_t nov = nocc * nvir;
    if (!host) {
        FC_TRY(response_3c(y_ov + p0 * nov, c_occ, c_vir, nocc, nvir, nbf, np, w, g3c, st, stats));
        FC_CUDA(cudaStreamSynchronize(st));
        return FC_OK;
    }
    const size_t ny = (size_t)np * nov * 8, nco = (size_t)nbf * nocc * 8, ncv = (size_t)nbf * nvir * 8,
                 ng = (size_t)np * nbf * nbf * 8;
    void *dy, *dc, *dout;
    FC_TRY(ws_get(WS_B, ny, &dy));
    FC_TRY(ws_get(WS_EPS, nco + ncv, &dc));
    FC_TRY(ws_get(WS_HOSTOUT, ng, &dout));
    FC_CUDA(cudaMemcpyAsync(dy, y_ov + p0 * nov, ny, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync(dc, c_occ, nco, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync((char*)dc + nco, c_vir, ncv, cudaMemcpyHostToDevice, st));
    FC_TRY(response_3c((const double*)dy, (const double*)dc, (const double*)((char*)dc + nco), nocc, nvir, nbf, np, w,
                       (double*)dout, st, stats));
    FC_CUDA(cudaMemcpyAsync(g3c, dout, ng, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes += ny + nco + ncv;
        stats->d2h_bytes += ng;
    }
    return FC_OK;
}

}  // namespace

}  // namespace fc

using namespace fc;

extern "C" {

fc_status fc_rimp2_response_2c(const double* x_ov, const double* b_ov, const double* v_inv_sqrt, int64_t naux,
                               int64_t nov, double weight, double* y_ov, double* gamma_2c, fc_stats* stats) {
    return resp_2c_common(x_ov, b_ov, v_inv_sqrt, naux, nov, weight, y_ov, gamma_2c, true, nullptr, stats);
}

fc_status fc_rimp2_response_2c_dev(const double* x_ov, const double* b_ov, const double* v_inv_sqrt, int64_t naux,
                                   int64_t nov, double weight, double* y_ov, double* gamma_2c, void* stream,
                                   fc_stats* stats) {
    return resp_2c_common(x_ov, b_ov, v_inv_sqrt, naux, nov, weight, y_ov, gamma_2c, false, stream, stats);
}

fc_status fc_rimp2_response_3c(const double* y_ov, const double* c_occ, const double* c_vir, int64_t naux,
                               int64_t nocc, int64_t nvir, int64_t nbf, int64_t p0, int64_t np, double weight,
                               double* g3c, fc_stats* stats) {
    return resp_3c_common(y_ov, c_occ, c_vir, naux, nocc, nvir, nbf, p0, np, weight, g3c, true, nullptr, stats);
}

fc_status fc_rimp2_response_3c_dev(const double* y_ov, const double* c_occ, const double* c_vir, int64_t naux,
                                   int64_t nocc, int64_t nvir, int64_t nbf, int64_t p0, int64_t np, double weight,
                                   double* g3c, void* stream, fc_stats* stats) {
    return resp_3c_common(y_ov, c_occ, c_vir, naux, nocc, nvir, nbf, p0, np, weight, g3c, false, stream, stats);
}

}  // extern "C"
