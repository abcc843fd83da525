// RI Lagrangian Imat on the device, the first consumer of the RI-MP2 adjoint
// (x_ov = Gamma / 4) in the analytic gradient (build_imat_ri / imat_fill_rows,
// ferric-mp2/src/zvector.rs:735-832):
//     Imat[q, fo + i] = -2 sum_{P,a} x_ov[P, i*nv + a] b_full[P, q, nt + a]
//     Imat[q, nt + a] = -2 sum_{P,i} x_ov[P, i*nv + a] b_full[P, q, fo + i]
// (nt = fo + nocc; frozen-core columns stay zero).  Each is one GEMM once the
// operands are permuted so the contracted pair (P, a) or (P, i) is
// contiguous: G_vir[q][P*nv + a], X_occ[i][P*nv + a]; G_occ[q][P*no + i],
// X_vir[a][P*no + i].  FP64: DMMA; FC_PREC_MIXED: exact integer slices on
// tcgen05 with the k-panel FP64 flush (K = naux*nvir or naux*nocc).
#include <algorithm>
#include <vector>

#include "dgemm_tn.cuh"
#include "fc_internal.cuh"
#include "fx_split.cuh"
#include "tmap.cuh"
#include "xgemm.cuh"

namespace fc {

namespace {

int64_t rup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// g[q][P*len + k] = b_full[P][q][lo + k]
__global__ void imat_gather_kernel(const double* __restrict__ bf, int64_t naux, int64_t nmo, int64_t lo,
                                   int64_t len, double* __restrict__ g) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = nmo * naux * len;
    if (e >= total) return;
    const int64_t k = e % len, p = (e / len) % naux, q = e / (len * naux);
    g[e] = bf[(p * nmo + q) * nmo + lo + k];
}

// occ = true: xo[i][P*nv + a] = x[P][i*nv + a]; else xv[a][P*no + i] = x[P][i*nv + a]
__global__ void imat_permute_x_kernel(const double* __restrict__ x, int64_t naux, int64_t no, int64_t nv,
                                      bool occ, double* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= naux * no * nv) return;
    const int64_t p = e / (no * nv), i = (e / nv) % no, a = e % nv;
    const double v = x[e];
    if (occ) out[(i * naux + p) * nv + a] = v;
    else out[(a * naux + p) * no + i] = v;
}

// Row r of an FP64 matrix (pitch Kv) -> three slices [3][slice_rows][ldk], scale s[r].
__global__ void __launch_bounds__(256) imat_split_kernel(const double* __restrict__ x, int64_t Kv, int64_t ldk,
                                                         int64_t slice_rows, double* __restrict__ s,
                                                         __nv_bfloat16* __restrict__ xs, int* bad) {
    const int64_t r = blockIdx.x;
    bool nf = false;
    for (int64_t k = threadIdx.x; k < Kv; k += 256) nf |= !(fabs(x[r * Kv + k]) <= 1.0e300);
    if (nf) atomicOr(bad, 1);
    split_fx_qrows_body(x, 1, Kv, ldk, ldk, slice_rows, s, xs, r);
}

// split-K partial tile of the exact-slice GEMM: part[item][row][col] = s_m s_n acc
struct EpiTile {
    const double* sa;
    const double* sb;
    double* part;
    int M, N;
    __device__ void operator()(int64_t t, int4 it, int row, int c0, const double (&acc)[32]) const {
        const int m = it.x * xg::BM + row;
        double* dst = part + t * (128 * 128) + row * 128 + c0;
        const double s = m < M ? sa[m] : 0.0;
#pragma unroll
        for (int c = 0; c < 32; c += 2) {
            const int n = it.y * 128 + c0 + c;
            const double v0 = (m < M && n < N) ? s * sb[n] * acc[c] : 0.0;
            const double v1 = (m < M && n + 1 < N) ? s * sb[n + 1] * acc[c + 1] : 0.0;
            *reinterpret_cast<double2*>(dst + c) = make_double2(v0, v1);
        }
    }
};

// out[m * ldo + col0 + n] = alpha * sum over the splits (in order) of the
// partials; tiled (tile-major, split-minor, 128 x 128) or plain [split][m][n].
__global__ void imat_fold_kernel(const double* __restrict__ part, int nsplit, int tiled, int ntm, int M, int N,
                                 double alpha, double* __restrict__ out, int64_t ldo, int64_t col0) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)M * N) return;
    const int m = (int)(e / N), n = (int)(e % N);
    double s = 0.0;
    if (tiled) {
        const int64_t tile = (int64_t)(n / 128) * ntm + m / 128;
        const int64_t off = (int64_t)(m % 128) * 128 + (n % 128);
        for (int sp = 0; sp < nsplit; ++sp) s += part[(tile * nsplit + sp) * (128 * 128) + off];
    } else {
        for (int sp = 0; sp < nsplit; ++sp) s += part[(int64_t)sp * M * N + e];
    }
    out[(int64_t)m * ldo + col0 + n] = alpha * s;
}

bool g_imat_attr = false;

fc_status imat_attrs() {
    if (g_imat_attr) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiSplit>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(xgemm_kernel<128, EpiTile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 xg::Cfg<128>::SMEM));
    g_imat_attr = true;
    return FC_OK;
}

// out[:, col0 : col0 + N] = alpha A B^T with A (M x K), B (N x K) row-major.
// Tall-skinny (M = nmo, N = nocc or nvir, K = naux * (nvir or nocc)): split
// over K into about two items per SM, partials folded in a fixed order.
fc_status imat_gemm(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double alpha, double* out,
                    int64_t ldo, int64_t col0, int precision, cudaStream_t st, int* flags) {
    const int sms = ctx().sm_count;
    void* vpart;
    if (precision == FC_PREC_F64) {
        const int tm = (int)((M + DG_BM - 1) / DG_BM), tn = (int)((N + DG_BN - 1) / DG_BN);
        int nsplit = std::max(1, std::min<int>(64, (2 * sms + tm * tn - 1) / (tm * tn)));
        int64_t kps = rup((K + nsplit - 1) / nsplit, DG_BK);
        nsplit = (int)((K + kps - 1) / kps);
        FC_TRY(ws_get(WS_PART, (size_t)nsplit * M * N * 8, &vpart));
        dim3 g((unsigned)tn, (unsigned)tm, (unsigned)nsplit);
        EpiSplit epi{(double*)vpart, M * N, (int)N};
        dgemm_tn_kernel<EpiSplit><<<g, 256, DG_SMEM, st>>>(A, K, B, K, (int)M, (int)N, K, kps, 0, epi);
        imat_fold_kernel<<<(unsigned)((M * N + 255) / 256), 256, 0, st>>>((const double*)vpart, nsplit, 0, 0, (int)M,
                                                                          (int)N, alpha, out, ldo, col0);
        return check_launch("Imat GEMM (FP64)");
    }
    const int64_t ldk = rup(K, 8), mp = rup(M, 128), np = rup(N, 128);
    void *vs, *vsc, *vtab;
    FC_TRY(ws_get(WS_SPLIT, (size_t)3 * (mp + np) * ldk * 2, &vs));
    FC_TRY(ws_get(WS_SCALE, (size_t)(mp + np) * 8, &vsc));
    __nv_bfloat16* as = (__nv_bfloat16*)vs;
    __nv_bfloat16* bs = as + (size_t)3 * mp * ldk;
    double* sa = (double*)vsc;
    double* sb = sa + mp;
    imat_split_kernel<<<(unsigned)M, 256, 0, st>>>(A, K, ldk, mp, sa, as, flags);
    imat_split_kernel<<<(unsigned)N, 256, 0, st>>>(B, K, ldk, np, sb, bs, flags);
    FC_TRY(check_launch("Imat splits"));
    const int ntm = (int)(mp / 128), ntn = (int)(np / 128), nks = (int)((K + 63) / 64);
    int nsplit = std::max(1, std::min<int>(nks, (sms + ntm * ntn - 1) / (ntm * ntn)));
    const int kps = (nks + nsplit - 1) / nsplit;
    nsplit = (nks + kps - 1) / kps;
    std::vector<int4> items;
    for (int tn = 0; tn < ntn; ++tn)
        for (int tm = 0; tm < ntm; ++tm)
            for (int sp = 0; sp < nsplit; ++sp) items.push_back(make_int4(tm, tn, sp * kps, std::min(kps, nks - sp * kps)));
    FC_TRY(ws_get(WS_PAIRS, items.size() * sizeof(int4), &vtab));
    FC_TRY(ws_get(WS_PART, items.size() * 128 * 128 * 8, &vpart));
    FC_CUDA(cudaMemcpyAsync(vtab, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    CUtensorMap ta, tb;
    FC_TRY(make_tmap_bf16_2d(&ta, as, K, 3 * mp, ldk * 2, 64, 128));
    FC_TRY(make_tmap_bf16_2d(&tb, bs, K, 3 * np, ldk * 2, 64, 128));
    XArgs a{(const int4*)vtab, (int64_t)items.size(), (int)mp, (int)np, flags + 1};
    EpiTile epi{sa, sb, (double*)vpart, (int)M, (int)N};
    const int grid = (int)std::min<int64_t>((int64_t)items.size(), sms);
    xgemm_kernel<128, EpiTile><<<grid, xg::Cfg<128>::THREADS, xg::Cfg<128>::SMEM, st>>>(ta, tb, a, epi);
    imat_fold_kernel<<<(unsigned)((M * N + 255) / 256), 256, 0, st>>>((const double*)vpart, nsplit, 1, ntm, (int)M,
                                                                      (int)N, alpha, out, ldo, col0);
    FC_TRY(check_launch("Imat GEMM (exact slices)"));
    // the slices and partials are reused by the next GEMM: finish this one first
    FC_CUDA(cudaStreamSynchronize(st));
    return FC_OK;
}

}  // namespace

fc_status rimp2_imat(const double* x_ov, const double* b_full, int64_t naux, int64_t nmo, int64_t nocc,
                     int64_t nvir, int64_t fo, int precision, double* imat, cudaStream_t st, fc_stats* stats) {
    FC_TRY(imat_attrs());
    Context& c = ctx();
    const int64_t nt = fo + nocc;
    void *vg, *vx, *vf;
    const int64_t big = std::max(nocc, nvir);
    FC_TRY(ws_get(WS_T, (size_t)nmo * naux * big * 8, &vg));
    FC_TRY(ws_get(WS_TS, (size_t)naux * nocc * nvir * 8, &vx));
    FC_TRY(ws_get(WS_OUT, 256, &vf));
    int* flags = (int*)vf;
    FC_CUDA(cudaMemsetAsync(vf, 0, 256, st));
    FC_CUDA(cudaMemsetAsync(imat, 0, (size_t)nmo * nmo * 8, st));
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    const int64_t nx = naux * nocc * nvir;
    // occupied columns: K = (P, a)
    imat_gather_kernel<<<(unsigned)((nmo * naux * nvir + 255) / 256), 256, 0, st>>>(b_full, naux, nmo, nt, nvir,
                                                                                   (double*)vg);
    imat_permute_x_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, st>>>(x_ov, naux, nocc, nvir, true, (double*)vx);
    FC_TRY(check_launch("Imat permutes"));
    FC_TRY(imat_gemm((const double*)vg, (const double*)vx, nmo, nocc, naux * nvir, -2.0, imat, nmo, fo, precision,
                     st, flags));
    // virtual columns: K = (P, i)
    imat_gather_kernel<<<(unsigned)((nmo * naux * nocc + 255) / 256), 256, 0, st>>>(b_full, naux, nmo, fo, nocc,
                                                                                   (double*)vg);
    imat_permute_x_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, st>>>(x_ov, naux, nocc, nvir, false, (double*)vx);
    FC_TRY(check_launch("Imat permutes"));
    FC_TRY(imat_gemm((const double*)vg, (const double*)vx, nmo, nvir, naux * nocc, -2.0, imat, nmo, nt, precision,
                     st, flags));
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "Imat: a non-finite operand element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "Imat: a pipeline wait ran out");
    if (stats) {
        FC_CUDA(cudaEventRecord(c.ev1, st));
        FC_CUDA(cudaEventSynchronize(c.ev1));
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        stats->flops = 4.0 * (double)nmo * naux * (double)nocc * nvir;
        stats->precision = precision == FC_PREC_F64 ? FC_PREC_F64 : FC_PREC_MIXED;
        stats->launches += precision == FC_PREC_F64 ? 6 : 10;
        stats->main_launches = 2;
        stats->main_ms = ms;
        stats->main_flops = stats->flops;
    }
    return FC_OK;
}

}  // namespace fc

using namespace fc;

namespace {

fc_status imat_common(const double* x_ov, const double* b_full, int64_t naux, int64_t nmo, int64_t nocc, int64_t nvir,
                      int64_t first_occ, int32_t precision, double* imat, bool host, void* stream, fc_stats* stats) {
    if (!x_ov || !b_full || !imat) return fail(FC_ERR_INVALID, "fc_rimp2_imat: null argument");
    if (naux <= 0 || nocc <= 0 || nvir <= 0 || first_occ < 0 || first_occ + nocc + nvir > nmo)
        return fail(FC_ERR_LAYOUT, "fc_rimp2_imat: need naux, nocc, nvir > 0 and first_occ + nocc + nvir <= nmo");
    if (precision != FC_PREC_F64 && precision != FC_PREC_MIXED)
        return fail(FC_ERR_INVALID, "fc_rimp2_imat: precision is FC_PREC_F64 or FC_PREC_MIXED");
    if (nmo * naux * std::max(nocc, nvir) > (int64_t)1 << 40 || nmo > INT32_MAX)
        return fail(FC_ERR_LAYOUT, "fc_rimp2_imat: shape too large");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx().stream;
    if (!host) return rimp2_imat(x_ov, b_full, naux, nmo, nocc, nvir, first_occ, precision, imat, st, stats);
    const size_t nx = (size_t)naux * nocc * nvir * 8, nb = (size_t)naux * nmo * nmo * 8, ni = (size_t)nmo * nmo * 8;
    void *dx, *db, *di;
    FC_TRY(ws_get(WS_B, nb, &db));
    FC_TRY(ws_get(WS_GAMMA, nx, &dx));
    FC_TRY(ws_get(WS_HOSTOUT, ni, &di));
    FC_CUDA(cudaMemcpyAsync(db, b_full, nb, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync(dx, x_ov, nx, cudaMemcpyHostToDevice, st));
    FC_TRY(rimp2_imat((const double*)dx, (const double*)db, naux, nmo, nocc, nvir, first_occ, precision, (double*)di,
                      st, stats));
    FC_CUDA(cudaMemcpyAsync(imat, di, ni, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes += nx + nb;
        stats->d2h_bytes += ni;
    }
    return FC_OK;
}

}  // namespace

extern "C" {

fc_status fc_rimp2_imat(const double* x_ov, const double* b_full, int64_t naux, int64_t nmo, int64_t nocc,
                        int64_t nvir, int64_t first_occ, int32_t precision, double* imat, fc_stats* stats) {
    return imat_common(x_ov, b_full, naux, nmo, nocc, nvir, first_occ, precision, imat, true, nullptr, stats);
}

fc_status fc_rimp2_imat_dev(const double* x_ov, const double* b_full, int64_t naux, int64_t nmo, int64_t nocc,
                            int64_t nvir, int64_t first_occ, int32_t precision, double* imat, void* stream,
                            fc_stats* stats) {
    return imat_common(x_ov, b_full, naux, nmo, nocc, nvir, first_occ, precision, imat, false, stream, stats);
}

}  // extern "C"
