// MO transform and metric dressing of the 3-index tensor on the device:
//     (Q|lr)      = sum_{mu nu} C_left[mu, l] (Q|mu nu) C_right[nu, r]
//     B[P, l*nr+r] = sum_Q M[P, Q] (Q|lr)
// with M = V^-1/2 or L^-1 of the Coulomb metric; the restatement of
// stream_dressed_mo_band (ferric-mp2/src/rimp2.rs:648-737), whose output
// B_ov (l = occupied, r = virtual) feeds the RI-MP2 path.
//
// Per chunk of aux rows Q (the reference streams the same way):
//   half      H[(q, nu)][l] = sum_mu (Q|nu mu) C_left[mu, l]     (FP64 DMMA GEMM;
//             (Q|mu nu) is symmetric in mu nu), stored as H[(q, l)][nu]
//   MO        (Q|lr) = sum_nu H[(q, l)][nu] C_right[nu, r]        (FP64 DMMA GEMM),
//             stored transposed, MOt[l*nr + r][Q], for the dressing
// then once:
//   dressing  B = M MOt^T: 2 naux^2 nl nr flops, the dominant term.  FC_PREC_F64:
//             FP64 DMMA; FC_PREC_MIXED: both operands split into exact integer
//             slices (a scale per row) and contracted on tcgen05 with the
//             k-panel FP64 flush (xgemm.cuh), so the result carries the slices'
//             ~24 significant bits per row and no accumulation error.
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

// C (n x k, row-major) -> Ct (k x n).
__global__ void dress_transpose_kernel(const double* __restrict__ c, int64_t n, int64_t k,
                                       double* __restrict__ ct) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    const int64_t r = e / k, col = e % k;
    ct[col * n + r] = c[e];
}

// half transform: value(m = q*n + nu, l) -> H[(q*nl + l)*n + nu]
struct EpiHalf {
    double* H;
    int64_t n;
    int nl;
    __device__ __forceinline__ void operator()(int m, int l, double v, int) const {
        const int64_t q = m / n, nu = m % n;
        H[((int64_t)q * nl + l) * n + nu] = v;
    }
};

// MO transform: value(m = q_local*nl + l, r) -> MOt[(l*nr + r)*ldq + q0 + q_local]
struct EpiMoT {
    double* mot;
    int64_t ldq;
    int nl, nr, q0;
    __device__ __forceinline__ void operator()(int m, int r, double v, int) const {
        const int q = m / nl, l = m % nl;
        mot[((int64_t)l * nr + r) * ldq + q0 + q] = v;
    }
};

// Row r of an FP64 matrix (pitch Kv) -> three slices [3][slice_rows][K] at
// pitch K >= Kv, scale s[r]; a non-finite element raises *bad.
__global__ void __launch_bounds__(256) dress_split_rows_kernel(const double* __restrict__ x, int64_t Kv,
                                                               int64_t K, int64_t slice_rows,
                                                               double* __restrict__ s,
                                                               __nv_bfloat16* __restrict__ xs, int* bad) {
    const int64_t r = blockIdx.x;
    bool nf = false;
    for (int64_t k = threadIdx.x; k < Kv; k += 256) nf |= !(fabs(x[r * Kv + k]) <= 1.0e300);
    if (nf) atomicOr(bad, 1);
    split_fx_qrows_body(x, 1, Kv, K, K, slice_rows, s, xs, r);
}

// out[P * ldo + w] = s_P s_w acc for the dressing GEMM (tile 128 x 128)
struct EpiDress {
    const double* sa;
    const double* sb;
    double* out;
    int64_t ldo;
    int M, N;
    __device__ void operator()(int64_t, int4 it, int row, int col0, const double (&acc)[32]) const {
        const int p = it.x * xg::BM + row;
        if (p >= M) return;
        const double s = sa[p];
        double* o = out + (int64_t)p * ldo;
#pragma unroll
        for (int c = 0; c < 32; ++c) {
            const int w = it.y * 128 + col0 + c;
            if (w < N) o[w] = s * sb[w] * acc[c];
        }
    }
};

bool g_dress_attr = false;

fc_status dress_attrs() {
    if (g_dress_attr) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiHalf>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiMoT>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(xgemm_kernel<128, EpiDress>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 xg::Cfg<128>::SMEM));
    g_dress_attr = true;
    return FC_OK;
}

}  // namespace

// eri3 is a device pointer when host == false; otherwise a host array whose
// aux chunks are copied in as they are needed.
fc_status mo_dress(const double* eri3, bool host, int64_t naux, int64_t n, const double* m, const double* c_left,
                   int64_t nl, const double* c_right, int64_t nr, int precision, double* b, cudaStream_t st,
                   size_t chunk_bytes, fc_stats* stats) {
    FC_TRY(dress_attrs());
    Context& cx = ctx();
    const int64_t width = nl * nr;
    if ((naux + DG_BM - 1) / DG_BM > 65535 || n * naux > INT32_MAX || width > INT32_MAX)
        return fail(FC_ERR_LAYOUT, "MO dressing: shape too large");
    // aux rows per chunk: the chunk's (Q|mu nu) (when copied in) and H
    int64_t qc = (int64_t)(chunk_bytes / ((size_t)n * (n + nl) * 8 + 1));
    qc = std::max<int64_t>(1, std::min<int64_t>(qc, naux));
    if (qc * n > INT32_MAX || qc * nl > INT32_MAX) qc = std::max<int64_t>(1, INT32_MAX / std::max(n, nl) / 2);
    void *vct, *vh, *vmot, *vchunk = nullptr;
    FC_TRY(ws_get(WS_MISC, (size_t)(nl + nr) * n * 8, &vct));
    FC_TRY(ws_get(WS_TS, (size_t)qc * nl * n * 8, &vh));
    FC_TRY(ws_get(WS_T, (size_t)width * naux * 8, &vmot));
    if (host) FC_TRY(ws_get(WS_SPLIT, (size_t)qc * n * n * 8, &vchunk));
    double* clt = (double*)vct;  // C_left^T (nl x n)
    double* crt = clt + nl * n;  // C_right^T (nr x n)
    double* H = (double*)vh;
    double* mot = (double*)vmot;
    if (stats) FC_CUDA(cudaEventRecord(cx.ev0, st));
    dress_transpose_kernel<<<(unsigned)((n * nl + 255) / 256), 256, 0, st>>>(c_left, n, nl, clt);
    dress_transpose_kernel<<<(unsigned)((n * nr + 255) / 256), 256, 0, st>>>(c_right, n, nr, crt);
    FC_TRY(check_launch("dress_transpose_kernel"));
    int launches = 2;
    for (int64_t q0 = 0; q0 < naux; q0 += qc) {
        const int64_t qn = std::min(qc, naux - q0);
        const double* t3 = eri3 + q0 * n * n;
        if (host) {
            FC_CUDA(cudaMemcpyAsync(vchunk, t3, (size_t)qn * n * n * 8, cudaMemcpyHostToDevice, st));
            t3 = (const double*)vchunk;
            if (stats) stats->h2d_bytes += (uint64_t)qn * n * n * 8;
        }
        {  // H[(q, nu)][l] = sum_mu (Q|nu mu) C_left[mu, l]
            const int M = (int)(qn * n);
            dim3 g((unsigned)((nl + DG_BN - 1) / DG_BN), (unsigned)((M + DG_BM - 1) / DG_BM), 1);
            EpiHalf epi{H, n, (int)nl};
            dgemm_tn_kernel<EpiHalf><<<g, 256, DG_SMEM, st>>>(t3, n, clt, n, M, (int)nl, n, n, 0, epi);
        }
        {  // (Q|lr) = sum_nu H[(q, l)][nu] C_right[nu, r] -> MOt[l*nr + r][Q]
            const int M = (int)(qn * nl);
            dim3 g((unsigned)((nr + DG_BN - 1) / DG_BN), (unsigned)((M + DG_BM - 1) / DG_BM), 1);
            EpiMoT epi{mot, naux, (int)nl, (int)nr, (int)q0};
            dgemm_tn_kernel<EpiMoT><<<g, 256, DG_SMEM, st>>>(H, n, crt, n, M, (int)nr, n, n, 0, epi);
        }
        FC_TRY(check_launch("MO transform GEMMs"));
        launches += 2;
    }
    cudaEvent_t* ev = nullptr;
    if (stats) {
        FC_TRY(timing_events(1, &ev));
        FC_CUDA(cudaEventRecord(ev[0], st));
    }
    if (precision == FC_PREC_F64) {
        // B[P][w] = sum_Q M[P][Q] MOt[w][Q]
        dim3 g((unsigned)((width + DG_BN - 1) / DG_BN), (unsigned)((naux + DG_BM - 1) / DG_BM), 1);
        if (g.x > 2147483647u) return fail(FC_ERR_LAYOUT, "MO dressing: width too large");
        EpiStore epi{b, width, 1.0, 0};
        dgemm_tn_kernel<EpiStore><<<g, 256, DG_SMEM, st>>>(m, naux, mot, naux, (int)naux, (int)width, naux, naux,
                                                            0, epi);
        FC_TRY(check_launch("dressing GEMM (FP64)"));
        launches += 1;
    } else {
        // both operands as exact slices, rows padded to 128, K = naux padded to 8
        const int64_t ldk = rup(naux, 8), mp = rup(naux, 128), np = rup(width, 128);
        void *vms, *vws, *vsc, *vflag, *vtab;
        FC_TRY(ws_get(WS_SPLIT2, (size_t)3 * (mp + np) * ldk * 2, &vms));
        vws = (char*)vms + (size_t)3 * mp * ldk * 2;
        FC_TRY(ws_get(WS_SCALE, (size_t)(mp + np) * 8, &vsc));
        FC_TRY(ws_get(WS_OUT, 256, &vflag));
        int* flags = (int*)vflag;
        double* sa = (double*)vsc;
        double* sb = sa + mp;
        FC_CUDA(cudaMemsetAsync(vflag, 0, 256, st));
        // rows of M and of MOt (pitch naux) -> slices at pitch ldk; the tensor
        // maps' inner extent is naux, so the TMA zero-fills the K tail, and
        // padding rows only reach masked outputs
        dress_split_rows_kernel<<<(unsigned)naux, 256, 0, st>>>(m, naux, ldk, mp, sa, (__nv_bfloat16*)vms, flags);
        dress_split_rows_kernel<<<(unsigned)width, 256, 0, st>>>(mot, naux, ldk, np, sb, (__nv_bfloat16*)vws,
                                                                 flags);
        FC_TRY(check_launch("dressing splits"));
        std::vector<int4> items;
        const int ntm = (int)(mp / 128), ntn = (int)(np / 128), nks = (int)((naux + 63) / 64);
        for (int tn = 0; tn < ntn; ++tn)
            for (int tm = 0; tm < ntm; ++tm) items.push_back(make_int4(tm, tn, 0, nks));
        FC_TRY(ws_get(WS_PAIRS, items.size() * sizeof(int4), &vtab));
        FC_CUDA(cudaMemcpyAsync(vtab, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
        CUtensorMap ta, tb;
        FC_TRY(make_tmap_bf16_2d(&ta, vms, naux, 3 * mp, ldk * 2, 64, 128));
        FC_TRY(make_tmap_bf16_2d(&tb, vws, naux, 3 * np, ldk * 2, 64, 128));
        XArgs a{(const int4*)vtab, (int64_t)items.size(), (int)mp, (int)np, flags + 1};
        EpiDress epi{sa, sb, b, width, (int)naux, (int)width};
        const int grid = (int)std::min<int64_t>((int64_t)items.size(), cx.sm_count);
        xgemm_kernel<128, EpiDress><<<grid, xg::Cfg<128>::THREADS, xg::Cfg<128>::SMEM, st>>>(ta, tb, a, epi);
        FC_TRY(check_launch("dressing GEMM (exact slices)"));
        launches += 3;
        int hf[2];
        FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
        FC_CUDA(cudaStreamSynchronize(st));
        if (hf[0]) return fail(FC_ERR_RANGE, "MO dressing: a non-finite element in M or the MO tensor");
        if (hf[1]) return fail(FC_ERR_TIMEOUT, "MO dressing: a pipeline wait ran out");
    }
    if (stats) {
        FC_CUDA(cudaEventRecord(ev[1], st));
        FC_CUDA(cudaEventRecord(cx.ev1, st));
        FC_CUDA(cudaEventSynchronize(cx.ev1));
        float ms = 0.f, m4 = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, cx.ev0, cx.ev1));
        FC_CUDA(cudaEventElapsedTime(&m4, ev[0], ev[1]));
        stats->kernel_ms = ms;
        stats->flops = 2.0 * naux * (double)n * n * nl + 2.0 * naux * (double)nl * n * nr +
                       2.0 * (double)naux * naux * width;
        stats->precision = precision == FC_PREC_F64 ? FC_PREC_F64 : FC_PREC_MIXED;
        stats->launches += launches;
        stats->tile_m = 128;
        stats->tile_n = precision == FC_PREC_F64 ? DG_BN : 128;
        stats->k_panel = precision == FC_PREC_F64 ? 0 : xg::KP * xg::KT;
        stats->main_launches = 1;
        stats->main_ms = m4;
        stats->main_flops = 2.0 * (double)naux * naux * width;
        stats->main_bytes = 8.0 * ((double)naux * naux + 2.0 * (double)naux * width);
    }
    return FC_OK;
}

}  // namespace fc

using namespace fc;

namespace {

fc_status dress_common(const double* eri3, bool host, int64_t naux, int64_t n, const double* m, const double* cl,
                       int64_t nl, const double* cr, int64_t nr, int32_t precision, double* b, void* stream,
                       fc_stats* stats) {
    if (!eri3 || !m || !cl || !cr || !b) return fail(FC_ERR_INVALID, "fc_mo_dress: null argument");
    if (naux <= 0 || n <= 0 || nl <= 0 || nr <= 0) return fail(FC_ERR_LAYOUT, "fc_mo_dress: sizes must be > 0");
    if (precision != FC_PREC_F64 && precision != FC_PREC_MIXED)
        return fail(FC_ERR_INVALID, "fc_mo_dress: precision is FC_PREC_F64 or FC_PREC_MIXED");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    Context& c = ctx();
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    const int64_t width = nl * nr;
    if (!host) return mo_dress(eri3, false, naux, n, m, cl, nl, cr, nr, precision, b, st, (size_t)1 << 30, stats);
    // host arrays: M, C in; B out (eri3 copied chunk by chunk)
    void *vm, *vc, *vb;
    FC_TRY(ws_get(WS_EPS, (size_t)(naux * naux + n * (nl + nr)) * 8, &vm));
    vc = (double*)vm + naux * naux;
    FC_TRY(ws_get(WS_GAMMA, (size_t)naux * width * 8, &vb));
    FC_CUDA(cudaMemcpyAsync(vm, m, (size_t)naux * naux * 8, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync(vc, cl, (size_t)n * nl * 8, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync((double*)vc + n * nl, cr, (size_t)n * nr * 8, cudaMemcpyHostToDevice, st));
    FC_TRY(mo_dress(eri3, true, naux, n, (const double*)vm, (const double*)vc, nl, (const double*)vc + n * nl, nr,
                    precision, (double*)vb, st, (size_t)1 << 30, stats));
    FC_CUDA(cudaMemcpyAsync(b, vb, (size_t)naux * width * 8, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes += (uint64_t)(naux * naux + n * (nl + nr)) * 8;
        stats->d2h_bytes += (uint64_t)naux * width * 8;
    }
    return FC_OK;
}

}  // namespace

extern "C" {

fc_status fc_mo_dress(const double* eri3, int64_t naux, int64_t n, const double* m, const double* c_left,
                      int64_t nleft, const double* c_right, int64_t nright, int32_t precision, double* b,
                      fc_stats* stats) {
    return dress_common(eri3, true, naux, n, m, c_left, nleft, c_right, nright, precision, b, nullptr, stats);
}

fc_status fc_mo_dress_dev(const double* eri3, int64_t naux, int64_t n, const double* m, const double* c_left,
                          int64_t nleft, const double* c_right, int64_t nright, int32_t precision, double* b,
                          void* stream, fc_stats* stats) {
    return dress_common(eri3, false, naux, n, m, c_left, nleft, c_right, nright, precision, b, stream, stats);
}

}  // extern "C"
