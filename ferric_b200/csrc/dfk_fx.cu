// Exact-slice DF-K (FC_PREC_MIXED) on the tcgen05 GEMM.
//
// K = sum_Q (B_Q C)(B_Q C)^T for C = C_occ (n x nocc), no occupation factor
// (KBuilder::build_from_occ, ferric-scf/src/fock.rs:22-52; the occupied
// path of ferric-scf/src/df_k.rs:1409-1520, 1575-1660):
//   once per handle  B rows (Q, mu) split into three int8 integer slices at a
//                    power-of-two scale per row (fx_split.cuh): 3 bytes per
//                    element, the bytes of the HBM-bound stage 1, stored in
//                    128-byte column blocks so each k-step's box is
//                    contiguous
//   per build        C^T rows (one per occupied orbital) split the same way
//   stage 1          W[mu, (Q, i)] = sum_nu B[Q, mu, nu] C[nu, i]: int8
//                    exact-slice GEMM (kind::i8, exact int32 levels),
//                    128 x 64 tiles over the naux*n rows of B (each B slice
//                    read once), FP32 W
//   split            rows mu of W, three slices at a scale per row
//   stage 2          K = W W^T: upper 128 x 128 tiles, split over (Q, i) into
//                    about one item per SM, k-panel flush into FP64 registers
//                    (xgemm.cuh), FP64 partial tiles
//   fold             K[mu, nu] = K[nu, mu] = fixed-order sum of the partials
//                    of the upper element (the final FP64 symmetrisation)
// Results are deterministic and exactly symmetric.  Error: the slices carry
// about 24 significant bits of each row; W is rounded to FP32 once.
#include <algorithm>
#include <vector>

#include "dfjk.cuh"
#include "fx_split.cuh"
#include "tmap.cuh"
#include "xgemm.cuh"

namespace fc {

namespace {

int64_t rup(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Row r = (Q, mu) of the square tensor -> int8 slices in k-blocks:
// [3][nkb][rows][128] (column nu of row r at block nu / 128, byte nu % 128;
// zero past n), scale s[r].  Stage 1 reads one 128-byte column block of 128
// rows per k-step: contiguous 16 KB, not 128 bytes of each row at the row
// pitch (DRAM pages stay open along a k-step's box).
__global__ void __launch_bounds__(256) dfk_split_b_kblk_kernel(const double* __restrict__ b, int64_t n,
                                                               int64_t nkb, int64_t rows, double* __restrict__ s,
                                                               int8_t* __restrict__ bs) {
    __shared__ double red[32];
    const int64_t r = blockIdx.x;
    const double* row = b + r * n;
    double m = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += 256) m = fmax(m, fabs(row[k]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double sc = SliceI8::scale(red[0]);
    if (threadIdx.x == 0) s[r] = sc;
    const double inv = 1.0 / sc;
    const int64_t ss = nkb * rows * 128;  // bytes between slices
    for (int64_t k = threadIdx.x; k < nkb * 128; k += 256) {
        int8_t c1 = 0, c2 = 0, c3 = 0;
        if (k < n) fx_slices<SliceI8>(row[k], inv, c1, c2, c3);
        const int64_t d = ((k >> 7) * rows + r) * 128 + (k & 127);
        bs[d] = c1;
        bs[ss + d] = c2;
        bs[2 * ss + d] = c3;
    }
}

// Column i of C (n x nocc) -> row i of the int8 C^T slices [3][npad][ldk], scale sc[i].
__global__ void __launch_bounds__(256) dfk_split_c_kernel(const double* __restrict__ c, int64_t n, int64_t nocc,
                                                          int64_t ldk, int64_t npad, double* __restrict__ sc,
                                                          int8_t* __restrict__ cs, int* bad) {
    __shared__ double red[32];
    const int64_t i = blockIdx.x;
    double m = 0.0;
    bool nf = false;
    for (int64_t nu = threadIdx.x; nu < n; nu += 256) {
        const double v = fabs(c[nu * nocc + i]);
        nf |= !(v <= 1.0e300);
        m = fmax(m, v);
    }
    if (nf) atomicOr(bad, 1);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double s = SliceI8::scale(red[0]);
    if (threadIdx.x == 0) sc[i] = s;
    const double inv = 1.0 / s;
    const int64_t ss = npad * ldk;
    for (int64_t nu = threadIdx.x; nu < n; nu += 256) {
        int8_t c1, c2, c3;
        fx_slices<SliceI8>(c[nu * nocc + i], inv, c1, c2, c3);
        cs[i * ldk + nu] = c1;
        cs[ss + i * ldk + nu] = c2;
        cs[2 * ss + i * ldk + nu] = c3;
    }
}

// Row mu of the FP32 W -> int8 slices [3][mp][ldw] at the row scale sw[mu],
// from the row maximum the stage-1 epilogue gathered, so W is read once.
// blockIdx.y cuts the row into gridDim.y column ranges (more CTAs in flight).
__global__ void __launch_bounds__(256) dfk_split_w_kernel(const float* __restrict__ w, int64_t ldw, int64_t mp,
                                                          double* __restrict__ sw, int8_t* __restrict__ ws,
                                                          const unsigned* __restrict__ wmax) {
    const int64_t mu = blockIdx.x;
    const double s = SliceI8::scale((double)__uint_as_float(wmax[mu]));
    if (blockIdx.y == 0 && threadIdx.x == 0) sw[mu] = s;
    const double inv = 1.0 / s;
    const int64_t k4 = ldw / 4, per = (k4 + gridDim.y - 1) / gridDim.y;
    const int64_t k0 = blockIdx.y * per, k1 = k0 + per < k4 ? k0 + per : k4;
    const float4* row = reinterpret_cast<const float4*>(w + mu * ldw);
    const int64_t ss = mp * ldw;
    int8_t* o0 = ws + mu * ldw;
    struct alignas(4) Q4 { int8_t e[4]; };
    for (int64_t k = k0 + threadIdx.x; k < k1; k += 256) {
        const float4 v = row[k];
        Q4 pa, pb, pc;
        fx_slices<SliceI8>(v.x, inv, pa.e[0], pb.e[0], pc.e[0]);
        fx_slices<SliceI8>(v.y, inv, pa.e[1], pb.e[1], pc.e[1]);
        fx_slices<SliceI8>(v.z, inv, pa.e[2], pb.e[2], pc.e[2]);
        fx_slices<SliceI8>(v.w, inv, pa.e[3], pb.e[3], pc.e[3]);
        reinterpret_cast<Q4*>(o0)[k] = pa;
        reinterpret_cast<Q4*>(o0 + ss)[k] = pb;
        reinterpret_cast<Q4*>(o0 + 2 * ss)[k] = pc;
    }
}

// Stage 1 store: row r = (Q, mu) of B, column i: W[mu * ldw + Q * nocc_p + i].
// Also, per thread, the max |W| of its values (atomicMax into wmax[mu]: the
// order-free maximum of non-negative FP32 bits), so W's split reads W once.
struct EpiW {
    const double* sa;  // [naux*n] B row scales
    const double* sc;  // [npad] C^T row scales
    float* w;
    int64_t ldw, rows;
    int n, nocc, nocc_p;
    unsigned* wmax;     // [n]
    __device__ void operator()(int64_t, int4 it, int row, int col0, const double (&acc)[32]) const {
        const int64_t r = (int64_t)it.x * xg::BM + row;
        if (r >= rows) return;
        const int64_t q = r / n, mu = r % n;
        const int i0 = it.y * 64 + col0;
        if (i0 >= nocc_p) return;
        const double s = sa[r];
        float* dst = w + mu * ldw + q * nocc_p + i0;
        float m = 0.f;
#pragma unroll
        for (int c4 = 0; c4 < 32; c4 += 4) {
            if (i0 + c4 >= nocc_p) break;  // nocc_p is a multiple of 16
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int i = i0 + c4 + e;
                v[e] = i < nocc ? (float)(s * sc[i] * acc[c4 + e]) : 0.f;
                m = fmaxf(m, fabsf(v[e]));
            }
            *reinterpret_cast<float4*>(dst + c4) = make_float4(v[0], v[1], v[2], v[3]);
        }
        atomicMax(wmax + mu, __float_as_uint(m));
    }
};

// Stage 2 store: the item's FP64 partial tile [128][128], zero outside n x n.
struct EpiPart {
    const double* sw;  // [mp] W row scales
    double* part;
    int n;
    __device__ void operator()(int64_t t, int4 it, int row, int col0, const double (&acc)[32]) const {
        const int mu = it.x * xg::BM + row;
        double* dst = part + t * (xg::BM * 128) + row * 128 + col0;
        const double smu = mu < n ? sw[mu] : 0.0;
#pragma unroll
        for (int c2 = 0; c2 < 32; c2 += 2) {
            const int nu = it.y * 128 + col0 + c2;
            const double v0 = (mu < n && nu < n) ? smu * sw[nu] * acc[c2] : 0.0;
            const double v1 = (mu < n && nu + 1 < n) ? smu * sw[nu + 1] * acc[c2 + 1] : 0.0;
            *reinterpret_cast<double2*>(dst + c2) = make_double2(v0, v1);
        }
    }
};

// K[mu, nu] = K[nu, mu] = sum over the splits (in order) of the upper element.
__global__ void __launch_bounds__(256) dfk_fold_fx_kernel(const double* __restrict__ part,
                                                          const int* __restrict__ tix, int nsplit, int nt,
                                                          int64_t n, double* __restrict__ k) {
    const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (e >= n * n) return;
    const int64_t r = e / n, c = e % n;
    const int64_t lo = r < c ? r : c, hi = r < c ? c : r;
    const int tm = (int)(lo / 128), tn = (int)(hi / 128);
    const int64_t base = (int64_t)tix[tm * nt + tn] * nsplit;
    const int64_t off = (lo % 128) * 128 + (hi % 128);
    double s = 0.0;
    for (int sp = 0; sp < nsplit; ++sp) s += part[(base + sp) * (128 * 128) + off];
    k[e] = s;
}

bool g_attr_done = false;

fc_status xg_attrs() {
    if (g_attr_done) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(xgemm_kernel<64, EpiW, true, LdKBlocksA>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, xg::Cfg<64, true>::SMEM));
    FC_CUDA(cudaFuncSetAttribute(xgemm_kernel<128, EpiPart, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 xg::Cfg<128, true>::SMEM));
    g_attr_done = true;
    return FC_OK;
}

}  // namespace

// Split of the square tensor for the tensor-core stages (mixed square
// handles): three int8 slices per row (Q, mu) in 128-byte column blocks.
fc_status dfk_prepare_split(fc_dfjk* h, cudaStream_t st) {
    const int64_t rows = h->naux * h->n, nkb = (h->n + 127) / 128;
    const size_t sbytes = (size_t)3 * nkb * rows * 128, scl = (size_t)rows * 8;
    const size_t bytes = rup((int64_t)sbytes, 256) + scl;
    if (rows > INT32_MAX || 3 * nkb * rows > INT32_MAX) return fail(FC_ERR_LAYOUT, "DF-K: naux*n too large");
    FC_TRY(pool_reserve(bytes));
    FC_CUDA(cudaMalloc(&h->sq_split, bytes));
    h->bytes += bytes;
    h->sq_scale = (double*)((char*)h->sq_split + rup((int64_t)sbytes, 256));
    dfk_split_b_kblk_kernel<<<(unsigned)rows, 256, 0, st>>>(h->b_sq, h->n, nkb, rows, h->sq_scale,
                                                            (int8_t*)h->sq_split);
    return check_launch("dfk_split_b_kblk_kernel");
}

fc_status dfk_build_mixed(fc_dfjk* h, const double* c_occ, int64_t nocc, double* kout, cudaStream_t st,
                          fc_stats* stats, const JFork* jf) {
    if (!h->sq_split)
        return fail(FC_ERR_KERNEL, "DF-K: handle has no int8 slice copy (created with FC_PREC_F64)");
    FC_TRY(xg_attrs());
    Context& cx = ctx();
    const int64_t n = h->n, naux = h->naux, ldk = rup(n, 16);
    const int64_t rows = naux * n;
    // nocc_p a multiple of 16: W's rows (ldw = naux nocc_p bytes as int8 slices) stay 16-byte aligned
    const int64_t nocc_p = rup(nocc, 16), npad = rup(nocc, 64), ldw = naux * nocc_p, mp = rup(n, 128);

    if (rows > INT32_MAX || 3 * rows > (int64_t)UINT32_MAX || mp > 65536 || ldw > INT32_MAX)
        return fail(FC_ERR_LAYOUT, "DF-K mixed: shape too large");
    // stage-1 and stage-2 work items
    std::vector<int4> items;
    const int ntm1 = (int)((rows + 127) / 128), ntn1 = (int)(npad / 64), nks1 = (int)((n + 127) / 128);
    for (int tm = 0; tm < ntm1; ++tm)
        for (int tn = 0; tn < ntn1; ++tn) items.push_back(make_int4(tm, tn, 0, nks1));
    const int64_t n1 = (int64_t)items.size();
    const int nt = (int)(mp / 128);
    const int ntile = nt * (nt + 1) / 2;
    const int nks2 = (int)((ldw + 127) / 128);  // k-steps of 128 int8
    int want = std::max(1, cx.sm_count / ntile);
    const int kps = (nks2 + want - 1) / want;
    const int nsplit = (nks2 + kps - 1) / kps;
    std::vector<int> tix((size_t)nt * nt, 0);
    int tcount = 0;
    for (int tm = 0; tm < nt; ++tm)
        for (int tn = tm; tn < nt; ++tn) {
            tix[tm * nt + tn] = tcount++;
            for (int sp = 0; sp < nsplit; ++sp) {
                const int k0 = sp * kps;
                items.push_back(make_int4(tm, tn, k0, std::min(kps, nks2 - k0)));
            }
        }
    const int64_t n2 = (int64_t)items.size() - n1;

    void *vc, *vout, *vw, *vws, *vsw, *vpart, *vtab;
    const size_t cs_bytes = (size_t)3 * npad * ldk;
    FC_TRY(ws_get(WS_MISC, rup((int64_t)cs_bytes, 256) + npad * 8, &vc));
    FC_TRY(ws_get(WS_OUT, 256, &vout));
    FC_TRY(ws_get(WS_T, (size_t)n * ldw * 4, &vw));
    FC_TRY(ws_get(WS_TS, (size_t)3 * mp * ldw, &vws));
    FC_TRY(ws_get(WS_SCALE, (size_t)mp * 8 + (size_t)rup(n, 64) * 4, &vsw));
    unsigned* wmax = (unsigned*)((double*)vsw + mp);  // [n] row maxima of |W| (FP32 bits)

    FC_TRY(ws_get(WS_PART, (size_t)n2 * 128 * 128 * 8, &vpart));
    FC_TRY(ws_get(WS_PAIRS, items.size() * sizeof(int4) + tix.size() * sizeof(int), &vtab));
    int* flags = (int*)vout;  // [0] range, [1] timeout
    double* sc = (double*)((char*)vc + rup((int64_t)cs_bytes, 256));
    FC_CUDA(cudaMemcpyAsync(vtab, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    int* dtix = (int*)((int4*)vtab + items.size());
    FC_CUDA(cudaMemcpyAsync(dtix, tix.data(), tix.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemsetAsync(vout, 0, 256, st));
    FC_CUDA(cudaMemsetAsync(vc, 0, cs_bytes, st));

    CUtensorMap tb, tcm, tw;
    const int64_t nkb = (n + 127) / 128;  // k-blocks of the B slices
    FC_TRY(make_tmap_i8_2d(&tb, h->sq_split, 128, 3 * nkb * rows, 128, 128, 128));
    FC_TRY(make_tmap_i8_2d(&tcm, vc, n, 3 * npad, ldk, 128, 64));
    FC_TRY(make_tmap_i8_2d(&tw, vws, ldw, 3 * mp, ldw, 128, 128));

    if (stats) FC_CUDA(cudaEventRecord(cx.ev0, st));
    FC_CUDA(cudaMemsetAsync(wmax, 0, (size_t)n * 4, st));
    dfk_split_c_kernel<<<(unsigned)nocc, 256, 0, st>>>(c_occ, n, nocc, ldk, npad, sc, (int8_t*)vc, flags);
    cudaEvent_t* ev = nullptr;
    if (stats) {
        FC_TRY(timing_events(2, &ev));
        FC_CUDA(cudaEventRecord(ev[0], st));
    }
    {
        XArgs a{(const int4*)vtab, n1, (int)rows, (int)npad, flags + 1, (int)nkb};
        EpiW epi{h->sq_scale, sc, (float*)vw, ldw, rows, (int)n, (int)nocc, (int)nocc_p, wmax};
        const int grid = (int)std::min<int64_t>(n1, cx.sm_count);
        xgemm_kernel<64, EpiW, true, LdKBlocksA>
            <<<grid, xg::Cfg<64, true>::THREADS, xg::Cfg<64, true>::SMEM, st>>>(tb, tcm, a, epi);
    }
    if (stats) FC_CUDA(cudaEventRecord(ev[1], st));
    if (jf) {  // J: pass-1 vector from the FP32 W (each element rounded once), second pass forked off
        const int64_t dq = dfj_d_rows(nocc, 4);  // nocc_p: a multiple of 16 floats
        dfj_d_from_w_kernel<float, 4><<<dim3((unsigned)((naux + dq - 1) / dq), DFJ_DY), 256, 0, st>>>(
            (const float*)vw, ldw, nocc_p, n, nocc, naux, dq, c_occ, jf->dpart);
        dfj_d_sum_kernel<<<(unsigned)((naux + 255) / 256), 256, 0, st>>>(jf->dpart, naux, jf->dp);
        FC_TRY(dfj_fork_pass2(h, *jf, st));
    }
    dfk_split_w_kernel<<<dim3((unsigned)n, 4), 256, 0, st>>>((const float*)vw, ldw, mp, (double*)vsw, (int8_t*)vws,
                                                              wmax);
    if (stats) FC_CUDA(cudaEventRecord(ev[2], st));
    {
        XArgs a{(const int4*)vtab + n1, n2, (int)mp, (int)mp, flags + 1};
        EpiPart epi{(const double*)vsw, (double*)vpart, (int)n};
        const int grid = (int)std::min<int64_t>(n2, cx.sm_count);
        xgemm_kernel<128, EpiPart, true><<<grid, xg::Cfg<128, true>::THREADS, xg::Cfg<128, true>::SMEM, st>>>(
            tw, tw, a, epi);
    }
    if (stats) FC_CUDA(cudaEventRecord(ev[3], st));
    dfk_fold_fx_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, st>>>((const double*)vpart, dtix, nsplit, nt, n,
                                                                         kout);
    FC_TRY(check_launch("exact-slice DF-K kernels"));
    if (jf) {  // join J's second pass
        FC_CUDA(cudaEventRecord(cx.join, cx.side));
        FC_CUDA(cudaStreamWaitEvent(st, cx.join, 0));
    }
    if (stats) FC_CUDA(cudaEventRecord(cx.ev1, st));
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "split-BF16 DF-K: C_occ has a non-finite element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "split-BF16 DF-K: a pipeline wait ran out");
    if (stats) {
        float ms = 0.f, m1 = 0.f, m2 = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, cx.ev0, cx.ev1));
        FC_CUDA(cudaEventElapsedTime(&m1, ev[0], ev[1]));
        FC_CUDA(cudaEventElapsedTime(&m2, ev[2], ev[3]));
        stats->kernel_ms = ms;
        stats->flops = 4.0 * (double)naux * (double)n * (double)n * (double)nocc;
        stats->precision = FC_PREC_MIXED;
        stats->launches += 5;
        stats->tile_m = 128;
        stats->tile_n = 64;
        stats->k_panel = xg::KP * xg::KT;
        stats->main_launches = 2;
        stats->main_ms = (double)m1 + (double)m2;
        stats->main_flops = stats->flops;
        stats->main_bytes = 3.0 * (double)rows * (double)n;  // the int8 B slices, read once
        stats->h2d_bytes += items.size() * sizeof(int4) + tix.size() * sizeof(int);
        stats->d2h_bytes += sizeof(hf);
    }
    return FC_OK;
}

}  // namespace fc
