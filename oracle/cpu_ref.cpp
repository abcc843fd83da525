// CPU restatement of the reference's host algorithms for the timed CPU
// baseline (TEST INFRASTRUCTURE: the oracle's C++ arm, never the product).
//
// g++ -O3 with OpenMP over independent work units and OpenBLAS at one thread
// inside each unit, the reference's own threading (rayon over occupied i,
// BLAS single-threaded inside: ferric-mp2/src/rimp2.rs:1471-1486):
//
//  * RI-MP2 energy + adjoint (cr_rimp2_units).  A unit is (i, j0, j1): the
//    block G = B_i^T B_J over j in [j0, j1) (one BLAS3 product, the
//    per-i G_i = B_i^T B_tail of rimp2.rs:1473-1474 cut into column blocks),
//    the pair terms for j >= i with weights 1 (i == j) and 2 (rimp2.rs:
//    1399-1441), the weighted amplitudes Tt_ij = (2 g - g^T) / D (tt_block,
//    ferric-mp2/src/zvector.rs:651-703), the adjoint x_ov[:, i] += B_J Tt^T
//    (build_x_ov_weighted, zvector.rs:651-703; Gamma = 4 x_ov, rimp2.rs:
//    1832-1836), and the t Tt sums of dE/deps (oo_rimp2.rs:1170-1191).  The
//    units of one i cover all j, so the amplitudes are recomputed, never
//    stored (t2 is nov^2 doubles).
//  * DF-J (cr_dfj): packed density weights, pass 1 d_P = Bp w over aux-row
//    chunks, pass 2 J = Bp^T c over packed-column chunks
//    (ferric-scf/src/df_j.rs:1134-1150, 1199-1245); the metric is the
//    identity for a dressed tensor.
//  * DF-K (cr_dfk): per aux row M_Q = B_Q C (DSYMM, B_Q symmetric) and one
//    DSYRK K += W W^T per aux chunk, chunks folded in order
//    (occ_chunk_k / occ_half_panel, ferric-scf/src/df_k.rs:1575-1660).
//
// BLAS is numpy's OpenBLAS (scipy_openblas64: 64-bit integers, prefixed
// symbols), linked by oracle/build_cpu_ref.py.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" {
// CBLAS of scipy_openblas64 (enums as int: RowMajor 101, NoTrans 111, Trans 112,
// Upper 121, Lower 122, Left 141)
void scipy_cblas_dgemm64_(int order, int ta, int tb, int64_t m, int64_t n, int64_t k, double alpha,
                          const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c,
                          int64_t ldc);
void scipy_cblas_dgemv64_(int order, int ta, int64_t m, int64_t n, double alpha, const double* a, int64_t lda,
                          const double* x, int64_t incx, double beta, double* y, int64_t incy);
void scipy_cblas_dsymm64_(int order, int side, int uplo, int64_t m, int64_t n, double alpha, const double* a,
                          int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc);
void scipy_cblas_dsyrk64_(int order, int uplo, int trans, int64_t n, int64_t k, double alpha, const double* a,
                          int64_t lda, double beta, double* c, int64_t ldc);
void scipy_openblas_set_num_threads64_(int n);
}

namespace {
constexpr int ROW = 101, NT = 111, TR = 112, LO = 122, LEFT = 141;

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

extern "C" {

// Units (i, j0, j1) of the RI-MP2 energy + adjoint, OpenMP over units.
//   b: (naux, nocc*nvir) row-major, eo[nocc], ev[nvir].
//   e_out[2 * u]: (E_os, E_ss) of unit u's pairs with j >= i (weights 1 / 2);
//   x_out (optional, naux x nocc*nvir, zeroed by the caller): x_ov of every
//   unit added in (units of one i must not run concurrently when it is given);
//   occ_out[u] (optional): sum of t Tt over the unit's ordered pairs (i, j).
// Returns the wall seconds of the parallel region.
double cr_rimp2_units(const double* b, int64_t naux, int64_t nocc, int64_t nvir, const double* eo,
                      const double* ev, const int64_t* units, int64_t nunits, int nthreads, double* e_out,
                      double* x_out, double* occ_out) {
    scipy_openblas_set_num_threads64_(1);
    const int64_t nov = nocc * nvir;
    const double t0 = now();
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> g, tt, x((size_t)naux * nvir);
#pragma omp for schedule(dynamic, 1)
        for (int64_t u = 0; u < nunits; ++u) {
            const int64_t i = units[3 * u], j0 = units[3 * u + 1], j1 = units[3 * u + 2];
            const int64_t w = (j1 - j0) * nvir;
            g.resize((size_t)nvir * w);
            tt.resize((size_t)nvir * w);
            // G[a, (j, b)] = sum_Q B[Q, ia] B[Q, jb]
            scipy_cblas_dgemm64_(ROW, TR, NT, nvir, w, naux, 1.0, b + i * nvir, nov, b + j0 * nvir, nov, 0.0,
                                 g.data(), w);
            double e_os = 0.0, e_ss = 0.0, occ = 0.0;
            for (int64_t j = j0; j < j1; ++j) {
                const double wt = j == i ? 1.0 : 2.0;
                const int64_t off = (j - j0) * nvir;
                double po = 0.0, ps = 0.0;
                for (int64_t a = 0; a < nvir; ++a) {
                    const double* ga = g.data() + a * w + off;
                    double* ta = tt.data() + a * w + off;
                    const double da = eo[i] + eo[j] - ev[a];
                    for (int64_t bb = 0; bb < nvir; ++bb) {
                        const double x1 = ga[bb];                     // (ia|jb)
                        const double x2 = g[bb * w + off + a];        // (ib|ja)
                        const double r = 1.0 / (da - ev[bb]);
                        po += x1 * x1 * r;
                        ps += x1 * (x1 - x2) * r;
                        const double t = (2.0 * x1 - x2) * r;
                        ta[bb] = t;
                        occ += x1 * r * t;
                    }
                }
                if (j >= i) {
                    e_os += wt * po;
                    e_ss += wt * ps;
                }
            }
            // x[Q, a] = sum_{(j, b)} B[Q, jb] Tt[a, (j, b)]
            scipy_cblas_dgemm64_(ROW, NT, TR, naux, nvir, w, 1.0, b + j0 * nvir, nov, tt.data(), w, 0.0, x.data(),
                                 nvir);
            if (x_out) {
                for (int64_t q = 0; q < naux; ++q) {
                    double* dst = x_out + q * nov + i * nvir;
                    const double* src = x.data() + q * nvir;
                    for (int64_t a = 0; a < nvir; ++a) dst[a] += src[a];
                }
            }
            e_out[2 * u] = e_os;
            e_out[2 * u + 1] = e_ss;
            if (occ_out) occ_out[u] = occ;
        }
    }
    return now() - t0;
}

// DF-J on packed rows bp (naux, npair): J_packed = Bp^T (Bp w), chunks of
// rows (pass 1) and of packed columns (pass 2) over the threads, folded in
// order.  Returns the wall seconds.
double cr_dfj(const double* bp, int64_t naux, int64_t npair, const double* w, double* j_packed, int nthreads) {
    scipy_openblas_set_num_threads64_(1);
    const double t0 = now();
    std::vector<double> d((size_t)naux);
    const int64_t rc = std::max<int64_t>(1, (naux + 4 * nthreads - 1) / (4 * nthreads));
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int64_t p0 = 0; p0 < naux; p0 += rc) {
        const int64_t np = std::min(rc, naux - p0);
        scipy_cblas_dgemv64_(ROW, NT, np, npair, 1.0, bp + p0 * npair, npair, w, 1, 0.0, d.data() + p0, 1);
    }
    const int64_t cc = std::max<int64_t>(64, (npair + 4 * nthreads - 1) / (4 * nthreads));
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int64_t k0 = 0; k0 < npair; k0 += cc) {
        const int64_t nk = std::min(cc, npair - k0);
        scipy_cblas_dgemv64_(ROW, TR, naux, nk, 1.0, bp + k0, npair, d.data(), 1, 0.0, j_packed + k0, 1);
    }
    return now() - t0;
}

// DF-K occupied path on the square dressed tensor b (naux, n, n):
// K = sum_Q (B_Q C)(B_Q C)^T, one DSYMM per aux row and one DSYRK per chunk
// of qc rows, chunk results folded in chunk order.  k: (n, n), full
// (symmetrised).  Returns the wall seconds.
double cr_dfk(const double* b, int64_t naux, int64_t n, const double* c, int64_t nocc, int64_t qc, double* k,
              int nthreads) {
    scipy_openblas_set_num_threads64_(1);
    const double t0 = now();
    const int64_t nch = (naux + qc - 1) / qc;
    std::vector<std::vector<double>> kc((size_t)nch);
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> wq((size_t)n * qc * nocc);
#pragma omp for schedule(dynamic, 1)
        for (int64_t ch = 0; ch < nch; ++ch) {
            const int64_t q0 = ch * qc, nq = std::min(qc, naux - q0);
            // W[mu, (Q, i)] = (B_Q C)[mu, i]
            for (int64_t q = 0; q < nq; ++q)
                scipy_cblas_dsymm64_(ROW, LEFT, LO, n, nocc, 1.0, b + (q0 + q) * n * n, n, c, nocc, 0.0,
                                     wq.data() + q * nocc, qc * nocc);
            kc[(size_t)ch].assign((size_t)n * n, 0.0);
            scipy_cblas_dsyrk64_(ROW, LO, NT, n, nq * nocc, 1.0, wq.data(), qc * nocc, 0.0, kc[(size_t)ch].data(),
                                 n);
        }
    }
    std::fill(k, k + n * n, 0.0);
    for (int64_t ch = 0; ch < nch; ++ch)
        for (int64_t r = 0; r < n; ++r)
            for (int64_t s = 0; s <= r; ++s) k[r * n + s] += kc[(size_t)ch][r * n + s];
    for (int64_t r = 0; r < n; ++r)
        for (int64_t s = 0; s < r; ++s) k[s * n + r] = k[r * n + s];
    return now() - t0;
}

}  // extern "C"
