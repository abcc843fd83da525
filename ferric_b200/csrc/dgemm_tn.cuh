// All-FP64 tile GEMM on the DMMA tensor path:
//     value(m, n) = sum_{k in split} A(m, k) * B(n, k)
// with each operand K-major (row-major M x K and N x K, the default "TN"
// form) or, with TA / TB, MN-major (stored K x M / K x N), and a functor
// epilogue, so one kernel serves the gradient's second contraction
// (Gamma = 4 B_ov Tt^T), the DF-K half-transform and rank update, the MP2
// densities and the RI response products.
//
// Tile 128 x 64 x 16, 8 warps (4 x 2), each warp 32 x 32 = 4 x 4 DMMA tiles;
// 3-stage cp.async pipeline; split-K over blockIdx.z.  Shared-memory rows are
// padded to 20 doubles so the fragment reads (g*20 + t) hit distinct banks.
#pragma once
#include "dmma.cuh"

namespace fc {

constexpr int DG_BM = 128, DG_BN = 64, DG_BK = 16, DG_LDK = 20, DG_STAGES = 3;
constexpr int DG_SMEM = DG_STAGES * (DG_BM + DG_BN) * DG_LDK * 8;

// The tile body.  A(m, k) = TA ? A[k*lda + m] : A[m*lda + k], and B(n, k) the
// same with TB: a transposed (MN-major) operand is read with consecutive
// threads on consecutive m (n), so its global loads stay coalesced.  The
// epilogue gets `z` (the split or the batch index).
template <class Epi, bool TA, bool TB>
__device__ __forceinline__ void dgemm_tile(const double* __restrict__ A, int64_t lda, const double* __restrict__ B,
                                           int64_t ldb, int M, int N, int64_t kbeg, int64_t kend, int upper_only,
                                           const Epi& epi, int z) {
    extern __shared__ __align__(16) double dg_smem[];
    double* sA = dg_smem;                                   // [STAGES][BM][LDK]
    double* sB = dg_smem + DG_STAGES * DG_BM * DG_LDK;      // [STAGES][BN][LDK]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp & 3, wn = warp >> 2;
    const int m0 = blockIdx.y * DG_BM, n0 = blockIdx.x * DG_BN;
    if (upper_only && m0 > n0 + DG_BN - 1) return;  // tile strictly below the diagonal
    if (kbeg >= kend) return;
    const int nk = (int)((kend - kbeg + DG_BK - 1) / DG_BK);

    auto load = [&](int stage, int kt) {
        const int64_t kb = kbeg + (int64_t)kt * DG_BK;
        double* a = sA + stage * DG_BM * DG_LDK;
        double* b = sB + stage * DG_BN * DG_LDK;
#pragma unroll
        for (int e = 0; e < (DG_BM * DG_BK) / 256; ++e) {
            const int idx = tid + 256 * e;
            const int row = TA ? idx % DG_BM : idx >> 4, kk = TA ? idx / DG_BM : idx & 15;
            const int gm = m0 + row;
            const int64_t gk = kb + kk;
            const bool ok = gm < M && gk < kend;
            cp_async8(a + row * DG_LDK + kk, ok ? (TA ? A + gk * lda + gm : A + (int64_t)gm * lda + gk) : A, ok);
        }
#pragma unroll
        for (int e = 0; e < (DG_BN * DG_BK) / 256; ++e) {
            const int idx = tid + 256 * e;
            const int row = TB ? idx % DG_BN : idx >> 4, kk = TB ? idx / DG_BN : idx & 15;
            const int gn = n0 + row;
            const int64_t gk = kb + kk;
            const bool ok = gn < N && gk < kend;
            cp_async8(b + row * DG_LDK + kk, ok ? (TB ? B + gk * ldb + gn : B + (int64_t)gn * ldb + gk) : B, ok);
        }
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < DG_STAGES - 1; ++s) {
        if (s < nk) load(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<DG_STAGES - 2>();
        __syncthreads();
        const int pf = kt + DG_STAGES - 1;
        if (pf < nk) load(pf % DG_STAGES, pf);
        cp_async_commit();
        const double* a = sA + (kt % DG_STAGES) * DG_BM * DG_LDK;
        const double* b = sB + (kt % DG_STAGES) * DG_BN * DG_LDK;
#pragma unroll
        for (int ks = 0; ks < DG_BK / 4; ++ks) {
            double af[4], bf[4];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) af[mt] = a[(wm * 32 + mt * 8 + g) * DG_LDK + ks * 4 + t];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) bf[nt] = b[(wn * 32 + nt * 8 + g) * DG_LDK + ks * 4 + t];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) dmma_8x8x4(acc[mt][nt], af[mt], bf[nt]);
        }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int m = m0 + wm * 32 + mt * 8 + g;
                const int n = n0 + wn * 32 + nt * 8 + 2 * t + h;
                if (m < M && n < N) epi(m, n, acc[mt][nt][h], z);
            }
}

template <class Epi, bool TA = false, bool TB = false>
__global__ void __launch_bounds__(256) dgemm_tn_kernel(const double* __restrict__ A, int64_t lda,
                                                       const double* __restrict__ B, int64_t ldb,
                                                       int M, int N, int64_t K, int64_t k_per_split,
                                                       int upper_only, Epi epi) {
    const int64_t kbeg = (int64_t)blockIdx.z * k_per_split;
    const int64_t kend = kbeg + k_per_split < K ? kbeg + k_per_split : K;
    dgemm_tile<Epi, TA, TB>(A, lda, B, ldb, M, N, kbeg, kend, upper_only, epi, (int)blockIdx.z);
}

// Batched over blockIdx.z: operands z * sa and z * sb elements on, all of K.
template <class Epi, bool TA = false, bool TB = false>
__global__ void __launch_bounds__(256) dgemm_batched_kernel(const double* __restrict__ A, int64_t lda, int64_t sa,
                                                            const double* __restrict__ B, int64_t ldb, int64_t sb,
                                                            int M, int N, int64_t K, Epi epi) {
    const int z = (int)blockIdx.z;
    dgemm_tile<Epi, TA, TB>(A + z * sa, lda, B + z * sb, ldb, M, N, 0, K, 0, epi, z);
}

// value * alpha -> C[m*ldc + n]
struct EpiStore {
    double* C;
    int64_t ldc;
    double alpha;
    int accumulate;  // C += alpha v instead of C = alpha v
    __device__ __forceinline__ void operator()(int m, int n, double v, int) const {
        double* c = C + (int64_t)m * ldc + n;
        *c = accumulate ? *c + alpha * v : alpha * v;
    }
};

// split-K partial -> P[split][m*N + n]
struct EpiSplit {
    double* P;
    int64_t split_stride;
    int N;
    __device__ __forceinline__ void operator()(int m, int n, double v, int split) const {
        P[(int64_t)split * split_stride + (int64_t)m * N + n] = v;
    }
};

}  // namespace fc
