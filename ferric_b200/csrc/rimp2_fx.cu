// Split-BF16 RI-MP2 with exact tensor-core accumulation (FC_PREC_MIXED).
//
// Why: the tcgen05 FP32 accumulator does not round to nearest -- measured on
// B200, every accumulation step loses about 2^-24 of the running sum toward
// zero, so a floating hi/lo split accumulated over naux = 4800 is biased by
// ~1e-5 relative in E (the effect the reference measured for its f32 path,
// ferric-core/src/gpu/mixed.rs:18-21).  Here every FP32 partial sum is an
// integer below 2^24, which FP32 holds exactly whatever the rounding mode.
//
// Split.  Each operand row r (an (i, a) column of B_ov over Q for the pair
// products, a Q row over (j, b) for the adjoint contraction) gets a power of
// two s_r with max|x| / s_r in [64, 128), and three bf16 slices holding
// integers in [-128, 128]:
//     x / s_r = c1 + c2 / 256 + c3 / 65536 + eps,   |eps| <= 2^-17.
// Products.  Three levels, one TMEM accumulator each, exact in FP32:
//     L0 = c1 c1',  L1 = c1 c2' + c2 c1',  L2 = c1 c3' + c2 c2' + c3 c1'
// (6 bf16 tensor-core products), combined in FP64 in the epilogue:
//     g = s_r s_r' (L0 + L1 / 256 + L2 / 65536).
//
// Pair kernel (this file): item = (pair, a-tile 128, b-tile 128); the X phase
// accumulates (ia|jb) into the three level accumulators (3 x 128 TMEM
// columns), the epilogue parks it in registers (FP32, round to nearest), and
// the Y phase accumulates (ib|ja) = G_ji[a, b] into the same columns, so each
// thread holds an element and its exchange partner.  128 x 128 UMMAs keep the
// shared-memory operand reads at 128 B/clk (128 x 64 ones need 192 B/clk, more
// than an SM delivers).  Energy mode: unordered pairs, E_OS += (X^2 + Y^2)/D,
// E_SS += (X - Y)^2/D (i == j: X phase only, E_SS = 0), the reference pair
// loop of ferric-mp2/src/rimp2.rs:1399-1544 over both orderings.  Gradient
// mode: ordered pairs of an occupied chunk; writes Tt_ij = (2X - Y)/D (FP32)
// and the dE/deps partials; the adjoint contraction Gamma = 4 B Tt^T runs in
// gemm_fx_kernel with the same exact-level scheme.
#include "fc_internal.cuh"
#include "rimp2.cuh"
#include "tc.cuh"
#include "tmap.cuh"

namespace fc {

namespace fx {

constexpr int BM = 128, BN = 128, KT = 64;
constexpr int A_BYTES = BM * KT * 2;  // 16 KiB
constexpr int B_BYTES = BN * KT * 2;  // 16 KiB
constexpr int NSL = 3;
constexpr int STAGE_BYTES = NSL * (A_BYTES + B_BYTES);  // 96 KiB
constexpr int STAGES = 2;
constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 7168;
constexpr uint32_t IDESC = tc::idesc_bf16_f32(128, 128);
constexpr double L1W = 1.0 / 256.0, L2W = 1.0 / 65536.0;

// products: (A slice, B slice, level)
__constant__ int8_t kPA[6] = {0, 0, 1, 0, 1, 2};
__constant__ int8_t kPB[6] = {0, 1, 0, 2, 1, 0};
__constant__ int8_t kPL[6] = {0, 1, 1, 2, 2, 2};
__constant__ int8_t kPFirst[6] = {1, 1, 0, 1, 0, 0};  // first product of its level

}  // namespace fx

// ---------------------------------------------------------- split kernels --

// cmax[c] = max over rows of |B[r, c]| (as ordered uint64 bits of a double).
__global__ void colmax_kernel(const double* __restrict__ B, int64_t rows, int64_t cols,
                              int64_t rows_per_split, unsigned long long* cmax, int* bad) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const int64_t r0 = (int64_t)blockIdx.y * rows_per_split;
    const int64_t r1 = r0 + rows_per_split < rows ? r0 + rows_per_split : rows;
    double m = 0.0;
    bool nf = false;
    for (int64_t r = r0; r < r1; ++r) {
        const double v = fabs(B[r * cols + c]);
        nf |= !(v <= 1.0e300);
        m = v > m ? v : m;
    }
    if (nf) atomicOr(bad, 1);
    atomicMax(cmax + c, (unsigned long long)__double_as_longlong(m));
}

// Power-of-two scale with max / s in [64, 128).
__device__ __forceinline__ double pow2_scale(double mx) {
    if (!(mx > 0.0) || !(mx <= 1.0e300)) return 1.0;
    int k;
    frexp(mx, &k);           // mx = m 2^k, m in [0.5, 1)
    return ldexp(1.0, k - 7);
}

// scl[i*a_pad + a] from the column maxima of B_ov (1 for padding rows).
__global__ void row_scale_kernel(const unsigned long long* __restrict__ cmax, int64_t nocc, int64_t nvir,
                                 int64_t a_pad, double* __restrict__ scl) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nocc * a_pad) return;
    const int64_t i = r / a_pad, a = r % a_pad;
    scl[r] = a < nvir ? pow2_scale(__longlong_as_double((long long)cmax[i * nvir + a])) : 1.0;
}

__device__ __forceinline__ void fx_slices(double x, double inv_s, __nv_bfloat16& c1, __nv_bfloat16& c2,
                                          __nv_bfloat16& c3) {
    const double y = x * inv_s;
    const double a = rint(y);
    const double y2 = (y - a) * 256.0;
    const double b = rint(y2);
    const double c = rint((y2 - b) * 256.0);
    c1 = __double2bfloat16(a);
    c2 = __double2bfloat16(b);
    c3 = __double2bfloat16(c);
}

// B[q, ia] -> Bt[s][i][a][q] (q < q_pad) integer slices at scale scl[i*a_pad+a].
__global__ void __launch_bounds__(256) split_fx_transpose_kernel(const double* __restrict__ B, int64_t naux,
                                                                 int64_t nocc, int64_t nvir, int64_t a_pad,
                                                                 int64_t q_pad, const double* __restrict__ scl,
                                                                 __nv_bfloat16* __restrict__ Bt) {
    __shared__ double tile[64][65];
    const int64_t nov = nocc * nvir;
    const int64_t q0 = (int64_t)blockIdx.y * 64, ia0 = (int64_t)blockIdx.x * 64;
    const int tid = threadIdx.x;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const int idx = tid + 256 * e, r = idx >> 6, c = idx & 63;
        const int64_t q = q0 + r, ia = ia0 + c;
        tile[r][c] = (q < naux && ia < nov) ? B[q * nov + ia] : 0.0;
    }
    __syncthreads();
    const int64_t ss = nocc * a_pad * q_pad;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = tid + 256 * e, c = idx >> 5, qq = (idx & 31) * 2;
        const int64_t ia = ia0 + c;
        if (ia >= nov) continue;
        const int64_t i = ia / nvir, a = ia % nvir;
        const double inv = 1.0 / scl[i * a_pad + a];
        __nv_bfloat16 a0, b0, c0, a1, b1, c1;
        fx_slices(tile[qq][c], inv, a0, b0, c0);
        fx_slices(tile[qq + 1][c], inv, a1, b1, c1);
        const int64_t off = (i * a_pad + a) * q_pad + q0 + qq;
        *reinterpret_cast<__nv_bfloat162*>(Bt + off) = __halves2bfloat162(a0, a1);
        *reinterpret_cast<__nv_bfloat162*>(Bt + ss + off) = __halves2bfloat162(b0, b1);
        *reinterpret_cast<__nv_bfloat162*>(Bt + 2 * ss + off) = __halves2bfloat162(c0, c1);
    }
}

__global__ void fill_kernel(double* __restrict__ x, int64_t n, double v) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) x[k] = v;
}

// Per-Q-row split of B_ov over (j, b) with b padded to a_pad:
// Bq[s][q][j*a_pad + b] (q < q_rows), scale qs[q].  One CTA per Q row.
__global__ void __launch_bounds__(256) split_fx_qrows_kernel(const double* __restrict__ B, int64_t naux,
                                                             int64_t nocc, int64_t nvir, int64_t a_pad,
                                                             int64_t q_rows, double* __restrict__ qs,
                                                             __nv_bfloat16* __restrict__ Bq) {
    __shared__ double red[32];
    const int64_t q = blockIdx.x;
    const int64_t nov = nocc * nvir, K = nocc * a_pad;
    const double* row = B + q * nov;
    double m = 0.0;
    for (int64_t k = threadIdx.x; k < nov; k += 256) m = fmax(m, fabs(row[k]));
    // block max (fixed order)
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double s = pow2_scale(red[0]);
    if (threadIdx.x == 0) qs[q] = s;
    const double inv = 1.0 / s;
    const int64_t ss = q_rows * K;
    __nv_bfloat16* o0 = Bq + q * K;
    for (int64_t k = threadIdx.x; k < nov; k += 256) {
        const int64_t j = k / nvir, b = k % nvir;
        __nv_bfloat16 c1, c2, c3;
        fx_slices(row[k], inv, c1, c2, c3);
        const int64_t d = j * a_pad + b;
        o0[d] = c1;
        o0[ss + d] = c2;
        o0[2 * ss + d] = c3;
    }
}

// Per-row split of the FP32 amplitude chunk T[rows][K] -> Ts[s][rows][K],
// ts[row].  One CTA per row; the row is read twice (max, then slices).
__global__ void __launch_bounds__(256) split_fx_rows_f32_kernel(const float* __restrict__ T, int64_t K,
                                                                int64_t slice_rows, double* __restrict__ ts,
                                                                __nv_bfloat16* __restrict__ Ts) {
    __shared__ double red[32];
    const int64_t r = blockIdx.x;
    const float4* row = reinterpret_cast<const float4*>(T + r * K);
    const int64_t K4 = K / 4;
    float m = 0.f;
    for (int64_t k = threadIdx.x; k < K4; k += 256) {
        const float4 v = row[k];
        m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double s = pow2_scale(red[0]);
    if (threadIdx.x == 0) ts[r] = s;
    const double inv = 1.0 / s;
    const int64_t ss = slice_rows * K;
    __nv_bfloat16* o0 = Ts + r * K;
    for (int64_t k = threadIdx.x; k < K4; k += 256) {
        const float4 v = row[k];
        __nv_bfloat16 a[4], b[4], c[4];
        fx_slices(v.x, inv, a[0], b[0], c[0]);
        fx_slices(v.y, inv, a[1], b[1], c[1]);
        fx_slices(v.z, inv, a[2], b[2], c[2]);
        fx_slices(v.w, inv, a[3], b[3], c[3]);
        uint2 pa, pb, pc;
        __nv_bfloat162 t0 = __halves2bfloat162(a[0], a[1]), t1 = __halves2bfloat162(a[2], a[3]);
        pa.x = *reinterpret_cast<uint32_t*>(&t0);
        pa.y = *reinterpret_cast<uint32_t*>(&t1);
        t0 = __halves2bfloat162(b[0], b[1]);
        t1 = __halves2bfloat162(b[2], b[3]);
        pb.x = *reinterpret_cast<uint32_t*>(&t0);
        pb.y = *reinterpret_cast<uint32_t*>(&t1);
        t0 = __halves2bfloat162(c[0], c[1]);
        t1 = __halves2bfloat162(c[2], c[3]);
        pc.x = *reinterpret_cast<uint32_t*>(&t0);
        pc.y = *reinterpret_cast<uint32_t*>(&t1);
        reinterpret_cast<uint2*>(o0)[k] = pa;
        reinterpret_cast<uint2*>(o0 + ss)[k] = pb;
        reinterpret_cast<uint2*>(o0 + 2 * ss)[k] = pc;
    }
}

// ------------------------------------------------------------ pair kernel --

struct PairFxArgs {
    const double* eo;
    const double* ev;
    const double* scl;  // [nocc * a_pad] operand-row scales
    const int2* pairs;  // pairs of the launch
    const int2* tiles;  // (a-tile, b-tile) of each item of a pair
    int ntiles;         // tiles per pair
    int npairs;
    int nocc, nvir, a_pad, nTa, nTb, nk;
    int64_t items;
    double* part;  // [item][2]
    int* err;
    // gradient mode
    float* T;        // amplitude chunk [ci*a_pad][nocc*a_pad]
    int64_t ldt;     // nocc * a_pad
    int i0;
    double* occ_part;  // [item]
    double* vir_part;  // [item][128]
};

template <int GRAD>
__global__ void __launch_bounds__(320, 1)
    pair_fx_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const PairFxArgs p) {
    using namespace fx;
    constexpr int S = STAGES;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_u32 = smem_u32(smem_raw);
    const uint32_t base_u32 = (raw_u32 + 1023u) & ~1023u;
    uint8_t* base = smem_raw + (base_u32 - raw_u32);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * STAGE_BYTES);
    uint64_t* full = bars;                // [S]
    uint64_t* empty = bars + S;           // [S]
    uint64_t* tfull = bars + 2 * S;       // [1] a phase's levels are complete in TMEM
    uint64_t* tempty = bars + 2 * S + 1;  // [1] the epilogue has read them out
    uint64_t* drain = bars + 2 * S + 2;   // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 3);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(bars + 2 * S + 4);  // [2][8][3]
    double* rowsh = red + 48;                                    // [128] row sums of the upper column half
    double* colsh = rowsh + 128;                                 // [4 quadrants][2 halves][64] column sums

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(tfull, 1);
        tc::mbar_init(tempty, 256);
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) {
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 512);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;
    const int64_t tpp = p.ntiles;  // tiles per pair

    auto sa = [&](int s, int sl) { return base_u32 + s * STAGE_BYTES + sl * A_BYTES; };
    auto sb = [&](int s, int sl) { return base_u32 + s * STAGE_BYTES + NSL * A_BYTES + sl * B_BYTES; };
    auto row_of = [&](int sl, int i, int r0) { return (sl * p.nocc + i) * p.a_pad + r0; };

    if (warp == 0) {
        // ------------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t g = 0;
            for (int64_t k = blockIdx.x; k < p.items && !*abort_flag; k += gridDim.x) {
                const int2 ij = p.pairs[k / tpp];
                const int2 tt = p.tiles[k % tpp];
                const int ta = tt.x, tb = tt.y;
                const int nph = ij.x == ij.y ? 1 : 2;
                for (int ph = 0; ph < nph; ++ph) {
                    const int ia = ph == 0 ? ij.x : ij.y, ib = ph == 0 ? ij.y : ij.x;
                    for (int kt = 0; kt < p.nk; ++kt, ++g) {
                        const int s = g % S;
                        const uint32_t u = g / S;
                        if (!tc::mbar_wait(&empty[s], (u & 1) ^ 1, abort_flag, p.err)) goto prod_done;
                        tc::mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
#pragma unroll
                        for (int sl = 0; sl < NSL; ++sl) {
                            tc::tma_load_2d(base + (sa(s, sl) - base_u32), &tmA, &full[s], kt * KT,
                                            row_of(sl, ia, ta * BM));
                            tc::tma_load_2d(base + (sb(s, sl) - base_u32), &tmB, &full[s], kt * KT,
                                            row_of(sl, ib, tb * BN));
                        }
                    }
                }
            }
        prod_done:
            for (uint32_t q = 0; q < (uint32_t)S && q < g; ++q) {
                const uint32_t gg = g - 1 - q;
                int no_abort = 0;
                tc::mbar_wait(&full[gg % S], (gg / S) & 1, &no_abort, p.err);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------ UMMA issuer
        if (lane == 0) {
            uint32_t g = 0, pc = 0;  // pc: phases issued (TMEM hand-overs)
            for (int64_t k = blockIdx.x; k < p.items && !*abort_flag; k += gridDim.x) {
                const int2 ij = p.pairs[k / tpp];
                const int nph = ij.x == ij.y ? 1 : 2;
                for (int ph = 0; ph < nph; ++ph, ++pc) {
                    if (!tc::mbar_wait(tempty, (pc & 1) ^ 1, abort_flag, p.err)) goto mma_done;
                    tc::fence_after_sync();
                    for (int kt = 0; kt < p.nk; ++kt, ++g) {
                        const int s = g % S;
                        const uint32_t u = g / S;
                        if (!tc::mbar_wait(&full[s], u & 1, abort_flag, p.err)) goto mma_done;
                        tc::fence_after_sync();
#pragma unroll
                        for (int pr = 0; pr < 6; ++pr) {
                            const uint32_t a0 = sa(s, kPA[pr]), b0 = sb(s, kPB[pr]);
                            const uint32_t dcol = tmem_base + kPL[pr] * BN;
#pragma unroll
                            for (int kk = 0; kk < KT / 16; ++kk)
                                tc::umma_bf16(dcol, tc::sdesc_k128(a0 + kk * 32), tc::sdesc_k128(b0 + kk * 32),
                                              IDESC, (kt > 0 || kk > 0 || !kPFirst[pr]) ? 1u : 0u);
                        }
                        tc::umma_commit(&empty[s]);
                    }
                    tc::umma_commit(tfull);
                }
            }
        mma_done:
            tc::umma_commit(drain);
            int no_abort = 0;
            tc::mbar_wait(drain, 0, &no_abort, p.err);
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- epilogue
        // 8 warps: lane quadrant q = warp % 4 (TMEM lanes 32q..32q+31), column
        // half h = (warp - 2) / 4; each thread owns row `row`, columns [64h, 64h + 64).
        constexpr int HC = BN / 2;
        const int q = warp & 3;
        const int h = (warp - 2) >> 2;
        const int row = q * 32 + lane;  // a within the tile
        const int et = tid - 64;        // 0..255
        const uint32_t tl = tmem_base + ((uint32_t)(q * 32) << 16) + h * HC;
        uint32_t li = 0, pc = 0;
        for (int64_t k = blockIdx.x; k < p.items; k += gridDim.x, ++li) {
            const int2 ij = p.pairs[k / tpp];
            const int i = ij.x, j = ij.y;
            const bool diag = i == j;
            const int2 tt2 = p.tiles[k % tpp];
            const int ta = tt2.x, tb = tt2.y;
            // tiles ta <= tb only: X_ba = Y_ab, so the mirrored tile (tb, ta) is this
            // tile transposed.  Energy mode weights it 2; gradient mode also
            // writes its amplitudes (transposed) and its derivative terms.
            const double wt = (!GRAD && ta < tb) ? 2.0 : 1.0;
            const bool mir = GRAD && ta < tb;
            const int a = ta * BM + row;
            const bool va = a < p.nvir;
            const double dA = p.eo[i] + p.eo[j] - (va ? p.ev[a] : 0.0);
            const double sxa = p.scl[(int64_t)i * p.a_pad + a];
            const double sya = p.scl[(int64_t)j * p.a_pad + a];
            const int b0 = tb * BN + h * HC;  // first column of this thread
            const double* sxb = p.scl + (int64_t)j * p.a_pad + b0;
            const double* syb = p.scl + (int64_t)i * p.a_pad + b0;
            const double* evb = p.ev + b0;
            const int bmax = p.nvir - b0;    // columns c < bmax are real virtuals

            // X phase: park (ia|jb) of this half row in registers (FP32, round to nearest)
            if (!tc::mbar_wait(tfull, pc & 1, abort_flag, p.err)) break;
            tc::fence_after_sync();
            float xr[HC];
#pragma unroll
            for (int c0 = 0; c0 < HC; c0 += 16) {
                float l0[16], l1[16], l2[16];
                tc::tmem_ld16(tl + c0, l0);
                tc::tmem_ld16(tl + BN + c0, l1);
                tc::tmem_ld16(tl + 2 * BN + c0, l2);
                tc::tmem_wait_ld();
#pragma unroll
                for (int cc = 0; cc < 16; ++cc)
                    xr[c0 + cc] = (float)(sxa * sxb[c0 + cc] *
                                          ((double)l0[cc] + (double)l1[cc] * L1W + (double)l2[cc] * L2W));
            }
            tc::fence_before_sync();
            tc::mbar_arrive(tempty);
            ++pc;
            if (!diag) {
                if (!tc::mbar_wait(tfull, pc & 1, abort_flag, p.err)) break;
                tc::fence_after_sync();
            }
            // plain FP64 sums over this thread's 64 terms (relative error <= 64 u);
            // the tile partials are summed compensated
            double os = 0.0, ss = 0.0, oc = 0.0, rowc = 0.0;
#pragma unroll
            for (int c0 = 0; c0 < HC; c0 += 8) {
                float y0[8], y1[8], y2[8];
                if (!diag) {
                    tc::tmem_ld8(tl + c0, y0);
                    tc::tmem_ld8(tl + BN + c0, y1);
                    tc::tmem_ld8(tl + 2 * BN + c0, y2);
                    tc::tmem_wait_ld();
                    if (c0 + 8 == HC) {  // every level of this phase is read: release TMEM
                        tc::fence_before_sync();
                        tc::mbar_arrive(tempty);
                    }
                }
                float tt8[8], mv8[8];
#pragma unroll
                for (int cc = 0; cc < 8; ++cc) {
                    const double x = (double)xr[c0 + cc];
                    const double y = diag ? x
                                          : sya * syb[c0 + cc] *
                                                ((double)y0[cc] + (double)y1[cc] * L1W + (double)y2[cc] * L2W);
                    float tval = 0.f, mval = 0.f, colv = 0.f;
                    if (va && c0 + cc < bmax) {
                        const double r = 1.0 / (dA - evb[c0 + cc]);
                        if (GRAD) {
                            const double tt = (2.0 * x - y) * r;   // Tt_ij[a, b]
                            const double cd = x * r * tt;          // t Tt at (a, b)
                            tval = (float)tt;
                            os += x * x * r;
                            ss += x * (x - y) * r;
                            oc += cd;
                            rowc += cd;
                            if (mir) {
                                const double tm = (2.0 * y - x) * r;  // Tt_ij[b, a]
                                const double cm = y * r * tm;         // t Tt at (b, a)
                                mval = (float)tm;
                                colv = (float)cm;
                                os += y * y * r;
                                ss += y * (y - x) * r;
                                oc += cm;
                            }
                        } else if (diag) {
                            os += x * x * r;
                        } else {
                            os += (x * x + y * y) * r;
                            ss += (x - y) * (x - y) * r;
                        }
                    }
                    tt8[cc] = tval;
                    mv8[cc] = mval;
                    if (GRAD) xr[c0 + cc] = colv;  // x of this column is consumed: keep cm there
                }
                if (GRAD) {
                    float* trow = p.T + ((int64_t)(i - p.i0) * p.a_pad) * p.ldt + (int64_t)j * p.a_pad;
                    float4* dst = reinterpret_cast<float4*>(trow + (int64_t)a * p.ldt + b0 + c0);
                    dst[0] = make_float4(tt8[0], tt8[1], tt8[2], tt8[3]);
                    dst[1] = make_float4(tt8[4], tt8[5], tt8[6], tt8[7]);
                    if (mir) {
#pragma unroll
                        for (int cc = 0; cc < 8; ++cc)  // lanes hold consecutive a: coalesced
                            trow[(int64_t)(b0 + c0 + cc) * p.ldt + a] = mv8[cc];
                    }
                }
            }
            if (!diag) ++pc;
            const double vo = warp_sum(os), vs = warp_sum(ss);
            const double vc = GRAD ? warp_sum(oc) : 0.0;
            double* rb = red + (li & 1) * 24;
            if (lane == 0) {
                rb[(warp - 2) * 3 + 0] = vo;
                rb[(warp - 2) * 3 + 1] = vs;
                rb[(warp - 2) * 3 + 2] = vc;
            }
            if (GRAD && h == 1) rowsh[row] = rowc;
            if (mir) {
                // column sums of the mirrored terms over this warp's 32 rows: a
                // reduce-scatter butterfly leaves columns 2*lane, 2*lane+1 in xr[0..1]
#pragma unroll
                for (int half = HC / 2, off = 16; off > 0; half >>= 1, off >>= 1) {
                    const bool up = (lane & off) != 0;
#pragma unroll
                    for (int c = 0; c < half; ++c) {
                        const float send = up ? xr[c] : xr[c + half];
                        const float recv = __shfl_xor_sync(0xffffffffu, send, off);
                        xr[c] = (up ? xr[c + half] : xr[c]) + recv;
                    }
                }
                colsh[(q * 2 + h) * 64 + 2 * lane] = (double)xr[0];
                colsh[(q * 2 + h) * 64 + 2 * lane + 1] = (double)xr[1];
            }
            asm volatile("bar.sync 1, 256;" ::: "memory");
            if (GRAD && h == 0) p.vir_part[k * 2 * BM + row] = rowc + rowsh[row];
            if (mir && et < BM) {
                const int hh = et >> 6, c = et & 63;
                double v = 0.0;
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) v += colsh[(qq * 2 + hh) * 64 + c];
                p.vir_part[k * 2 * BM + BM + et] = v;
            }
            if (et == 0) {
                KSum so, sn, sc;
#pragma unroll
                for (int w = 0; w < 8; ++w) {
                    so.add(rb[w * 3]);
                    sn.add(rb[w * 3 + 1]);
                    sc.add(rb[w * 3 + 2]);
                }
                p.part[2 * k] = wt * so.value();
                p.part[2 * k + 1] = wt * sn.value();
                if (GRAD) p.occ_part[k] = sc.value();
            }
            // rowsh is rewritten next item only after every thread passed the next barrier
            asm volatile("bar.sync 1, 256;" ::: "memory");
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 1) {
        __syncwarp();
        tc::tmem_dealloc(tmem_base, 512);
    }
}

// --------------------------------------------------- adjoint contraction --

struct GemmFxArgs {
    const double* rs;  // [M] scales of the A rows (amplitude rows (i, a))
    const double* cs;  // [N] scales of the B rows (Q)
    int M, N, nk;      // padded to 128; nk = K / 64
    int nTm, nTn;
    int64_t tiles;
    int a_pad, nvir, naux, i0;
    int64_t nov;
    double alpha;
    double* out;  // Gamma (naux, nov)
    int* err;
};

constexpr int GF_STAGE = 3 * (16384 + 16384);  // 96 KiB
constexpr int GF_STAGES = 2;
constexpr int GF_SMEM = GF_STAGES * GF_STAGE + 1024 + 1024;
constexpr uint32_t GF_IDESC = tc::idesc_bf16_f32(128, 128);

// out[Q, i*nvir + a] = alpha * s_row s_Q (L0 + L1/256 + L2/65536), rows = (i - i0, a).
__global__ void __launch_bounds__(192, 1)
    gemm_fx_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const GemmFxArgs p) {
    using namespace fx;
    constexpr int S = GF_STAGES;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_u32 = smem_u32(smem_raw);
    const uint32_t base_u32 = (raw_u32 + 1023u) & ~1023u;
    uint8_t* base = smem_raw + (base_u32 - raw_u32);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * GF_STAGE);
    uint64_t* full = bars;
    uint64_t* empty = bars + S;
    uint64_t* tfull = bars + 2 * S;
    uint64_t* tempty = bars + 2 * S + 1;
    uint64_t* drain = bars + 2 * S + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 3);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(tfull, 1);
        tc::mbar_init(tempty, 128);
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) {
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 512);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;
    auto sa = [&](int s, int sl) { return base_u32 + s * GF_STAGE + sl * 16384; };
    auto sb = [&](int s, int sl) { return base_u32 + s * GF_STAGE + 3 * 16384 + sl * 16384; };

    if (warp == 0) {
        if (lane == 0) {
            uint32_t g = 0;
            for (int64_t t = blockIdx.x; t < p.tiles && !*abort_flag; t += gridDim.x) {
                const int tm = (int)(t / p.nTn), tn = (int)(t % p.nTn);
                for (int kt = 0; kt < p.nk; ++kt, ++g) {
                    const int s = g % S;
                    const uint32_t u = g / S;
                    if (!tc::mbar_wait(&empty[s], (u & 1) ^ 1, abort_flag, p.err)) goto prod_done;
                    tc::mbar_arrive_expect_tx(&full[s], GF_STAGE);
#pragma unroll
                    for (int sl = 0; sl < 3; ++sl) {
                        tc::tma_load_2d(base + (sa(s, sl) - base_u32), &tmA, &full[s], kt * KT, sl * p.M + tm * 128);
                        tc::tma_load_2d(base + (sb(s, sl) - base_u32), &tmB, &full[s], kt * KT, sl * p.N + tn * 128);
                    }
                }
            }
        prod_done:
            for (uint32_t q = 0; q < (uint32_t)S && q < g; ++q) {
                const uint32_t gg = g - 1 - q;
                int no_abort = 0;
                tc::mbar_wait(&full[gg % S], (gg / S) & 1, &no_abort, p.err);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            uint32_t g = 0, li = 0;
            for (int64_t t = blockIdx.x; t < p.tiles && !*abort_flag; t += gridDim.x, ++li) {
                if (!tc::mbar_wait(tempty, (li & 1) ^ 1, abort_flag, p.err)) break;
                tc::fence_after_sync();
                for (int kt = 0; kt < p.nk; ++kt, ++g) {
                    const int s = g % S;
                    const uint32_t u = g / S;
                    if (!tc::mbar_wait(&full[s], u & 1, abort_flag, p.err)) goto mma_done;
                    tc::fence_after_sync();
#pragma unroll
                    for (int pr = 0; pr < 6; ++pr) {
                        const uint32_t a0 = sa(s, kPA[pr]), b0 = sb(s, kPB[pr]);
                        const uint32_t dcol = tmem_base + kPL[pr] * 128;
#pragma unroll
                        for (int kk = 0; kk < KT / 16; ++kk)
                            tc::umma_bf16(dcol, tc::sdesc_k128(a0 + kk * 32), tc::sdesc_k128(b0 + kk * 32), GF_IDESC,
                                          (kt > 0 || kk > 0 || !kPFirst[pr]) ? 1u : 0u);
                    }
                    tc::umma_commit(&empty[s]);
                }
                tc::umma_commit(tfull);
            }
        mma_done:
            tc::umma_commit(drain);
            int no_abort = 0;
            tc::mbar_wait(drain, 0, &no_abort, p.err);
        }
        __syncwarp();
    } else {
        const int q = warp & 3;
        const int row = q * 32 + lane;
        uint32_t li = 0;
        for (int64_t t = blockIdx.x; t < p.tiles; t += gridDim.x, ++li) {
            const int tm = (int)(t / p.nTn), tn = (int)(t % p.nTn);
            if (!tc::mbar_wait(tfull, li & 1, abort_flag, p.err)) break;
            tc::fence_after_sync();
            const int m = tm * 128 + row;           // amplitude row (i - i0, a)
            const int il = m / p.a_pad, a = m % p.a_pad;
            const bool vm = a < p.nvir;
            const double sr = p.alpha * p.rs[m];
            double* orow = p.out + (int64_t)(p.i0 + il) * p.nvir + a;
            const uint32_t tl = tmem_base + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
            for (int c0 = 0; c0 < 128; c0 += 16) {
                float l0[16], l1[16], l2[16];
                tc::tmem_ld16(tl + c0, l0);
                tc::tmem_ld16(tl + 128 + c0, l1);
                tc::tmem_ld16(tl + 256 + c0, l2);
                tc::tmem_wait_ld();
                if (vm) {
#pragma unroll
                    for (int cc = 0; cc < 16; ++cc) {
                        const int Q = tn * 128 + c0 + cc;
                        if (Q < p.naux)
                            orow[(int64_t)Q * p.nov] =
                                sr * p.cs[Q] * ((double)l0[cc] + (double)l1[cc] * L1W + (double)l2[cc] * L2W);
                    }
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(tempty);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 1) {
        __syncwarp();
        tc::tmem_dealloc(tmem_base, 512);
    }
}

// ------------------------------------------------------------ reductions --

__global__ void __launch_bounds__(1024) fx_reduce_pairs_kernel(const double* __restrict__ part, int64_t n,
                                                               double* out) {
    __shared__ double so[1024], sss[1024];
    KSum a, b;
    for (int64_t k = threadIdx.x; k < n; k += 1024) {
        a.add(part[2 * k]);
        b.add(part[2 * k + 1]);
    }
    so[threadIdx.x] = a.value();
    sss[threadIdx.x] = b.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum x, y;
        for (int k = 0; k < 1024; ++k) {
            x.add(so[k]);
            y.add(sss[k]);
        }
        out[0] = x.value();
        out[1] = y.value();
    }
}

__global__ void __launch_bounds__(256) fx_reduce_occ_kernel(const double* __restrict__ occ_part,
                                                            int64_t items_per_i, int i0, double* de_docc) {
    __shared__ double sh[256];
    const int il = blockIdx.x;
    const double* src = occ_part + (int64_t)il * items_per_i;
    KSum a;
    for (int64_t k = threadIdx.x; k < items_per_i; k += 256) a.add(src[k]);
    sh[threadIdx.x] = a.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum x;
        for (int k = 0; k < 256; ++k) x.add(sh[k]);
        de_docc[i0 + il] = -2.0 * x.value();
    }
}

// acc_vir[v] += 2 * (sum over the chunk's items of the row partials of v, from
// direct tiles (ta, tb) with v in ta, and of the column partials, from the
// mirrored tiles (tb, ta) with v in tb).  Fixed order: deterministic.
__global__ void __launch_bounds__(256) fx_reduce_vir_kernel(const double* __restrict__ vir_part,
                                                            const int2* __restrict__ tiles, int64_t npairs,
                                                            int ntiles, int nvir, double* acc_vir) {
    const int v = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (v >= nvir) return;
    const int tv = v / fx::BM, rv = v % fx::BM;
    const int64_t nterm = npairs * ntiles;
    KSum s;
    for (int64_t k = lane; k < nterm; k += 32) {
        const int2 t = tiles[k % ntiles];
        if (t.x == tv) s.add(vir_part[k * 2 * fx::BM + rv]);
        if (t.y == tv && t.x < t.y) s.add(vir_part[k * 2 * fx::BM + fx::BM + rv]);
    }
    const double r = warp_sum(s.value());
    if (lane == 0) acc_vir[v] += 2.0 * r;
}

// ------------------------------------------------------------------ host --

namespace {

struct FxSplit {
    __nv_bfloat16* bt;
    double* scl;
    int64_t a_pad, q_pad;
    CUtensorMap tmA, tmB;
};

fc_status fx_split_pairs(const Rimp2Dev& d, cudaStream_t st, int* bad, FxSplit* o) {
    const int64_t a_pad = (d.nvir + fx::BM - 1) / fx::BM * fx::BM;
    const int64_t q_pad = (d.naux + fx::KT - 1) / fx::KT * fx::KT;
    const int64_t nov = d.nocc * d.nvir;
    const int64_t rows = (int64_t)fx::NSL * d.nocc * a_pad;
    void *vbt, *vscl;
    FC_TRY(ws_get(WS_SPLIT, (size_t)rows * q_pad * 2, &vbt));
    FC_TRY(ws_get(WS_SCALE, (size_t)(nov + d.nocc * a_pad) * 8 + 256, &vscl));
    unsigned long long* cmax = (unsigned long long*)vscl;
    double* scl = (double*)vscl + nov;
    FC_CUDA(cudaMemsetAsync(cmax, 0, nov * 8, st));
    FC_CUDA(cudaMemsetAsync(vbt, 0, (size_t)rows * q_pad * 2, st));
    {
        const int64_t rps = 64;
        dim3 g((unsigned)((nov + 255) / 256), (unsigned)((d.naux + rps - 1) / rps));
        colmax_kernel<<<g, 256, 0, st>>>(d.b_ov, d.naux, nov, rps, cmax, bad);
    }
    row_scale_kernel<<<(unsigned)((d.nocc * a_pad + 255) / 256), 256, 0, st>>>(cmax, d.nocc, d.nvir, a_pad, scl);
    {
        dim3 g((unsigned)((nov + 63) / 64), (unsigned)((d.naux + 63) / 64));
        if (g.y > 65535) return fail(FC_ERR_LAYOUT, "split: naux too large");
        split_fx_transpose_kernel<<<g, 256, 0, st>>>(d.b_ov, d.naux, d.nocc, d.nvir, a_pad, q_pad, scl,
                                                     (__nv_bfloat16*)vbt);
    }
    FC_TRY(check_launch("fixed-point split kernels"));
    if (rows > (int64_t)UINT32_MAX) return fail(FC_ERR_LAYOUT, "split: too many operand rows");
    FC_TRY(make_tmap_bf16_2d(&o->tmA, vbt, q_pad, rows, q_pad * 2, fx::KT, fx::BM));
    FC_TRY(make_tmap_bf16_2d(&o->tmB, vbt, q_pad, rows, q_pad * 2, fx::KT, fx::BN));
    o->bt = (__nv_bfloat16*)vbt;
    o->scl = scl;
    o->a_pad = a_pad;
    o->q_pad = q_pad;
    return FC_OK;
}

fc_status fx_attrs() {
    static bool done = false;
    if (done) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(pair_fx_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx::SMEM));
    FC_CUDA(cudaFuncSetAttribute(pair_fx_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, fx::SMEM));
    FC_CUDA(cudaFuncSetAttribute(gemm_fx_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GF_SMEM));
    done = true;
    return FC_OK;
}

}  // namespace

fc_status rimp2_energy_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss, fc_stats* stats) {
    FC_TRY(fx_attrs());
    if (d.nocc > (1 << 15)) return fail(FC_ERR_LAYOUT, "split-BF16: nocc too large");
    void* vout;
    FC_TRY(ws_get(WS_OUT, 256, &vout));
    double* out = (double*)vout;
    int* flags = (int*)(out + 4);  // [0] range, [1] timeout
    FC_CUDA(cudaMemsetAsync(vout, 0, 256, st));
    Context& c = ctx();
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    FxSplit sp;
    FC_TRY(fx_split_pairs(d, st, flags, &sp));
    const int nocc = (int)d.nocc;
    const int nT = (int)(sp.a_pad / fx::BM);
    std::vector<int2> pairs;
    for (int i = 0; i < nocc; ++i)
        for (int j = i; j < nocc; ++j) pairs.push_back(make_int2(i, j));
    const size_t npairs = pairs.size();
    for (int ta = 0; ta < nT; ++ta)
        for (int tb = ta; tb < nT; ++tb) pairs.push_back(make_int2(ta, tb));
    void* vtab;
    FC_TRY(ws_get(WS_PAIRS, pairs.size() * sizeof(int2), &vtab));
    FC_CUDA(cudaMemcpyAsync(vtab, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    PairFxArgs a{};
    a.eo = d.eps_occ;
    a.ev = d.eps_vir;
    a.scl = sp.scl;
    a.pairs = (const int2*)vtab;
    a.tiles = (const int2*)vtab + npairs;
    a.ntiles = nT * (nT + 1) / 2;
    a.npairs = (int)npairs;
    a.nocc = nocc;
    a.nvir = (int)d.nvir;
    a.a_pad = (int)sp.a_pad;
    a.nTa = (int)(sp.a_pad / fx::BM);
    a.nTb = (int)(sp.a_pad / fx::BN);
    a.nk = (int)(sp.q_pad / fx::KT);
    a.items = (int64_t)a.npairs * a.ntiles;
    void* vpart;
    FC_TRY(ws_get(WS_PART, a.items * 2 * sizeof(double), &vpart));
    a.part = (double*)vpart;
    a.err = flags + 1;
    const int grid = (int)(a.items < c.sm_count ? a.items : c.sm_count);
    cudaEvent_t* ev = nullptr;
    if (stats) {
        FC_TRY(timing_events(1, &ev));
        FC_CUDA(cudaEventRecord(ev[0], st));
    }
    pair_fx_kernel<0><<<grid, 320, fx::SMEM, st>>>(sp.tmA, sp.tmB, a);
    FC_TRY(check_launch("pair_fx_kernel<energy>"));
    if (stats) FC_CUDA(cudaEventRecord(ev[1], st));
    fx_reduce_pairs_kernel<<<1, 1024, 0, st>>>((const double*)vpart, a.items, out);
    FC_TRY(check_launch("fx_reduce_pairs_kernel"));
    if (stats) FC_CUDA(cudaEventRecord(c.ev1, st));
    double h[2];
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "split-BF16: B_ov has a non-finite element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "split-BF16 pair kernel: a pipeline wait ran out");
    *e_os = h[0];
    *e_ss = h[1];
    if (stats) {
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        const double P = (double)d.nocc * (d.nocc + 1) / 2.0;
        stats->flops = 2.0 * (double)d.naux * (double)d.nvir * (double)d.nvir * P;
        stats->precision = FC_PREC_MIXED;
        stats->launches += 6;
        stats->tile_m = fx::BM;
        stats->tile_n = fx::BN;
        stats->k_panel = 0;
        stats->main_launches = 1;
        FC_TRY(timing_sum(1, &stats->main_ms));
        stats->main_flops = stats->flops;
        stats->main_bytes = 6.0 * (double)d.naux * (double)(d.nocc * d.nvir);
        stats->h2d_bytes += pairs.size() * sizeof(int2);
        stats->d2h_bytes += sizeof(h) + sizeof(hf);
    }
    return FC_OK;
}

fc_status rimp2_grad_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss, double* gamma,
                        double* de_docc, double* de_dvir, fc_stats* stats) {
    FC_TRY(fx_attrs());
    if (d.nocc > (1 << 15)) return fail(FC_ERR_LAYOUT, "split-BF16: nocc too large");
    const int64_t nocc = d.nocc, nvir = d.nvir, naux = d.naux, nov = nocc * nvir;
    void* vout;
    FC_TRY(ws_get(WS_OUT, (size_t)(2 * nocc + 16) * 8, &vout));
    double* e_chunks = (double*)vout;
    int* flags = (int*)(e_chunks + 2 * nocc + 8);
    FC_CUDA(cudaMemsetAsync(vout, 0, (size_t)(2 * nocc + 16) * 8, st));
    Context& c = ctx();
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    FxSplit sp;
    FC_TRY(fx_split_pairs(d, st, flags, &sp));
    const int64_t a_pad = sp.a_pad;
    const int64_t K2 = nocc * a_pad;                        // adjoint contraction length (j, b_pad)
    const int64_t q_rows = (naux + 127) / 128 * 128;
    // per-Q-row split of B_ov for the adjoint contraction
    const int64_t npairs_all = nocc * nocc;
    const int64_t ntile_all = (a_pad / fx::BM) * (a_pad / fx::BM + 1) / 2;
    const size_t tab_bytes = (((npairs_all + ntile_all) * sizeof(int2) + 255) / 256) * 256;
    void *vbq, *vtab;
    FC_TRY(ws_get(WS_SPLIT2, (size_t)3 * q_rows * K2 * 2, &vbq));
    FC_TRY(ws_get(WS_PAIRS, tab_bytes + q_rows * 8, &vtab));
    double* qs = (double*)((char*)vtab + tab_bytes);
    FC_CUDA(cudaMemsetAsync(vbq, 0, (size_t)3 * q_rows * K2 * 2, st));
    fill_kernel<<<(unsigned)((q_rows + 255) / 256), 256, 0, st>>>(qs, q_rows, 1.0);
    split_fx_qrows_kernel<<<(unsigned)naux, 256, 0, st>>>(d.b_ov, naux, nocc, nvir, a_pad, q_rows, qs,
                                                          (__nv_bfloat16*)vbq);
    FC_TRY(check_launch("split_fx_qrows_kernel"));
    CUtensorMap tmBq;
    FC_TRY(make_tmap_bf16_2d(&tmBq, vbq, K2, 3 * q_rows, K2 * 2, fx::KT, 128));

    // occupied chunk: ci rows of amplitudes, FP32 (written by the pair kernel)
    // and as three slices (read by the adjoint contraction)
    const int64_t per_i = a_pad * K2 * (4 + 6);
    int64_t ci = d.chunk_bytes / (per_i > 0 ? per_i : 1);
    if (ci < 1) ci = 1;
    if (ci > nocc) ci = nocc;
    const int nTa = (int)(a_pad / fx::BM), nTb = (int)(a_pad / fx::BN);
    const int ntiles = nTa * (nTa + 1) / 2;  // tiles ta <= tb (nTa == nTb)
    const int64_t items_per_i = nocc * (int64_t)ntiles;
    const size_t t_bytes = (size_t)ci * a_pad * K2 * 4;
    void *vT, *vTs, *vpart;
    FC_TRY(ws_get(WS_T, t_bytes + (size_t)ci * a_pad * 8, &vT));
    FC_TRY(ws_get(WS_TS, (size_t)3 * ci * a_pad * K2 * 2, &vTs));
    FC_TRY(ws_get(WS_PART, (size_t)ci * items_per_i * (2 + 1 + 2 * fx::BM) * 8, &vpart));
    float* T = (float*)vT;
    double* ts = (double*)((char*)vT + t_bytes);
    void* ts_slices = vTs;
    double* occ_part = (double*)vpart + ci * items_per_i * 2;
    double* vir_part = occ_part + ci * items_per_i;
    // pair table: ordered pairs, row-major by i; then every (a-tile, b-tile)
    std::vector<int2> pairs((size_t)npairs_all);
    for (int i = 0; i < nocc; ++i)
        for (int j = 0; j < nocc; ++j) pairs[(size_t)i * nocc + j] = make_int2(i, j);
    for (int ta = 0; ta < nTa; ++ta)
        for (int tb = ta; tb < nTb; ++tb) pairs.push_back(make_int2(ta, tb));
    FC_CUDA(cudaMemcpyAsync(vtab, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemsetAsync(de_dvir, 0, nvir * 8, st));

    CUtensorMap tmTs;
    FC_TRY(make_tmap_bf16_2d(&tmTs, ts_slices, K2, 3 * ci * a_pad, K2 * 2, fx::KT, 128));
    const int64_t nchunks = (nocc + ci - 1) / ci;
    cudaEvent_t* ev = nullptr;
    if (stats) FC_TRY(timing_events((int)(2 * nchunks), &ev));
    for (int64_t ch = 0; ch < nchunks; ++ch) {
        const int64_t i0 = ch * ci;
        const int64_t cn = i0 + ci <= nocc ? ci : nocc - i0;
        PairFxArgs a{};
        a.eo = d.eps_occ;
        a.ev = d.eps_vir;
        a.scl = sp.scl;
        a.pairs = (const int2*)vtab + i0 * nocc;
        a.tiles = (const int2*)vtab + npairs_all;
        a.ntiles = ntiles;
        a.npairs = (int)(cn * nocc);
        a.nocc = (int)nocc;
        a.nvir = (int)nvir;
        a.a_pad = (int)a_pad;
        a.nTa = nTa;
        a.nTb = nTb;
        a.nk = (int)(sp.q_pad / fx::KT);
        a.items = cn * items_per_i;
        a.part = (double*)vpart;
        a.err = flags + 1;
        a.T = T;
        a.ldt = K2;
        a.i0 = (int)i0;
        a.occ_part = occ_part;
        a.vir_part = vir_part;
        const int grid = (int)(a.items < c.sm_count ? a.items : c.sm_count);
        if (stats) FC_CUDA(cudaEventRecord(ev[2 * ch], st));
        pair_fx_kernel<1><<<grid, 320, fx::SMEM, st>>>(sp.tmA, sp.tmB, a);
        FC_TRY(check_launch("pair_fx_kernel<grad>"));
        if (stats) FC_CUDA(cudaEventRecord(ev[2 * ch + 1], st));
        fx_reduce_pairs_kernel<<<1, 1024, 0, st>>>((const double*)vpart, a.items, e_chunks + 2 * ch);
        fx_reduce_occ_kernel<<<(unsigned)cn, 256, 0, st>>>(occ_part, items_per_i, (int)i0, de_docc);
        fx_reduce_vir_kernel<<<(unsigned)((nvir + 7) / 8), 256, 0, st>>>(
            vir_part, (const int2*)vtab + npairs_all, cn * nocc, ntiles, (int)nvir, de_dvir);
        split_fx_rows_f32_kernel<<<(unsigned)(cn * a_pad), 256, 0, st>>>(T, K2, ci * a_pad, ts,
                                                                          (__nv_bfloat16*)ts_slices);
        FC_TRY(check_launch("gradient chunk reductions / split"));
        GemmFxArgs gargs{};
        gargs.rs = ts;
        gargs.cs = qs;
        gargs.M = (int)(ci * a_pad);   // slice stride of the chunk tensor map
        gargs.N = (int)q_rows;
        gargs.nk = (int)(K2 / fx::KT);
        gargs.nTm = (int)(cn * a_pad / 128);
        gargs.nTn = (int)(q_rows / 128);
        gargs.tiles = (int64_t)gargs.nTm * gargs.nTn;
        gargs.a_pad = (int)a_pad;
        gargs.nvir = (int)nvir;
        gargs.naux = (int)naux;
        gargs.i0 = (int)i0;
        gargs.nov = nov;
        gargs.alpha = 4.0;
        gargs.out = gamma;
        gargs.err = flags + 1;
        const int g2 = (int)(gargs.tiles < c.sm_count ? gargs.tiles : c.sm_count);
        gemm_fx_kernel<<<g2, 192, GF_SMEM, st>>>(tmTs, tmBq, gargs);
        FC_TRY(check_launch("gemm_fx_kernel"));
    }
    if (stats) FC_CUDA(cudaEventRecord(c.ev1, st));
    std::vector<double> h((size_t)(2 * nchunks));
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(h.data(), e_chunks, h.size() * 8, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "split-BF16: B_ov has a non-finite element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "split-BF16 gradient kernels: a pipeline wait ran out");
    double eo = 0.0, co = 0.0, es = 0.0, cs2 = 0.0;
    for (int64_t ch = 0; ch < nchunks; ++ch) {
        double v = h[2 * ch], t = eo + v;
        co += fabs(eo) >= fabs(v) ? (eo - t) + v : (v - t) + eo;
        eo = t;
        v = h[2 * ch + 1];
        t = es + v;
        cs2 += fabs(es) >= fabs(v) ? (es - t) + v : (v - t) + es;
        es = t;
    }
    *e_os = eo + co;
    *e_ss = es + cs2;
    if (stats) {
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        const double P = (double)nocc * (nocc + 1) / 2.0;
        stats->flops = 2.0 * naux * (double)nvir * nvir * P + 2.0 * naux * (double)nov * nov;
        stats->precision = FC_PREC_MIXED;
        stats->launches += (int)(6 * nchunks + 5);
        stats->tile_m = fx::BM;
        stats->tile_n = fx::BN;
        stats->main_launches = (int)nchunks;
        double tsum = 0.0;
        for (int64_t ch = 0; ch < nchunks; ++ch) {
            float x = 0.f;
            FC_CUDA(cudaEventElapsedTime(&x, ev[2 * ch], ev[2 * ch + 1]));
            tsum += x;
        }
        stats->main_ms = tsum;
        stats->main_flops = 2.0 * naux * (double)nov * nov;
        stats->main_bytes = 6.0 * naux * (double)nov * (double)nchunks;
        stats->h2d_bytes += pairs.size() * sizeof(int2);
        stats->d2h_bytes += h.size() * 8 + sizeof(hf);
    }
    return FC_OK;
}

}  // namespace fc
