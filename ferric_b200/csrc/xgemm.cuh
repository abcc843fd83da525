// Generic exact-slice GEMM on tcgen05 with a k-panel flush:
//     C[m, n] = sum_k A[m, k] B[n, k]
// for A, B given as three integer slices each (the exact split of
// fx_split.cuh; row scales are applied by the epilogue functor): bf16 slices
// (weights 1/256, tcgen05.mma kind::f16, FP32 accumulators) or, with I8,
// int8 slices (weights 1/254, kind::i8, int32 accumulators).  A k-step is
// 128 bytes of each operand row either way (64 bf16 or 128 int8 elements).
//
// Each work item is (m-tile of 128 rows, n-tile of BN rows, first k-step,
// k-steps); a persistent CTA takes items round-robin.  The MMA warp
// accumulates the three product levels
//     L0 = c1 c1',  L1 = c1 c2' + c2 c1',  L2 = c1 c3' + c2 c2' + c3 c1'
// in TMEM over a panel of at most KP = 8 k-steps (512 of K): every FP32 level
// sum is then an integer of magnitude below 2^24 (at most 512 * 3 * 2^14),
// i.e. exact.  The epilogue warps drain each panel into FP64 registers,
//     acc += L0 + L1 / 256 + L2 / 65536     (exact in FP64),
// so the result is exact up to the slicing itself for any K -- the
// k-panelled FP64 flush of the reference's mixed GEMM
// (ferric-core/src/gpu/mixed.rs:122-192), here inside one kernel.  The
// int8 form's panels (1024 of K) are far inside its int32 range
// (3 * 127^2 * 1024 < 2^26) and combine as L0 + L1 / 254 + L2 / 254^2.
//
// Where an item's rows are is the loader policy's (Ld): LdTiles takes the
// m-tile / n-tile of a 2-D map per slice; LdRows takes first rows it.x / it.y
// directly (tiles at any row); LdPlanes takes one row (it.z) of each of 128
// planes of a 3-D map (rows strided by a plane: the occupied index of an
// amplitude slab at fixed virtual).  LdRows and LdPlanes are int8 only and
// let a panel run 256 k-steps: 3 * 127^2 * 32768 < 2^31 keeps every int32
// level sum exact, so one drain per item suffices for K <= 32768.
//
// Roles: warp 0 TMA producer, warp 1 UMMA issuer, warps 2 .. 2 + BN/8 - 1
// epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows) and
// columns 32 ((w - 2) / 4) .. + 31 of each level.  With BN = 64 two
// accumulator sets alternate (6 x 64 of the 512 TMEM columns), so the drain
// of one panel overlaps the next panel's MMAs.
#pragma once
#include <cuda.h>
#include <cstdint>

#include "fc_internal.cuh"
#include "tc.cuh"

namespace fc {
namespace xg {

constexpr int BM = 128, KT = 64, KP = 8;
constexpr double L1W = 1.0 / 256.0, L2W = 1.0 / 65536.0;
constexpr double I8L1W = 1.0 / 254.0, I8L2W = 1.0 / (254.0 * 254.0);


template <int BN, bool I8 = false>
struct Cfg {
    static_assert(BN == 64 || BN == 128, "BN is 64 or 128");
    static constexpr int KTE = I8 ? 2 * KT : KT;   // elements of K per k-step (128 bytes)
    static constexpr int A_BYTES = BM * KT * 2;
    static constexpr int B_BYTES = BN * KT * 2;
    static constexpr int STAGE = 3 * (A_BYTES + B_BYTES);
    static constexpr int STAGES = BN == 128 ? 2 : 3;
    static constexpr int NEW = BN / 8;             // epilogue warps
    static constexpr int THREADS = 64 + 32 * NEW;
    static constexpr int NSET = BN == 64 ? 2 : 1;  // TMEM accumulator sets
    static constexpr int TCOLS = NSET * 3 * BN <= 256 ? 256 : 512;
    static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
    static constexpr uint32_t IDESC = I8 ? tc::idesc_i8_s32(128, BN) : tc::idesc_bf16_f32(128, BN);
    static constexpr uint32_t IDESC2 = I8 ? tc::idesc_i8_s32(128, 2 * BN) : tc::idesc_bf16_f32(128, 2 * BN);
};

}  // namespace xg

struct XArgs {
    const int4* items;  // (m-tile, n-tile, first k-step, k-steps) for LdTiles
    int64_t nitems;
    int Ma, Nb;  // rows (LdPlanes: planes) between the slices of the A and B tensor maps
    int* err;
    int nka;     // LdKBlocksA: k-blocks of A per slice
};

struct LdTiles {
    static constexpr int KP = xg::KP;
    __device__ static int k0(int4 it) { return it.z; }
    template <int BN, int KTE>
    __device__ static void load(void* da, void* db, const CUtensorMap* ta, const CUtensorMap* tb, uint64_t* bar,
                                const XArgs& p, int4 it, int kt, int sl) {
        tc::tma_load_2d(da, ta, bar, kt * KTE, sl * p.Ma + it.x * xg::BM);
        tc::tma_load_2d(db, tb, bar, kt * KTE, sl * p.Nb + it.y * BN);
    }
};

// A in 128-byte column blocks ([slice][k-block][Ma rows][128 B], a 2-D map
// 128 bytes wide), B as LdTiles.
struct LdKBlocksA {
    static constexpr int KP = xg::KP;
    __device__ static int k0(int4 it) { return it.z; }
    template <int BN, int KTE>
    __device__ static void load(void* da, void* db, const CUtensorMap* ta, const CUtensorMap* tb, uint64_t* bar,
                                const XArgs& p, int4 it, int kt, int sl) {
        tc::tma_load_2d(da, ta, bar, 0, (sl * p.nka + kt) * p.Ma + it.x * xg::BM);
        tc::tma_load_2d(db, tb, bar, kt * KTE, sl * p.Nb + it.y * BN);
    }
};

struct LdRows {  // item (A row, B row, first k-step, k-steps)
    static constexpr int KP = 256;
    __device__ static int k0(int4 it) { return it.z; }
    template <int BN, int KTE>
    __device__ static void load(void* da, void* db, const CUtensorMap* ta, const CUtensorMap* tb, uint64_t* bar,
                                const XArgs& p, int4 it, int kt, int sl) {
        tc::tma_load_2d(da, ta, bar, kt * KTE, sl * p.Ma + it.x);
        tc::tma_load_2d(db, tb, bar, kt * KTE, sl * p.Nb + it.y);
    }
};

struct LdPlanes {  // item (A plane tile, B plane tile, row in every plane, k-steps from 0)
    static constexpr int KP = 256;
    __device__ static int k0(int4) { return 0; }
    template <int BN, int KTE>
    __device__ static void load(void* da, void* db, const CUtensorMap* ta, const CUtensorMap* tb, uint64_t* bar,
                                const XArgs& p, int4 it, int kt, int sl) {
        tc::tma_load_3d(da, ta, bar, kt * KTE, it.z, sl * p.Ma + it.x * xg::BM);
        tc::tma_load_3d(db, tb, bar, kt * KTE, it.z, sl * p.Nb + it.y * BN);
    }
};

// Epi: __device__ void operator()(int64_t item, int4 it, int row, int col0,
//                                 const double (&acc)[32]) const
template <int BN, class Epi, bool I8 = false, class Ld = LdTiles>
__global__ void __launch_bounds__(xg::Cfg<BN, I8>::THREADS, 1)
    xgemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const XArgs p,
                 const Epi epi) {
    using C = xg::Cfg<BN, I8>;
    using namespace xg;
    constexpr int S = C::STAGES, NS = C::NSET, KP = Ld::KP;
    static_assert(I8 || KP == xg::KP, "FP32 level sums are exact over 8 k-steps only");
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_u32 = smem_u32(smem_raw);
    const uint32_t base_u32 = (raw_u32 + 1023u) & ~1023u;
    uint8_t* base = smem_raw + (base_u32 - raw_u32);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * C::STAGE);
    uint64_t* full = bars;                 // [S]
    uint64_t* empty = bars + S;            // [S]
    uint64_t* tfull = bars + 2 * S;        // [NS]
    uint64_t* tempty = bars + 2 * S + 2;   // [NS]
    uint64_t* drain = bars + 2 * S + 4;    // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < NS; ++b) {
            tc::mbar_init(&tfull[b], 1);
            tc::mbar_init(&tempty[b], 32 * C::NEW);
        }
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) {
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, C::TCOLS);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;
    auto sa = [&](int s, int sl) { return base_u32 + s * C::STAGE + sl * C::A_BYTES; };
    auto sb = [&](int s, int sl) { return base_u32 + s * C::STAGE + 3 * C::A_BYTES + sl * C::B_BYTES; };

    if (warp == 0) {
        if (lane == 0) {
            uint32_t g = 0;
            for (int64_t t = blockIdx.x; t < p.nitems && !*abort_flag; t += gridDim.x) {
                const int4 it = p.items[t];
                const int kb = Ld::k0(it);
                for (int kt = kb; kt < kb + it.w; ++kt, ++g) {
                    const int s = g % S;
                    const uint32_t u = g / S;
                    if (!tc::mbar_wait(&empty[s], (u & 1) ^ 1, abort_flag, p.err)) goto prod_done;
                    tc::mbar_arrive_expect_tx(&full[s], C::STAGE);
#pragma unroll
                    for (int sl = 0; sl < 3; ++sl)
                        Ld::template load<BN, C::KTE>(base + (sa(s, sl) - base_u32), base + (sb(s, sl) - base_u32),
                                                      &tmA, &tmB, &full[s], p, it, kt, sl);
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
            uint32_t g = 0, pc = 0;  // k-steps consumed, panels issued
            for (int64_t t = blockIdx.x; t < p.nitems && !*abort_flag; t += gridDim.x) {
                const int4 it = p.items[t];
                for (int k0 = 0; k0 < it.w; k0 += KP, ++pc) {
                    const int b = (int)(pc % NS);
                    const uint32_t u = pc / NS;
                    if (!tc::mbar_wait(&tempty[b], (u & 1) ^ 1, abort_flag, p.err)) goto mma_done;
                    tc::fence_after_sync();
                    const uint32_t dset = tmem_base + b * 3 * BN;
                    const int k1 = k0 + KP < it.w ? k0 + KP : it.w;
                    for (int kq = k0; kq < k1; ++kq, ++g) {
                        const int s = g % S;
                        const uint32_t uu = g / S;
                        if (!tc::mbar_wait(&full[s], uu & 1, abort_flag, p.err)) goto mma_done;
                        tc::fence_after_sync();
                        // four MMAs: A0 B0 (level 0), A0 [B1; B2] (levels 1, 2: the B
                        // slices are adjacent, BN rows apart, and so are the levels in
                        // TMEM, so one N = 2 BN MMA reads A0 once for both), A1 [B0; B1]
                        // (levels 1, 2), A2 B0 (level 2); the first two start the levels
                        constexpr int kXA[4] = {0, 0, 1, 2}, kXB[4] = {0, 1, 0, 0};
#pragma unroll
                        for (int pr = 0; pr < 4; ++pr) {
                            const uint32_t a0 = sa(s, kXA[pr]), b0 = sb(s, kXB[pr]);
                            const uint32_t dcol = dset + (kXA[pr] + kXB[pr]) * BN;
#pragma unroll
                            for (int kk = 0; kk < 4; ++kk) {  // 32 bytes of K per MMA
                                const uint32_t acc = (kq > k0 || kk > 0 || pr > 1) ? 1u : 0u;
                                const uint32_t id = (pr == 1 || pr == 2) ? C::IDESC2 : C::IDESC;
                                if constexpr (I8)
                                    tc::umma_i8(dcol, tc::sdesc_k128(a0 + kk * 32), tc::sdesc_k128(b0 + kk * 32),
                                                id, acc);
                                else
                                    tc::umma_bf16(dcol, tc::sdesc_k128(a0 + kk * 32), tc::sdesc_k128(b0 + kk * 32),
                                                  id, acc);
                            }
                        }
                        tc::umma_commit(&empty[s]);
                    }
                    tc::umma_commit(&tfull[b]);
                }
            }
        mma_done:
            tc::umma_commit(drain);
            int no_abort = 0;
            tc::mbar_wait(drain, 0, &no_abort, p.err);
        }
        __syncwarp();
    } else {
        const int q = warp & 3;            // TMEM lane quarter of this warp
        const int cg = (warp - 2) >> 2;    // column group of 32
        const int row = q * 32 + lane;
        const uint32_t tl = tmem_base + ((uint32_t)(q * 32) << 16) + cg * 32;
        uint32_t pc = 0;
        bool ok = true;
        for (int64_t t = blockIdx.x; t < p.nitems && ok; t += gridDim.x) {
            const int4 it = p.items[t];
            double acc[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) acc[c] = 0.0;
            for (int k0 = 0; k0 < it.w; k0 += KP, ++pc) {
                const int b = (int)(pc % NS);
                const uint32_t u = pc / NS;
                if (!tc::mbar_wait(&tfull[b], u & 1, abort_flag, p.err)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t ts = tl + b * 3 * BN;
#pragma unroll
                for (int c0 = 0; c0 < 32; c0 += 8) {
                    float l0[8], l1[8], l2[8];
                    tc::tmem_ld8(ts + c0, l0);
                    tc::tmem_ld8(ts + BN + c0, l1);
                    tc::tmem_ld8(ts + 2 * BN + c0, l2);
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int cc = 0; cc < 8; ++cc) {
                        if constexpr (I8)
                            acc[c0 + cc] += tc::i32_to_f64(l0[cc]) + tc::i32_to_f64(l1[cc]) * I8L1W +
                                            tc::i32_to_f64(l2[cc]) * I8L2W;
                        else
                            acc[c0 + cc] += (double)l0[cc] + (double)l1[cc] * L1W + (double)l2[cc] * L2W;
                    }
                }
                tc::fence_before_sync();
                tc::mbar_arrive(&tempty[b]);
            }
            if (ok) epi(t, it, row, cg * 32, acc);
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 1) {
        __syncwarp();
        tc::tmem_dealloc(tmem_base, C::TCOLS);
    }
}

}  // namespace fc
