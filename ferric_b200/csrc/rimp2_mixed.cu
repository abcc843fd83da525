// Split-BF16 RI-MP2 kernels on the 5th-generation tensor cores (tcgen05).
//
// Operands.  B_ov (FP64) is split once per call into TERMS bf16 terms,
//     x = hi + lo (+ mid),  hi = RN(x), lo = RN(x - hi), ...
// and stored transposed and padded as Bt[term][i][a_pad][q_pad] so every
// operand tile (128 virtual rows x 64 aux columns) is K-major with 128-byte
// rows: the canonical TMA / UMMA layout.  Padding rows and columns are zero.
//
// Products.  (ia|jb) = sum over term pairs with combined weight above the
// dropped ones: TERMS = 2 -> hi*hi + hi*lo + lo*hi (3 products),
// TERMS = 3 -> hh + hm + mh + hl + lh + mm (6 products); FP32 accumulation
// in TMEM over the whole aux range, the denominator and the energy sums in
// FP64 (compensated) in the epilogue.  (ia|jb) never reaches HBM.
//
// Work item = (pair i <= j, a-tile, b-tile), 128 x 128.  For i < j the item
// accumulates X = (ia|jb) and Y = (ib|ja) = G_ji[a, b] in two TMEM
// accumulators (X phase then Y phase over the same smem ring), so the
// exchange partner of every element is in the same TMEM lane and column:
//     E_OS += (X^2 + Y^2)/D,  E_SS += (X - Y)^2/D
// For i == j, G_ii is symmetric: only a-tile <= b-tile, X phase only, weight 2
// off the tile diagonal, and E_SS = 0 (ferric-mp2/src/rimp2.rs:1399-1441,
// 1506-1544 summed over both orderings of every pair).
//
// Warp roles (192 threads, one CTA per SM, persistent, static round-robin
// over items): warp 0 TMA producer, warp 1 TMEM owner and UMMA issuer,
// warps 2-5 epilogue (TMEM lane quadrant = warp % 4).  TMEM holds two
// 256-column accumulator sets so the epilogue of one item overlaps the MMAs
// of the next.
#include "fc_internal.cuh"
#include "rimp2.cuh"
#include "tc.cuh"
#include "tmap.cuh"

namespace fc {

constexpr int TC_TILE = 128;  // virtual rows per tile
constexpr int TC_KT = 64;     // aux columns per pipeline stage (128-byte rows)
constexpr int TC_TILE_BYTES = TC_TILE * TC_KT * 2;
constexpr uint32_t TC_IDESC = tc::idesc_bf16_f32(128, 128);

template <int TERMS>
struct TcCfg {
    static constexpr int STAGES = TERMS == 2 ? 3 : 2;
    static constexpr int STAGE_BYTES = 2 * TERMS * TC_TILE_BYTES;
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 /*align*/ + 512 /*barriers etc*/;
    static constexpr int NPROD = TERMS == 2 ? 3 : 6;
};

// (A term, B term) of each product, largest first.
__constant__ int8_t kProdA[6] = {0, 0, 1, 0, 2, 1};
__constant__ int8_t kProdB[6] = {0, 1, 0, 2, 0, 1};

// ---------------------------------------------------------------- split --

// B[q, ia] (FP64, naux x nov) -> Bt[t][i][a][q] bf16 terms (a < a_pad, q < q_pad).
// Flags non-finite or out-of-bf16-range inputs in *range_flag.
template <int TERMS>
__global__ void __launch_bounds__(256) split_transpose_kernel(const double* __restrict__ B, int64_t naux,
                                                              int64_t nocc, int64_t nvir, int64_t a_pad,
                                                              int64_t q_pad, __nv_bfloat16* __restrict__ Bt,
                                                              int* range_flag) {
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
    const int64_t term_stride = nocc * a_pad * q_pad;
    bool bad = false;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int idx = tid + 256 * e, c = idx >> 5, qq = (idx & 31) * 2;
        const int64_t ia = ia0 + c;
        if (ia >= nov) continue;
        const int64_t i = ia / nvir, a = ia % nvir;
        const double x0 = tile[qq][c], x1 = tile[qq + 1][c];
        bad |= !(fabs(x0) <= 3.0e38) || !(fabs(x1) <= 3.0e38);
        __nv_bfloat16 h0 = __double2bfloat16(x0), h1 = __double2bfloat16(x1);
        double r0 = x0 - (double)__bfloat162float(h0), r1 = x1 - (double)__bfloat162float(h1);
        __nv_bfloat16 m0 = __double2bfloat16(r0), m1 = __double2bfloat16(r1);
        const int64_t off = (i * a_pad + a) * q_pad + q0 + qq;
        *reinterpret_cast<__nv_bfloat162*>(Bt + off) = __halves2bfloat162(h0, h1);
        *reinterpret_cast<__nv_bfloat162*>(Bt + term_stride + off) = __halves2bfloat162(m0, m1);
        if (TERMS == 3) {
            r0 -= (double)__bfloat162float(m0);
            r1 -= (double)__bfloat162float(m1);
            *reinterpret_cast<__nv_bfloat162*>(Bt + 2 * term_stride + off) =
                __halves2bfloat162(__double2bfloat16(r0), __double2bfloat16(r1));
        }
    }
    if (bad) atomicOr(range_flag, 1);
}

// ------------------------------------------------------------ pair kernel --

struct PairTcArgs {
    const double* eo;
    const double* ev;
    const int2* pairs;   // off-diagonal pairs (i < j)
    const int2* dtiles;  // (ta, tb), ta <= tb, for diagonal pairs
    int n_off, nd;
    int nocc, nvir, a_pad, nT, nk;
    int64_t items;
    double* part;  // [item][2]
    int* err;
};

struct ItemDesc {
    int i, j, ta, tb;
    bool diag;
    double w;
};

__device__ __forceinline__ ItemDesc decode_item(const PairTcArgs& p, int64_t k) {
    ItemDesc d;
    const int64_t t2 = (int64_t)p.nT * p.nT;
    const int64_t noff = (int64_t)p.n_off * t2;
    if (k < noff) {
        const int64_t pi = k / t2, r = k % t2;
        const int2 ij = p.pairs[pi];
        d.i = ij.x;
        d.j = ij.y;
        d.ta = (int)(r / p.nT);
        d.tb = (int)(r % p.nT);
        d.diag = false;
        d.w = 1.0;
    } else {
        const int64_t k2 = k - noff;
        d.i = d.j = (int)(k2 / p.nd);
        const int2 tt = p.dtiles[k2 % p.nd];
        d.ta = tt.x;
        d.tb = tt.y;
        d.diag = true;
        d.w = tt.x < tt.y ? 2.0 : 1.0;
    }
    return d;
}

template <int TERMS>
__global__ void __launch_bounds__(192, 1)
    pair_tc_kernel(const __grid_constant__ CUtensorMap tmap, const PairTcArgs p) {
    using Cfg = TcCfg<TERMS>;
    constexpr int S = Cfg::STAGES;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw_u32 = smem_u32(smem_raw);
    const uint32_t base_u32 = (raw_u32 + 1023u) & ~1023u;
    uint8_t* base = smem_raw + (base_u32 - raw_u32);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S * Cfg::STAGE_BYTES);
    uint64_t* full = bars;               // [S]
    uint64_t* empty = bars + S;          // [S]
    uint64_t* tfull = bars + 2 * S;      // [2]
    uint64_t* tempty = bars + 2 * S + 2; // [2]
    uint64_t* drain = bars + 2 * S + 4;  // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 5);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    double* red = reinterpret_cast<double*>(bars + 2 * S + 6);  // [2][4][2]

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&tfull[b], 1);
            tc::mbar_init(&tempty[b], 128);
        }
        tc::mbar_init(drain, 1);
        *abort_flag = 0;
        tc::fence_barrier_init();
    }
    if (warp == 0 && lane == 0) tc::prefetch_tmap(&tmap);
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 512);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    auto stage_a = [&](int s, int t) { return base_u32 + s * Cfg::STAGE_BYTES + t * TC_TILE_BYTES; };
    auto stage_b = [&](int s, int t) { return base_u32 + s * Cfg::STAGE_BYTES + (TERMS + t) * TC_TILE_BYTES; };
    auto row_of = [&](int t, int i, int tile) { return (t * p.nocc + i) * p.a_pad + tile * TC_TILE; };

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t g = 0;
            for (int64_t k = blockIdx.x; k < p.items && !*abort_flag; k += gridDim.x) {
                const ItemDesc d = decode_item(p, k);
                const int nph = d.diag ? 1 : 2;
                for (int ph = 0; ph < nph; ++ph) {
                    const int ia = ph == 0 ? d.i : d.j, ib = ph == 0 ? d.j : d.i;
                    for (int kt = 0; kt < p.nk; ++kt, ++g) {
                        const int s = g % S;
                        const uint32_t u = g / S;
                        if (!tc::mbar_wait(&empty[s], (u & 1) ^ 1, abort_flag, p.err)) goto prod_done;
                        tc::mbar_arrive_expect_tx(&full[s], Cfg::STAGE_BYTES);
#pragma unroll
                        for (int t = 0; t < TERMS; ++t) {
                            tc::tma_load_2d(base + (stage_a(s, t) - base_u32), &tmap, &full[s], kt * TC_KT,
                                            row_of(t, ia, d.ta));
                            tc::tma_load_2d(base + (stage_b(s, t) - base_u32), &tmap, &full[s], kt * TC_KT,
                                            row_of(t, ib, d.tb));
                        }
                    }
                }
            }
        prod_done:
            // drain: loads issued into the last stages must land before exit
            for (uint32_t q = 0; q < (uint32_t)S && q < g; ++q) {
                const uint32_t gg = g - 1 - q;
                int dummy_abort = 0;
                tc::mbar_wait(&full[gg % S], (gg / S) & 1, &dummy_abort, p.err);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------ UMMA issuer
        if (lane == 0) {
            uint32_t g = 0, li = 0;
            for (int64_t k = blockIdx.x; k < p.items && !*abort_flag; k += gridDim.x, ++li) {
                const ItemDesc d = decode_item(p, k);
                const int buf = li & 1;
                if (!tc::mbar_wait(&tempty[buf], ((li >> 1) & 1) ^ 1, abort_flag, p.err)) break;
                tc::fence_after_sync();
                const int nph = d.diag ? 1 : 2;
                for (int ph = 0; ph < nph; ++ph) {
                    const uint32_t dcol = tmem_base + buf * 256 + ph * 128;
                    for (int kt = 0; kt < p.nk; ++kt, ++g) {
                        const int s = g % S;
                        const uint32_t u = g / S;
                        if (!tc::mbar_wait(&full[s], u & 1, abort_flag, p.err)) goto mma_done;
                        tc::fence_after_sync();
#pragma unroll
                        for (int pr = 0; pr < Cfg::NPROD; ++pr) {
                            const uint32_t a0 = stage_a(s, kProdA[pr]);
                            const uint32_t b0 = stage_b(s, kProdB[pr]);
#pragma unroll
                            for (int kk = 0; kk < TC_KT / 16; ++kk) {
                                tc::umma_bf16(dcol, tc::sdesc_k128(a0 + kk * 32), tc::sdesc_k128(b0 + kk * 32),
                                              TC_IDESC, (kt | pr | kk) != 0);
                            }
                        }
                        tc::umma_commit(&empty[s]);
                    }
                }
                tc::umma_commit(&tfull[buf]);
            }
        mma_done:
            tc::umma_commit(drain);
            int dummy_abort = 0;
            tc::mbar_wait(drain, 0, &dummy_abort, p.err);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------ epilogue
        const int q = warp & 3;
        const int row = q * 32 + lane;
        const int et = tid - 64;  // 0..127
        uint32_t li = 0;
        for (int64_t k = blockIdx.x; k < p.items; k += gridDim.x, ++li) {
            const ItemDesc d = decode_item(p, k);
            const int buf = li & 1;
            // one thread waits (bounded); the 128 epilogue threads leave together if
            // it gave up, since a named barrier follows
            if (!tc::bar_and<1, 128>(et != 0 || tc::mbar_wait(&tfull[buf], (li >> 1) & 1, abort_flag, p.err)))
                break;
            if (et != 0) tc::mbar_wait(&tfull[buf], (li >> 1) & 1, abort_flag, p.err);
            tc::fence_after_sync();
            const int a = d.ta * TC_TILE + row;
            const bool va = a < p.nvir;
            const double dA = p.eo[d.i] + p.eo[d.j] - (va ? p.ev[a] : 0.0);
            KSum os, ss;
            const uint32_t tl = tmem_base + ((uint32_t)(q * 32) << 16) + buf * 256;
#pragma unroll 1
            for (int c0 = 0; c0 < TC_TILE; c0 += 32) {
                float xv[32], yv[32];
                tc::tmem_ld32(tl + c0, xv);
                if (!d.diag) tc::tmem_ld32(tl + 128 + c0, yv);
                tc::tmem_wait_ld();
                if (va) {
                    const int bmax = p.nvir - (d.tb * TC_TILE + c0);
#pragma unroll
                    for (int cc = 0; cc < 32; ++cc) {
                        if (cc < bmax) {
                            const double D = dA - p.ev[d.tb * TC_TILE + c0 + cc];
                            const double r = 1.0 / D;
                            const double x = xv[cc];
                            if (d.diag) {
                                os.add(x * x * r);
                            } else {
                                const double y = yv[cc];
                                os.add((x * x + y * y) * r);
                                ss.add((x - y) * (x - y) * r);
                            }
                        }
                    }
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&tempty[buf]);
            // fixed-order reduction over the 128 epilogue threads
            const double vo = warp_sum(os.value()), vs = warp_sum(ss.value());
            double* rb = red + (li & 1) * 8;
            if (lane == 0) {
                rb[(warp - 2) * 2 + 0] = vo;
                rb[(warp - 2) * 2 + 1] = vs;
            }
            asm volatile("bar.sync 1, 128;" ::: "memory");
            if (et == 0) {
                double so = 0.0, sn = 0.0;
#pragma unroll
                for (int w = 0; w < 4; ++w) {
                    so += rb[w * 2];
                    sn += rb[w * 2 + 1];
                }
                p.part[2 * k] = d.w * so;
                p.part[2 * k + 1] = d.w * sn;
            }
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

__global__ void __launch_bounds__(1024) reduce_parts_kernel(const double* __restrict__ part, int64_t n,
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

// ------------------------------------------------------------------ host --

struct SplitB {
    __nv_bfloat16* bt;
    int64_t a_pad, q_pad;
    CUtensorMap tmap;
};

template <int TERMS>
static fc_status split_b(const Rimp2Dev& d, cudaStream_t st, int* range_flag, SplitB* out) {
    const int64_t a_pad = (d.nvir + TC_TILE - 1) / TC_TILE * TC_TILE;
    const int64_t q_pad = (d.naux + TC_KT - 1) / TC_KT * TC_KT;
    const int64_t rows = (int64_t)TERMS * d.nocc * a_pad;
    const size_t bytes = (size_t)rows * q_pad * 2;
    void* p;
    FC_TRY(ws_get(WS_SPLIT, bytes, &p));  // FC_PREC_MIXED_FAST operands
    FC_CUDA(cudaMemsetAsync(p, 0, bytes, st));
    const int64_t nov = d.nocc * d.nvir;
    dim3 g((unsigned)((nov + 63) / 64), (unsigned)((d.naux + 63) / 64));
    if (g.y > 65535) return fail(FC_ERR_LAYOUT, "split: naux too large");
    split_transpose_kernel<TERMS><<<g, 256, 0, st>>>(d.b_ov, d.naux, d.nocc, d.nvir, a_pad, q_pad,
                                                      (__nv_bfloat16*)p, range_flag);
    FC_TRY(check_launch("split_transpose_kernel"));
    out->bt = (__nv_bfloat16*)p;
    out->a_pad = a_pad;
    out->q_pad = q_pad;
    if (rows > (int64_t)UINT32_MAX) return fail(FC_ERR_LAYOUT, "split: too many operand rows for TMA");
    FC_TRY(make_tmap_bf16_2d(&out->tmap, p, (uint64_t)q_pad, (uint64_t)rows, (uint64_t)q_pad * 2, TC_KT,
                             TC_TILE));
    return FC_OK;
}

template <int TERMS>
static fc_status energy_mixed_impl(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                                   fc_stats* stats) {
    using Cfg = TcCfg<TERMS>;
    static bool attr = false;
    if (!attr) {
        FC_CUDA(cudaFuncSetAttribute(pair_tc_kernel<TERMS>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
        attr = true;
    }
    void* vout;
    FC_TRY(ws_get(WS_OUT, 256, &vout));
    double* out = (double*)vout;           // [0..1] energies
    int* flags = (int*)(out + 4);          // [0] range, [1] timeout
    FC_CUDA(cudaMemsetAsync(vout, 0, 256, st));
    SplitB sb;
    Context& c = ctx();
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    FC_TRY(split_b<TERMS>(d, st, flags, &sb));

    const int nT = (int)(sb.a_pad / TC_TILE);
    const int nocc = (int)d.nocc;
    std::vector<int2> tab;
    for (int i = 0; i < nocc; ++i)
        for (int j = i + 1; j < nocc; ++j) tab.push_back(make_int2(i, j));
    const int n_off = (int)tab.size();
    for (int a = 0; a < nT; ++a)
        for (int b = a; b < nT; ++b) tab.push_back(make_int2(a, b));
    const int nd = (int)tab.size() - n_off;
    void* vtab;
    FC_TRY(ws_get(WS_PAIRS, tab.size() * sizeof(int2), &vtab));
    FC_CUDA(cudaMemcpyAsync(vtab, tab.data(), tab.size() * sizeof(int2), cudaMemcpyHostToDevice, st));

    PairTcArgs a{};
    a.eo = d.eps_occ;
    a.ev = d.eps_vir;
    a.pairs = (const int2*)vtab;
    a.dtiles = (const int2*)vtab + n_off;
    a.n_off = n_off;
    a.nd = nd;
    a.nocc = nocc;
    a.nvir = (int)d.nvir;
    a.a_pad = (int)sb.a_pad;
    a.nT = nT;
    a.nk = (int)(sb.q_pad / TC_KT);
    a.items = (int64_t)n_off * nT * nT + (int64_t)nocc * nd;
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
    pair_tc_kernel<TERMS><<<grid, 192, Cfg::SMEM, st>>>(sb.tmap, a);
    FC_TRY(check_launch("pair_tc_kernel"));
    if (stats) FC_CUDA(cudaEventRecord(ev[1], st));
    reduce_parts_kernel<<<1, 1024, 0, st>>>((const double*)vpart, a.items, out);
    FC_TRY(check_launch("reduce_parts_kernel"));
    if (stats) FC_CUDA(cudaEventRecord(c.ev1, st));
    double h[4];
    int hf[2];
    FC_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    if (hf[0]) return fail(FC_ERR_RANGE, "split-BF16: B_ov has a non-finite element or one beyond the bf16 range");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "split-BF16 pair kernel: a pipeline wait ran out (device error)");
    *e_os = h[0];
    *e_ss = h[1];
    if (stats) {
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        const double P = (double)d.nocc * (d.nocc + 1) / 2.0;
        stats->flops = 2.0 * (double)d.naux * (double)d.nvir * (double)d.nvir * P;
        stats->precision = FC_PREC_MIXED_FAST;
        stats->launches += 3;
        stats->tile_m = TC_TILE;
        stats->tile_n = TC_TILE;
        stats->k_panel = 0;
        stats->main_launches = 1;
        FC_TRY(timing_sum(1, &stats->main_ms));
        stats->main_flops = stats->flops;
        stats->main_bytes = (double)TERMS * 2.0 * (double)d.naux * (double)(d.nocc * d.nvir);
        stats->h2d_bytes += tab.size() * sizeof(int2);
        stats->d2h_bytes += sizeof(h) + sizeof(hf);
    }
    return FC_OK;
}

fc_status rimp2_energy_mixed(const Rimp2Dev& d, int terms, cudaStream_t st, double* e_os, double* e_ss,
                             fc_stats* stats) {
    if (d.nocc > (1 << 16)) return fail(FC_ERR_LAYOUT, "split-BF16: nocc too large");
    (void)terms;
    return energy_mixed_impl<2>(d, st, e_os, e_ss, stats);
}

}  // namespace fc
