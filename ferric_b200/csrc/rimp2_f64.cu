// All-FP64 RI-MP2 kernels (the drop-in "plain" set).
//
// Work item = (occupied pair, a-tile, b-tile) of 64 x 64 virtual indices.
// For the pair (i, j) the item forms two tiles of the pair block on the DMMA
// tensor path, both in (a, b) orientation:
//     X[a, b] = (ia|jb) = sum_Q B[Q, i a] B[Q, j b]
//     Y[a, b] = (ib|ja) = sum_Q B[Q, j a] B[Q, i b]
// so the exchange partner of every element sits in the same thread and no
// transpose is needed.  The orbital-energy denominator and the energy sums
// are applied in the epilogue: (ia|jb) never reaches HBM.
//
// Energy mode (unordered pairs i <= j, weight 1/2 on i == j):
//     E_OS += (X^2 + Y^2) / D,   E_SS += (X - Y)^2 / D
// which is the reference's pair loop over the (i, j) and (j, i) orderings
// (ferric-mp2/src/rimp2.rs:1399-1441, 1506-1544).
//
// Gradient mode (unordered pairs of an occupied chunk pair (I, J)): the item
// writes Tt_ij[a, b] = (2X - Y)/D into the amplitude rows of i and, for
// i < j, Tt_ji[a, b] = (2Y - X)/D into the rows of j, plus the partials of
// c = t Tt of both orderings for dE/d eps (ferric-mp2/src/oo_rimp2.rs:1170-1191);
// the second contraction Gamma[:, I] += 4 B[:, J] Tt_IJ^T (and the same for J)
// runs in dgemm_tn.
//
// Cross-spin mode (unrestricted alpha-beta energy): X = G_iJ of two tensors,
// E_ab += X^2 / D (ferric-mp2/src/u_rimp2.rs:731-753).
#include <algorithm>

#include "fc_internal.cuh"
#include "dmma.cuh"
#include "dgemm_tn.cuh"
#include "rimp2.cuh"

namespace fc {

constexpr int PR_T = 64, PR_BK = 16, PR_LD = 68, PR_STAGES = 3;
constexpr int PR_SMEM = PR_STAGES * 4 * PR_BK * PR_LD * 8;  // 104,448 B

struct PairArgs {
    const double* B;
    int64_t ldb;
    int naux, nvir;
    const double* eo;
    const double* ev;
    const int2* pairs;
    const int2* tiles;  // (a-tile, b-tile) of each item of a pair
    int ntiles;         // items per pair
    int has_kappa;
    double kappa;
    double* part;  // [item][2] energy partials
    // gradient mode: unordered pairs (i, j), i in chunk I (from i0), j in chunk J (from j0)
    double* T;         // amplitude rows of I: [|I| nvir][ldt = |J| nvir]
    double* T2;        // amplitude rows of J: [|J| nvir][ldt2 = |I| nvir] (T when I == J)
    int64_t ldt, ldt2;
    int i0, j0;
    double* occ_part;  // [item][2]: t Tt summed for the orderings (i, j) and (j, i)
    double* vir_part;  // [item][64]: row-virtual sums of both orderings
    // cross-spin mode (MODE 2): pairs (i alpha, J beta), G = B_alpha_i^T B_beta_J
    const double* B2;
    int64_t ldb2;
    int nvir2;
    const double* eo2;
    const double* ev2;
};

// GRAD: 0 energy (unique pairs, X and Y = G_ji), 1 gradient, 2 cross-spin
// energy (X = G_iJ of B_alpha and B_beta only, E_ab += X^2 / D).
template <int GRAD>
__global__ void __launch_bounds__(256, 2) pair_f64_kernel(PairArgs p) {
    constexpr bool CROSS = GRAD == 2;
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[32];
    __shared__ double vsum[2][PR_T];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wr = warp & 3, wc = warp >> 2;
    const int64_t item = blockIdx.x;
    const int64_t pidx = item / p.ntiles;
    const int2 tt = p.tiles[item % p.ntiles];
    const int ta = tt.x, tb = tt.y;
    const int2 ij = p.pairs[pidx];
    const int i = ij.x, j = ij.y;
    const int A0 = ta * PR_T, B0 = tb * PR_T;
    const int nvir = p.nvir, naux = p.naux;
    const int64_t ldb = p.ldb;
    const int nvb = CROSS ? p.nvir2 : nvir;  // virtuals of the column side
    const int64_t ldb2 = CROSS ? p.ldb2 : ldb;
    const double* gAi = p.B + (int64_t)i * nvir + A0;
    const double* gAj = p.B + (int64_t)j * nvir + A0;
    const double* gBj = (CROSS ? p.B2 : p.B) + (int64_t)j * nvb + B0;
    const double* gBi = p.B + (int64_t)i * nvir + B0;
    const int nk = (naux + PR_BK - 1) / PR_BK;

    auto load = [&](int stage, int kt) {
        double* s = sm + stage * 4 * PR_BK * PR_LD;
#pragma unroll
        for (int e = 0; e < (PR_BK * PR_T) / 256; ++e) {
            const int idx = tid + 256 * e, r = idx >> 6, c = idx & 63;
            const int q = kt * PR_BK + r;
            const bool okA = q < naux && A0 + c < nvir;
            const bool okB = q < naux && B0 + c < nvb;
            const int64_t off = (int64_t)q * ldb + c;
            const int so = r * PR_LD + c;
            cp_async8(s + 0 * PR_BK * PR_LD + so, okA ? gAi + off : p.B, okA);
            cp_async8(s + 2 * PR_BK * PR_LD + so, okB ? gBj + (int64_t)q * ldb2 + c : p.B, okB);
            if (!CROSS) {
                cp_async8(s + 1 * PR_BK * PR_LD + so, okA ? gAj + off : p.B, okA);
                cp_async8(s + 3 * PR_BK * PR_LD + so, okB ? gBi + off : p.B, okB);
            }
        }
    };

    double X[2][4][2], Y[2][4][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) X[a][b][0] = X[a][b][1] = Y[a][b][0] = Y[a][b][1] = 0.0;

#pragma unroll
    for (int s = 0; s < PR_STAGES - 1; ++s) {
        if (s < nk) load(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<PR_STAGES - 2>();
        __syncthreads();
        const int pf = kt + PR_STAGES - 1;
        if (pf < nk) load(pf % PR_STAGES, pf);
        cp_async_commit();
        const double* s = sm + (kt % PR_STAGES) * 4 * PR_BK * PR_LD;
        const double* sAi = s;
        const double* sAj = s + PR_BK * PR_LD;
        const double* sBj = s + 2 * PR_BK * PR_LD;
        const double* sBi = s + 3 * PR_BK * PR_LD;
#pragma unroll
        for (int ks = 0; ks < PR_BK / 4; ++ks) {
            const int kr = (ks * 4 + t) * PR_LD;
            double ax[2], ay[2], bx[4], by[4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                ax[mt] = sAi[kr + wr * 16 + mt * 8 + g];
                ay[mt] = sAj[kr + wr * 16 + mt * 8 + g];
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                bx[nt] = sBj[kr + wc * 32 + nt * 8 + g];
                by[nt] = sBi[kr + wc * 32 + nt * 8 + g];
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) {
                    dmma_8x8x4(X[mt][nt], ax[mt], bx[nt]);
                    if (!CROSS) dmma_8x8x4(Y[mt][nt], ay[mt], by[nt]);
                }
        }
    }
    cp_async_wait<0>();

    const double eij = p.eo[i] + (CROSS ? p.eo2[j] : p.eo[j]);
    KSum os, ss, oc, oc2;
    double rowsum[2] = {0.0, 0.0};
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int a = A0 + wr * 16 + mt * 8 + g;
        const double ea = a < nvir ? p.ev[a] : 0.0;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int b = B0 + wc * 32 + nt * 8 + 2 * t + h;
                if (a < nvir && b < nvb) {
                    const double D = eij - ea - (CROSS ? p.ev2[b] : p.ev[b]);
                    const double x = X[mt][nt][h], y = Y[mt][nt][h];
                    double f = 1.0 / D;
                    if (CROSS) {
                        os.add(x * x * f);
                    } else if (GRAD) {
                        // pair (i, j): Tt_ij[a, b] into the rows of i; for i < j also
                        // pair (j, i): Tt_ji[a, b] = (2 G_ji - G_ij)[a, b] / D into the
                        // rows of j.  Both orderings put t Tt on the row virtual a.
                        const double tt = (2.0 * x - y) * f;
                        p.T[((int64_t)(i - p.i0) * nvir + a) * p.ldt + (int64_t)(j - p.j0) * nvir + b] = tt;
                        const double c = x * f * tt;
                        os.add(x * x * f);
                        ss.add(x * (x - y) * f);
                        oc.add(c);
                        rowsum[mt] += c;
                        if (i != j) {
                            const double t2 = (2.0 * y - x) * f;
                            p.T2[((int64_t)(j - p.j0) * nvir + a) * p.ldt2 + (int64_t)(i - p.i0) * nvir + b] = t2;
                            const double c2 = y * f * t2;
                            os.add(y * y * f);
                            ss.add(y * (y - x) * f);
                            oc2.add(c2);
                            rowsum[mt] += c2;
                        }
                    } else {
                        if (p.has_kappa) {
                            const double d1 = 1.0 - exp(p.kappa * D);
                            f *= d1 * d1;
                        }
                        os.add((x * x + y * y) * f);
                        ss.add((x - y) * (x - y) * f);
                    }
                }
            }
    }
    // energy mode visits tiles ta <= tb only: the summands are symmetric under
    // a <-> b (X_ba = Y_ab), so an off-diagonal tile counts twice
    const double w = GRAD ? 1.0 : (i == j ? 0.5 : 1.0) * (ta < tb ? 2.0 : 1.0);  // (CROSS: 1)
    const double vos = block_sum(os.value(), red);
    const double vss = block_sum(ss.value(), red);
    if (tid == 0) {
        p.part[item * 2 + 0] = w * vos;
        p.part[item * 2 + 1] = w * vss;
    }
    if (GRAD == 1) {
        const double voc = block_sum(oc.value(), red);
        const double voc2 = block_sum(oc2.value(), red);
        if (tid == 0) {
            p.occ_part[2 * item] = voc;
            p.occ_part[2 * item + 1] = voc2;
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            double r = rowsum[mt];
            r += __shfl_xor_sync(0xffffffffu, r, 1);
            r += __shfl_xor_sync(0xffffffffu, r, 2);
            if (t == 0) vsum[wc][wr * 16 + mt * 8 + g] = r;
        }
        __syncthreads();
        if (tid < PR_T) p.vir_part[item * PR_T + tid] = vsum[0][tid] + vsum[1][tid];
    }
}

// Fixed-order compensated sum of n (os, ss) partials -> out[0..1].
__global__ void __launch_bounds__(1024) reduce_pairs_kernel(const double* __restrict__ part,
                                                            int64_t n, double* out) {
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

// acc_occ[o] += sum of the t Tt partials of the ordering (o, *) of every item
// whose pair holds o (slot 0 when o is i, slot 1 when o is j != i), for o in
// I (blocks 0 .. ni-1) and J (the rest); fixed order.
__global__ void __launch_bounds__(256) reduce_occ_kernel(const double* __restrict__ occ_part,
                                                         const int2* __restrict__ pairs, int64_t npairs,
                                                         int ntile2, int i0, int ni, int j0,
                                                         double* acc_occ) {
    __shared__ double sh[256];
    const int o = (int)blockIdx.x < ni ? i0 + (int)blockIdx.x : j0 + ((int)blockIdx.x - ni);
    KSum a;
    const int64_t n = npairs * ntile2;
    for (int64_t k = threadIdx.x; k < n; k += 256) {
        const int2 pr = pairs[k / ntile2];
        if (pr.x == o) a.add(occ_part[2 * k]);
        else if (pr.y == o) a.add(occ_part[2 * k + 1]);
    }
    sh[threadIdx.x] = a.value();
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum x;
        for (int k = 0; k < 256; ++k) x.add(sh[k]);
        acc_occ[o] += x.value();
    }
}

__global__ void scale_copy_f64_kernel(const double* __restrict__ x, int64_t n, double s, double* __restrict__ y) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) y[k] = s * x[k];
}

// acc_vir[a] += 2 * sum over the chunk's items with a in their a-tile.
__global__ void __launch_bounds__(256) reduce_vir_kernel(const double* __restrict__ vir_part,
                                                         int64_t npairs, int ntile, int nvir,
                                                         double* acc_vir) {
    const int a = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (a >= nvir) return;
    const int ta = a / PR_T, ar = a % PR_T;
    const int64_t nterm = npairs * ntile;
    KSum s;
    for (int64_t k = lane; k < nterm; k += 32) {
        const int64_t pidx = k / ntile, tb = k % ntile;
        const int64_t item = (pidx * ntile + ta) * ntile + tb;
        s.add(vir_part[item * PR_T + ar]);
    }
    double v = warp_sum(s.value());
    if (lane == 0) acc_vir[a] += 2.0 * v;
}

static fc_status set_smem_once() {
    static std::atomic<uint64_t> done{0};
    uint64_t bit = 0;
    if (!attrs_needed(done, &bit)) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(pair_f64_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, PR_SMEM));
    FC_CUDA(cudaFuncSetAttribute(pair_f64_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, PR_SMEM));
    FC_CUDA(cudaFuncSetAttribute(pair_f64_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, PR_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    done.fetch_or(bit);
    return FC_OK;
}

fc_status rimp2_energy_f64(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                           fc_stats* stats) {
    FC_TRY(set_smem_once());
    const int64_t nocc = d.nocc, nvir = d.nvir;
    const int ntile = (int)((nvir + PR_T - 1) / PR_T);
    const int ntiles = ntile * (ntile + 1) / 2;  // tiles ta <= tb
    int64_t plo, phi;  // this shard's pairs (all of them unsharded)
    shard_pair_range(nocc, d.shard, d.nshards, &plo, &phi);
    const int64_t npairs = phi - plo;
    const int64_t items = npairs * ntiles;
    if (items > INT32_MAX) return fail(FC_ERR_LAYOUT, "RI-MP2: too many pair tiles for one launch");
    if (items == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        if (stats) stats->precision = FC_PREC_F64;
        return FC_OK;
    }

    void *vpairs, *vpart, *vout;
    FC_TRY(ws_get(WS_PAIRS, (npairs + ntiles) * sizeof(int2), &vpairs));
    FC_TRY(ws_get(WS_PART, items * 2 * sizeof(double), &vpart));
    FC_TRY(ws_get(WS_OUT, 64 * sizeof(double), &vout));
    std::vector<int2> hp;
    for (int64_t i = 0, k = 0; i < nocc; ++i)
        for (int64_t j = i; j < nocc; ++j, ++k)
            if (k >= plo && k < phi) hp.push_back(make_int2((int)i, (int)j));
    for (int ta = 0; ta < ntile; ++ta)
        for (int tb = ta; tb < ntile; ++tb) hp.push_back(make_int2(ta, tb));
    FC_CUDA(cudaMemcpyAsync(vpairs, hp.data(), hp.size() * sizeof(int2), cudaMemcpyHostToDevice, st));

    PairArgs a{};
    a.B = d.b_ov;
    a.ldb = nocc * nvir;
    a.naux = (int)d.naux;
    a.nvir = (int)nvir;
    a.eo = d.eps_occ;
    a.ev = d.eps_vir;
    a.pairs = (const int2*)vpairs;
    a.tiles = (const int2*)vpairs + npairs;
    a.ntiles = ntiles;
    a.has_kappa = d.has_kappa;
    a.kappa = d.kappa;
    a.part = (double*)vpart;

    Context& c = ctx();
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    pair_f64_kernel<0><<<(unsigned)items, 256, PR_SMEM, st>>>(a);
    FC_TRY(check_launch("pair_f64_kernel<energy>"));
    if (stats) FC_CUDA(cudaEventRecord(c.ev1, st));
    reduce_pairs_kernel<<<1, 1024, 0, st>>>((const double*)vpart, items, (double*)vout);
    FC_TRY(check_launch("reduce_pairs_kernel"));
    double h[2];
    FC_CUDA(cudaMemcpyAsync(h, vout, sizeof(h), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    *e_os = h[0];
    *e_ss = h[1];
    if (stats) {
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        stats->flops = 2.0 * (double)d.naux * (double)nvir * (double)nvir * (double)npairs;
        stats->precision = FC_PREC_F64;
        stats->launches += 2;
        stats->tile_m = PR_T;
        stats->tile_n = PR_T;
        stats->k_panel = 0;
        stats->d2h_bytes += sizeof(h);
        stats->h2d_bytes += hp.size() * sizeof(int2);
        stats->main_launches = 1;
        stats->main_ms = ms;
        stats->main_flops = stats->flops;
        stats->main_bytes = 8.0 * (double)d.naux * (double)(nocc * nvir);
    }
    return FC_OK;
}

fc_status rimp2_grad_f64(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                         double* gamma, double* de_docc, double* de_dvir, fc_stats* stats,
                         const GammaSink* sink, const DensOut* dens) {
    FC_TRY(set_smem_once());
    if (dens && d.nshards != 1) return fail(FC_ERR_INVALID, "RI-MP2 densities: no sharded form");
    const int64_t nocc = d.nocc, nvir = d.nvir, naux = d.naux, nov = nocc * nvir;
    const int ntile = (int)((nvir + PR_T - 1) / PR_T);
    const int ntile2 = ntile * ntile;  // every tile (ta, tb) of a pair, ta-major
    // Occupied chunks processed as chunk pairs (I, J), I <= J: each unordered
    // pair (i, j) is computed once and writes the amplitude rows of i (columns
    // of J) and of j (columns of I); both blocks (c nvir)^2 doubles fit the
    // chunk budget beside B and Gamma.
    // with densities the chunk is also bounded by the FP64 slabs (four chunk
    // budgets: the slabs are the densities' whole working set)
    const int64_t cc = dens ? dens_chunk_f64(nocc, nvir, grad_chunk_f64(nocc, nvir, d.chunk_bytes, 1),
                                             4 * d.chunk_bytes)
                            : grad_chunk_f64(nocc, nvir, d.chunk_bytes, d.nshards);
    const int64_t nch = (nocc + cc - 1) / cc;
    struct CP {
        int64_t i0, ni, j0, nj, p0, np;
    };
    std::vector<CP> cps;
    std::vector<int2> hp;
    std::vector<int64_t> cp_index((size_t)(nch * nch), -1);  // [I][J], I <= J
    for (int64_t I = 0; I < nch; ++I)
        for (int64_t J = I; J < nch; ++J) {
            cp_index[(size_t)(I * nch + J)] = (int64_t)cps.size();
            CP x;
            x.i0 = I * cc;
            x.ni = std::min(cc, nocc - x.i0);
            x.j0 = J * cc;
            x.nj = std::min(cc, nocc - x.j0);
            x.p0 = (int64_t)hp.size();
            for (int64_t i = x.i0; i < x.i0 + x.ni; ++i)
                for (int64_t j = (I == J ? i : x.j0); j < x.j0 + x.nj; ++j) hp.push_back(make_int2((int)i, (int)j));
            x.np = (int64_t)hp.size() - x.p0;
            cps.push_back(x);
        }
    const int64_t npairs_all = (int64_t)hp.size();
    for (int ta = 0; ta < ntile; ++ta)
        for (int tb = 0; tb < ntile; ++tb) hp.push_back(make_int2(ta, tb));
    const int64_t ncp = (int64_t)cps.size();
    const std::vector<int> owner = chunk_pair_owner(nocc, cc, d.nshards);
    int64_t max_items = 0;
    for (const auto& x : cps) max_items = std::max(max_items, x.np * ntile2);
    if (max_items > INT32_MAX) return fail(FC_ERR_LAYOUT, "RI-MP2 gradient: too many pair tiles per chunk pair");
    // The run order: each chunk pair once (gradient), or by column chunk K
    // with the block (I, K) of every I (densities; as in the mixed driver):
    // the pair kernel then writes that block straight into the slab.
    struct Step {
        int64_t x;
        int blk;    // 0: T, 1: T2, 2: both
        bool sums;  // take the chunk pair's energy and dE/deps terms
        bool last;  // last block of the column chunk
    };
    std::vector<Step> steps;
    if (!dens) {
        for (int64_t x = 0; x < ncp; ++x) steps.push_back({x, 2, true, false});
    } else {
        for (int64_t K = 0; K < nch; ++K)
            for (int64_t I = 0; I < nch; ++I)
                steps.push_back({cp_index[(size_t)(std::min(I, K) * nch + std::max(I, K))], I <= K ? 0 : 1, I <= K,
                                 I == nch - 1});
    }
    const int64_t nsteps = (int64_t)steps.size();
    DensF64 dx{};

    void *vpairs, *vpart, *vT, *vout;
    const size_t blk = (size_t)cc * nvir * cc * nvir;  // doubles of one amplitude block
    FC_TRY(ws_get(WS_PAIRS, hp.size() * sizeof(int2), &vpairs));
    FC_TRY(ws_get(WS_T, 2 * blk * sizeof(double), &vT));
    FC_TRY(ws_get(WS_PART, (size_t)max_items * (2 + 2 + PR_T) * sizeof(double), &vpart));
    FC_TRY(ws_get(WS_OUT, (size_t)(2 * ncp + nocc) * sizeof(double) + 64, &vout));
    double* part = (double*)vpart;
    double* occ = part + 2 * max_items;
    double* vir = occ + 2 * max_items;
    double* T1 = (double*)vT;
    double* T2 = T1 + blk;
    double* e_cp = (double*)vout;     // [ncp][2]
    double* acc_occ = e_cp + 2 * ncp;  // [nocc]
    FC_CUDA(cudaMemcpyAsync(vpairs, hp.data(), hp.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemsetAsync(de_dvir, 0, nvir * sizeof(double), st));
    FC_CUDA(cudaMemsetAsync(acc_occ, 0, nocc * sizeof(double), st));
    FC_CUDA(cudaMemsetAsync(e_cp, 0, 2 * ncp * sizeof(double), st));  // chunk pairs of other shards add nothing
    FC_CUDA(cudaMemsetAsync(gamma, 0, (size_t)naux * nov * sizeof(double), st));
    const int2* dpairs = (const int2*)vpairs;

    Context& c = ctx();
    cudaEvent_t* ev = nullptr;
    cudaEvent_t* ev2 = nullptr;
    int nadj = 0;
    double adj_flops = 0.0, adj_bytes = 0.0;
    if (stats) FC_TRY(timing_events((int)nsteps, &ev));
    if (stats) FC_TRY(timing_events2((int)(2 * nsteps), &ev2));
    if (stats) FC_CUDA(cudaEventRecord(c.ev0, st));
    if (dens) FC_TRY(dens_f64_alloc(nocc, nvir, cc, st, &dx));
    int64_t nl = 0, npair_launch = 0;
    // Gamma[:, rows of R] += 4 B_ov[:, columns of K] . T^T
    auto adjoint = [&](const double* T, int64_t r0, int64_t nr, int64_t k0, int64_t nk) -> fc_status {
        const int N = (int)(nr * nvir);
        dim3 grid((N + DG_BN - 1) / DG_BN, (unsigned)((naux + DG_BM - 1) / DG_BM), 1);
        EpiStore epi{gamma + r0 * nvir, nov, 4.0, 1};
        const int64_t K = nk * nvir;
        if (stats) FC_CUDA(cudaEventRecord(ev2[2 * nadj], st));
        dgemm_tn_kernel<EpiStore><<<grid, 256, DG_SMEM, st>>>(d.b_ov + k0 * nvir, nov, T, K, (int)naux, N, K, K, 0,
                                                               epi);
        if (stats) FC_CUDA(cudaEventRecord(ev2[2 * nadj + 1], st));
        ++nadj;
        adj_flops += 2.0 * (double)naux * (double)N * (double)K;
        adj_bytes += 8.0 * (double)naux * (double)K + 8.0 * (double)N * (double)K + 16.0 * (double)naux * (double)N;
        return check_launch("dgemm_tn_kernel<gamma>");
    };
    for (int64_t sx = 0; sx < nsteps; ++sx) {
        const Step& step = steps[(size_t)sx];
        const int64_t x = step.x;
        const CP& cp = cps[x];
        const bool same = cp.i0 == cp.j0;
        if (owner[x] != d.shard) {
            if (stats) {
                FC_CUDA(cudaEventRecord(ev[2 * sx], st));
                FC_CUDA(cudaEventRecord(ev[2 * sx + 1], st));
            }
            continue;
        }
        PairArgs a{};
        a.B = d.b_ov;
        a.ldb = nov;
        a.naux = (int)naux;
        a.nvir = (int)nvir;
        a.eo = d.eps_occ;
        a.ev = d.eps_vir;
        a.pairs = dpairs + cp.p0;
        a.tiles = dpairs + npairs_all;
        a.ntiles = ntile2;
        a.part = part;
        a.T = T1;
        a.ldt = cp.nj * nvir;
        a.T2 = same ? T1 : T2;
        a.ldt2 = same ? a.ldt : cp.ni * nvir;
        a.i0 = (int)cp.i0;
        a.j0 = (int)cp.j0;
        a.occ_part = occ;
        a.vir_part = vir;
        double* tb1 = T1;
        double* tb2 = same ? T1 : T2;
        if (dens) {  // the column chunk's block goes straight into the slab
            if (step.blk == 0) {
                tb1 = dx.ts + cp.i0 * nvir * a.ldt;
                if (same) tb2 = tb1;
            } else {
                tb2 = dx.ts + cp.j0 * nvir * a.ldt2;
            }
        }
        a.T = tb1;
        a.T2 = tb2;
        const int64_t nit = cp.np * ntile2;
        if (stats) FC_CUDA(cudaEventRecord(ev[2 * sx], st));
        pair_f64_kernel<1><<<(unsigned)nit, 256, PR_SMEM, st>>>(a);
        FC_TRY(check_launch("pair_f64_kernel<grad>"));
        if (stats) FC_CUDA(cudaEventRecord(ev[2 * sx + 1], st));
        ++npair_launch;
        if (step.sums) {
            reduce_pairs_kernel<<<1, 1024, 0, st>>>(part, nit, e_cp + 2 * x);
            reduce_occ_kernel<<<(unsigned)(same ? cp.ni : cp.ni + cp.nj), 256, 0, st>>>(
                occ, dpairs + cp.p0, cp.np, ntile2, (int)cp.i0, (int)cp.ni, (int)cp.j0, acc_occ);
            reduce_vir_kernel<<<(unsigned)((nvir + 7) / 8), 256, 0, st>>>(vir, cp.np, ntile, (int)nvir, de_dvir);
            FC_TRY(check_launch("rimp2 gradient reductions"));
            nl += 3;
        }
        ++nl;
        if (step.blk != 1) FC_TRY(adjoint(tb1, cp.i0, cp.ni, cp.j0, cp.nj));
        if (step.blk != 0 && !same) FC_TRY(adjoint(tb2, cp.j0, cp.nj, cp.i0, cp.ni));
        if (dens) {
            const bool t2 = step.blk == 1;
            const int64_t r0 = t2 ? cp.j0 : cp.i0, nr = t2 ? cp.nj : cp.ni, nk = t2 ? cp.ni : cp.nj;
            FC_TRY(dens_f64_block(dx, r0 * nvir, nr, nk, st, &nl));
            if (step.last) FC_TRY(dens_f64_slab(dx, nk, st, &nl));
        }
        // row I of the chunk pairs is done: Gamma's columns of chunk I are final
        if (!dens && sink && cp.j0 + cp.nj == nocc)
            FC_TRY(gamma_sink_block(sink, gamma, naux, nov, nvir, cp.i0, cp.ni, st));
    }
    if (dens) {
        FC_TRY(dens_f64_finish(dx, *dens, st, &nl));
        if (sink) FC_TRY(gamma_sink_block(sink, gamma, naux, nov, nvir, 0, nocc, st));
    }
    scale_copy_f64_kernel<<<(unsigned)((nocc + 255) / 256), 256, 0, st>>>(acc_occ, nocc, -2.0, de_docc);
    FC_TRY(check_launch("scale_copy_f64_kernel"));
    if (stats) FC_CUDA(cudaEventRecord(c.ev1, st));
    std::vector<double> h((size_t)(2 * ncp));
    FC_CUDA(cudaMemcpyAsync(h.data(), e_cp, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    double eo = 0.0, co = 0.0, es = 0.0, cs = 0.0;
    for (int64_t x = 0; x < ncp; ++x) {  // chunk-pair order, compensated
        double v = h[2 * x], tt = eo + v;
        co += (fabs(eo) >= fabs(v)) ? (eo - tt) + v : (v - tt) + eo;
        eo = tt;
        v = h[2 * x + 1];
        tt = es + v;
        cs += (fabs(es) >= fabs(v)) ? (es - tt) + v : (v - tt) + es;
        es = tt;
    }
    *e_os = eo + co;
    *e_ss = es + cs;
    if (stats) {
        float ms = 0.f;
        FC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        stats->kernel_ms = ms;
        const double P = (double)nocc * (nocc + 1) / 2.0;
        stats->flops = 2.0 * naux * (double)nvir * nvir * P + 2.0 * naux * (double)nov * nov;
        stats->precision = FC_PREC_F64;
        stats->launches += (int)(nl + nadj + 1);
        stats->tile_m = PR_T;
        stats->tile_n = PR_T;
        stats->k_panel = 0;
        stats->d2h_bytes += h.size() * sizeof(double);
        stats->h2d_bytes += hp.size() * sizeof(int2);
        // dominant kernel: the fused pair kernel, one launch per chunk pair,
        // forming G_ij and G_ji of every unordered pair
        stats->main_launches = (int)npair_launch;
        FC_TRY(timing_sum((int)nsteps, &stats->main_ms));
        const double rep = dens ? (double)nsteps / ncp : 1.0;  // densities: chunk pairs run per column
        stats->main_flops = 4.0 * naux * (double)nvir * nvir * P * rep;
        stats->main_bytes = (8.0 * naux * (double)nov * (double)nch + 8.0 * (double)nov * nov) * rep;
        stats->aux_launches = nadj;
        FC_TRY(timing_sum2(nadj, &stats->aux_ms));
        stats->aux_flops = adj_flops;
        stats->aux_bytes = adj_bytes;
    }
    return FC_OK;
}

// Opposite-spin (alpha-beta) energy of unrestricted RI-MP2 in FP64: every
// (i alpha, J beta) pair, every (a-tile, b-tile), X = G_iJ only
// (opposite_spin_block_energy, ferric-mp2/src/u_rimp2.rs:731-753).
fc_status ump2_cross_f64(const UmpSpin& A, const UmpSpin& Bs, int64_t naux, cudaStream_t st, double* e_ab,
                         fc_stats* stats) {
    FC_TRY(set_smem_once());
    const int nta = (int)((A.nvir + PR_T - 1) / PR_T), ntb = (int)((Bs.nvir + PR_T - 1) / PR_T);
    const int64_t npairs = A.nocc * Bs.nocc;
    const int ntiles = nta * ntb;
    const int64_t items = npairs * ntiles;
    if (items > INT32_MAX) return fail(FC_ERR_LAYOUT, "U-RI-MP2: too many pair tiles for one launch");
    void *vpairs, *vpart, *vout;
    FC_TRY(ws_get(WS_PAIRS, (npairs + ntiles) * sizeof(int2), &vpairs));
    FC_TRY(ws_get(WS_PART, items * 2 * sizeof(double), &vpart));
    FC_TRY(ws_get(WS_OUT, 64 * sizeof(double), &vout));
    std::vector<int2> hp;
    for (int i = 0; i < A.nocc; ++i)
        for (int j = 0; j < Bs.nocc; ++j) hp.push_back(make_int2(i, j));
    for (int ta = 0; ta < nta; ++ta)
        for (int tb = 0; tb < ntb; ++tb) hp.push_back(make_int2(ta, tb));
    FC_CUDA(cudaMemcpyAsync(vpairs, hp.data(), hp.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    PairArgs a{};
    a.B = A.b_ov;
    a.ldb = A.nocc * A.nvir;
    a.naux = (int)naux;
    a.nvir = (int)A.nvir;
    a.eo = A.eps_occ;
    a.ev = A.eps_vir;
    a.pairs = (const int2*)vpairs;
    a.tiles = (const int2*)vpairs + npairs;
    a.ntiles = ntiles;
    a.part = (double*)vpart;
    a.B2 = Bs.b_ov;
    a.ldb2 = Bs.nocc * Bs.nvir;
    a.nvir2 = (int)Bs.nvir;
    a.eo2 = Bs.eps_occ;
    a.ev2 = Bs.eps_vir;
    Context& c = ctx();
    cudaEvent_t* ev = nullptr;
    if (stats) {
        FC_TRY(timing_events(1, &ev));
        FC_CUDA(cudaEventRecord(ev[0], st));
    }
    pair_f64_kernel<2><<<(unsigned)items, 256, PR_SMEM, st>>>(a);
    FC_TRY(check_launch("pair_f64_kernel<cross>"));
    if (stats) FC_CUDA(cudaEventRecord(ev[1], st));
    reduce_pairs_kernel<<<1, 1024, 0, st>>>((const double*)vpart, items, (double*)vout);
    FC_TRY(check_launch("reduce_pairs_kernel"));
    double h[2];
    FC_CUDA(cudaMemcpyAsync(h, vout, sizeof(h), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    *e_ab = h[0];
    if (stats) {
        double ms = 0.0;
        FC_TRY(timing_sum(1, &ms));
        stats->main_ms += ms;
        stats->main_launches += 1;
        stats->main_flops += 2.0 * (double)naux * (double)(A.nocc * A.nvir) * (double)(Bs.nocc * Bs.nvir);
        stats->launches += 2;
        (void)c;
    }
    return FC_OK;
}

// ------------------------------------------------ allocation-free energy --
//
// fc_rimp2_energy_noalloc: the FP64 RI-MP2 energy with all of its scratch
// (pair table, per-tile partials, the two reduced sums) in one fixed
// device array that lives in this library's module, so the call allocates
// no device memory.  It exists for callers that cannot call cudaMalloc: code
// whose device memory is owned by another allocator (ferric's device-pool
// ledger charges every byte to a reservation and refuses beyond it; a
// framework's caching allocator may hold nearly all of the device), and
// inner-loop code that must not pay cudaMalloc/cudaFree's implicit device
// synchronisation.  Limits and sharing rules are in include/ferric_cuda.h.

namespace {

constexpr size_t kNoallocScratchBytes = size_t(4) << 20;  // 4 MiB, held by every device that loads the library
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kNoallocMaxDevices = 64;
void* g_noalloc_ptr[kNoallocMaxDevices] = {};  // device address of g_noalloc_scratch, per ordinal
std::mutex g_noalloc_mu;

// Unordered pairs (i <= j) in row-major order, one thread per i; then the
// tiles (ta <= tb) of a pair.
__global__ void noalloc_pairs_kernel(int nocc, int ntile, int2* pairs, int2* tiles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nocc) {
        const int64_t off = (int64_t)i * nocc - (int64_t)i * (i - 1) / 2;
        for (int j = i; j < nocc; ++j) pairs[off + (j - i)] = make_int2(i, j);
    }
    if (i < ntile) {
        const int off = i * ntile - i * (i - 1) / 2;
        for (int tb = i; tb < ntile; ++tb) tiles[off + (tb - i)] = make_int2(i, tb);
    }
}

}  // namespace

}  // namespace fc

extern "C" fc_status fc_rimp2_energy_noalloc(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                             const double* eps_occ, const double* eps_vir, int32_t has_kappa,
                                             double kappa, double* e_os, double* e_ss, void* stream) {
    using namespace fc;
    if (!e_os || !e_ss) return fail(FC_ERR_INVALID, "fc_rimp2_energy_noalloc: null output pointer");
    if (naux < 0 || nocc < 0 || nvir < 0) return fail(FC_ERR_LAYOUT, "fc_rimp2_energy_noalloc: negative dimension");
    if (has_kappa && !(kappa > 0.0 && kappa < 1e300))
        return fail(FC_ERR_INVALID, "fc_rimp2_energy_noalloc: kappa must be finite and > 0");
    if (naux == 0 || nocc == 0 || nvir == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        return FC_OK;
    }
    if (!b_ov || !eps_occ || !eps_vir) return fail(FC_ERR_INVALID, "fc_rimp2_energy_noalloc: null input pointer");
    if (nocc > (1 << 20) || nvir > (1 << 24) || naux > INT32_MAX)
        return fail(FC_ERR_LAYOUT, "fc_rimp2_energy_noalloc: dimension out of range");
    const int64_t npairs = nocc * (nocc + 1) / 2;
    const int64_t ntile = (nvir + PR_T - 1) / PR_T;
    const int64_t ntiles = ntile * (ntile + 1) / 2;
    // the pair and tile tables alone must fit before their product is formed
    // (npairs * ntiles can exceed int64 at the accepted dimension bounds)
    if ((size_t)(npairs + ntiles) * sizeof(int2) > kNoallocScratchBytes)
        return fail(FC_ERR_LAYOUT, "fc_rimp2_energy_noalloc: the pair and tile tables alone exceed the fixed scratch of " +
                                       std::to_string(kNoallocScratchBytes) + " B; use fc_rimp2_energy_dev");
    const int64_t items = npairs * ntiles;
    const size_t pair_bytes = ((size_t)(npairs + ntiles) * sizeof(int2) + 255) / 256 * 256;
    const size_t part_bytes = ((size_t)items * 2 * sizeof(double) + 255) / 256 * 256;
    const size_t need = pair_bytes + part_bytes + 256;
    if (items > INT32_MAX || need > kNoallocScratchBytes)
        return fail(FC_ERR_LAYOUT,
                    "fc_rimp2_energy_noalloc: needs " + std::to_string(need) + " B of scratch for " +
                        std::to_string(items) + " pair tiles; the fixed scratch holds " +
                        std::to_string(kNoallocScratchBytes) + " B (about " +
                        std::to_string((kNoallocScratchBytes - 512) / 16) +
                        " tiles of 64 x 64 virtuals); use fc_rimp2_energy_dev");

    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    int dev = -1;
    FC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoallocMaxDevices) return fail(FC_ERR_DEVICE, "fc_rimp2_energy_noalloc: device ordinal out of range");
    if (!g_noalloc_ptr[dev]) {
        // once per device, with that device current
        void* p = nullptr;
        FC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        FC_CUDA(cudaFuncSetAttribute(pair_f64_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, PR_SMEM));
        g_noalloc_ptr[dev] = p;
    }
    char* base = static_cast<char*>(g_noalloc_ptr[dev]);
    int2* pairs = reinterpret_cast<int2*>(base);
    double* part = reinterpret_cast<double*>(base + pair_bytes);
    double* out = reinterpret_cast<double*>(base + pair_bytes + part_bytes);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Every byte read below is written earlier in this call (pairs, then all
    // partials, then the sums), so contents left by a previous call are never read.
    const int64_t nthr = nocc > ntile ? nocc : ntile;
    noalloc_pairs_kernel<<<(unsigned)((nthr + 127) / 128), 128, 0, st>>>((int)nocc, (int)ntile, pairs,
                                                                         pairs + npairs);
    PairArgs a{};
    a.B = b_ov;
    a.ldb = nocc * nvir;
    a.naux = (int)naux;
    a.nvir = (int)nvir;
    a.eo = eps_occ;
    a.ev = eps_vir;
    a.pairs = pairs;
    a.tiles = pairs + npairs;
    a.ntiles = (int)ntiles;
    a.has_kappa = has_kappa;
    a.kappa = kappa;
    a.part = part;
    pair_f64_kernel<0><<<(unsigned)items, 256, PR_SMEM, st>>>(a);
    reduce_pairs_kernel<<<1, 1024, 0, st>>>(part, items, out);
    FC_TRY(check_launch("fc_rimp2_energy_noalloc kernels"));
    double h[2];
    FC_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaStreamSynchronize(st));
    *e_os = h[0];
    *e_ss = h[1];
    return FC_OK;
}
