// Unrelaxed MP2 densities on the device (build_mp2_density,
// ferric-mp2/src/oo_rimp2.rs:1170-1300):
//     P_ij = - sum_kab t_ik^ab Tt_jk^ab,      P_ab = sum_ijc t_ij^ac Tt_ij^bc,
// t_ij^ab = (ia|jb) / D_ij^ab and Tt = 2 t - t^T per (i, j) block (the
// weighted amplitudes the gradient forms anyway), so t = (2 Tt + Tt^T) / 3
// within each block.
//
// The gradient drivers run their chunk pairs column by column when the
// densities are wanted: the slab of column chunk K holds the amplitude blocks
// (I, K) of every occupied chunk I -- rows (i, a) of all i, columns (k, b) of
// k in K.  A chunk pair (I, K), I != K, is computed for both of its columns
// (its energy and dE/deps terms are taken once).  With a slab complete:
//     P_vv += sum_i  t[(i, .), slab] Tt[(i, .), slab]^T     (per i: nvir x nvir)
//     P_oo -= sum_a  t[(., a), slab] Tt[(., a), slab]^T     (per a: nocc x nocc)
// For fixed a, P_oo's operand rows (i, a) are tp rows apart: one row per
// plane of a 3-D tensor map.  Both totals are symmetric (the reference's
// sums over all (i, j), resp. all k, are), so tile pairs t1 <= t2 are
// computed and mirrored.
//
// FC_PREC_MIXED: each slab holds three int8 slices of Tt (the adjoint
// contraction's own operand) and of t, one scale per row (i, a).  An item is
// (i, tile pair) for P_vv and (a, tile pair) for P_oo over all of the slab's
// K = |K| tp columns: the int32 level sums are exact (K <= 32768 per drain),
// and the FP64 values scale by s_row s_col and add into a partial tile owned
// by the CTA (a CTA always gets the same tile pair and its items in a fixed
// order, so the result does not depend on timing).  The partials fold in
// group order at the end.
//
// FC_PREC_F64: FP64 slabs; P_vv one DMMA tile GEMM per i (upper tiles,
// accumulated in launch order), P_oo one split-K GEMM per slab with K =
// nvir |K| nvir (the rows of i are contiguous in the slab), splits folded in
// order.
#include <algorithm>

#include "dgemm_tn.cuh"
#include "fc_internal.cuh"
#include "fx_split.cuh"
#include "rimp2.cuh"
#include "tc.cuh"
#include "tmap.cuh"
#include "xgemm.cuh"

namespace fc {

namespace {

constexpr int DT = 128;            // density tile (rows and columns)
constexpr int DT2 = DT * DT;

// Tile pair x of n tiles per side (t1 <= t2, t1-major).
__host__ __device__ inline void tile_pair(int x, int n, int* t1, int* t2) {
    int a = 0;
    while (x >= n - a) {
        x -= n - a;
        ++a;
    }
    *t1 = a;
    *t2 = a + x;
}

// t from Tt within every tp x tp sub-block (i, k) of an amplitude block of
// nk sub-blocks per row of sub-blocks (pitch ld):
//     dst[a, b] = (2 src[a, b] + src[b, a]) / 3.
// One CTA per AT x AT tile pair (ta <= tb) of a sub-block (blockIdx.y); both
// tiles are read before either is written, so dst may be src.  A warp reads
// 64 consecutive elements of a row: the row pitch is the whole block's, so
// shorter runs cost DRAM row switches (32 x 32 FP32 tiles ran at 2.2 TB/s);
// FP64 tiles are 32 wide (two of 64 x 64 would pass the static shared limit).
template <typename T>
constexpr int amp_tile() { return sizeof(T) == 4 ? 64 : 32; }
template <typename T>
__global__ void __launch_bounds__(256) amp_from_tt_kernel(const T* src, T* dst, int64_t ld, int64_t tp, int nk,
                                                          int ntt) {
    constexpr int AT = amp_tile<T>(), RY = 256 / AT;  // tile side, rows per pass
    __shared__ T s1[AT][AT + 1], s2[AT][AT + 1];
    int ta, tb;
    tile_pair((int)blockIdx.x, ntt, &ta, &tb);
    const int64_t sb = blockIdx.y;
    const int64_t r0 = (sb / nk) * tp, c0 = (sb % nk) * tp;
    const int tx = threadIdx.x % AT, ty = threadIdx.x / AT;
    const int64_t a0 = (int64_t)ta * AT, b0 = (int64_t)tb * AT;
    for (int r = ty; r < AT; r += RY) {
        const int64_t a = a0 + r, b = b0 + tx;  // s1[r][tx] = src[a, b]
        s1[r][tx] = (a < tp && b < tp) ? src[(r0 + a) * ld + c0 + b] : (T)0;
        const int64_t a2 = b0 + r, b2 = a0 + tx;  // s2[r][tx] = src[a2, b2]
        s2[r][tx] = (a2 < tp && b2 < tp) ? src[(r0 + a2) * ld + c0 + b2] : (T)0;
    }
    __syncthreads();
    for (int r = ty; r < AT; r += RY) {
        const int64_t a = a0 + r, b = b0 + tx;  // src[b, a] = s2[tx][r]
        if (a < tp && b < tp)
            dst[(r0 + a) * ld + c0 + b] = (T)((2.0 * (double)s1[r][tx] + (double)s2[tx][r]) / 3.0);
        if (ta != tb) {
            const int64_t a2 = b0 + r, b2 = a0 + tx;  // src[b2, a2] = s1[tx][r]
            if (a2 < tp && b2 < tp)
                dst[(r0 + a2) * ld + c0 + b2] = (T)((2.0 * (double)s2[r][tx] + (double)s1[tx][r]) / 3.0);
        }
    }
}

// Three int8 slices of FP32 rows (pitch K) into a slab (slices slice_rows
// rows apart), one scale per row.
__global__ void __launch_bounds__(256) dens_split_rows_kernel(const float* __restrict__ T, int64_t K,
                                                              int64_t slice_rows, double* __restrict__ sc,
                                                              int8_t* __restrict__ out) {
    split_fx_rows_f32_body<SliceI8>(T, K, K, slice_rows, sc, out, blockIdx.x);
}

template <typename T>
fc_status amp_from_tt(const T* src, T* dst, int64_t ld, int64_t tp, int64_t nr, int64_t nk, cudaStream_t st) {
    const int ntt = (int)((tp + amp_tile<T>() - 1) / amp_tile<T>());
    const int64_t nsub = nr * nk;
    if (nsub > 65535) return fail(FC_ERR_LAYOUT, "MP2 densities: too many amplitude sub-blocks in one block");
    amp_from_tt_kernel<T><<<dim3((unsigned)(ntt * (ntt + 1) / 2), (unsigned)nsub), 256, 0, st>>>(src, dst, ld, tp,
                                                                                                 (int)nk, ntt);
    return check_launch("amp_from_tt_kernel");
}

// P_vv item (LdRows): A row it.x = i tp + t1 128 of the t slab, B row it.y =
// i tp + t2 128 of the Tt slab, it.w k-steps (0: a padding item).  Partial
// tiles are column-major (a warp's rows are consecutive).
struct EpiDensVV {
    const double* sa;
    const double* st;
    double* part;
    int64_t tp;
    int nvir;
    __device__ __forceinline__ void operator()(int64_t, int4 it, int row, int col0, const double (&acc)[32]) const {
        if (it.w == 0) return;
        const int64_t i = it.x / tp;
        const int a = (int)(it.x - i * tp) + row;
        if (a >= nvir) return;
        const int b0 = (int)(it.y - i * tp) + col0;
        const double s = sa[it.x + row];
        double* pc = part + (int64_t)blockIdx.x * DT2 + (int64_t)col0 * DT + row;
        // eight partials and scales loaded together, then updated (one chain
        // of eight loads in flight instead of 32 dependent read-modify-writes)
#pragma unroll
        for (int c0 = 0; c0 < 32; c0 += 8) {
            double sv[8], pv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const bool ok = b0 + c0 + u < nvir;
                sv[u] = ok ? __ldg(st + it.y + col0 + c0 + u) : 0.0;
                pv[u] = ok ? pc[(c0 + u) * DT] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (b0 + c0 + u < nvir) pc[(c0 + u) * DT] = pv[u] + s * sv[u] * acc[c0 + u];
        }
    }
};

// P_oo item (LdPlanes): planes (occupied i) it.x 128 .. of the t slab and
// it.y 128 .. of the Tt slab, row a = it.z of each plane.  The row scales
// come transposed (saT[a nocc + i], stT[a nocc + j]): a thread's 32
// columns are then 32 consecutive scales.
struct EpiDensOO {
    const double* saT;
    const double* stT;
    double* part;
    int nocc;
    __device__ __forceinline__ void operator()(int64_t, int4 it, int row, int col0, const double (&acc)[32]) const {
        if (it.w == 0) return;
        const int i = it.x * DT + row;
        if (i >= nocc) return;
        const int64_t a = it.z;
        const double s = -saT[a * nocc + i];
        const int j0 = it.y * DT + col0;
        const double* sj = stT + a * nocc + j0;
        double* pc = part + (int64_t)blockIdx.x * DT2 + (int64_t)col0 * DT + row;
#pragma unroll
        for (int c0 = 0; c0 < 32; c0 += 8) {
            double sv[8], pv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const bool ok = j0 + c0 + u < nocc;
                sv[u] = ok ? __ldg(sj + c0 + u) : 0.0;
                pv[u] = ok ? pc[(c0 + u) * DT] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (j0 + c0 + u < nocc) pc[(c0 + u) * DT] = pv[u] + s * sv[u] * acc[c0 + u];
        }
    }
};

// sT[a nocc + i] = s[i tp + a] for a < nvir, i < nocc (the P_oo scales)
__global__ void __launch_bounds__(256) scale_t_kernel(const double* __restrict__ s, int64_t nocc, int64_t nvir,
                                                      int64_t tp, double* __restrict__ sT) {
    const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (e >= nocc * nvir) return;
    const int64_t a = e / nocc, i = e % nocc;
    sT[e] = s[i * tp + a];
}

// out (n x n, row-major) from the partial tiles: slot g ntp + x holds tile
// pair x of group g; summed over g in order; pairs t1 < t2 mirrored, tiles
// on the diagonal made symmetric as (v + v^T) / 2.
__global__ void __launch_bounds__(256) dens_fold_kernel(const double* __restrict__ part, int ntp, int g, int ntile,
                                                        int n, double* __restrict__ out) {
    int t1, t2;
    tile_pair((int)blockIdx.y, ntile, &t1, &t2);
    const int e = blockIdx.x * 256 + threadIdx.x;  // column-major element of the tile
    if (e >= DT2) return;
    const int col = e / DT, row = e % DT;
    const int r = t1 * DT + row, c = t2 * DT + col;
    if (r >= n || c >= n) return;
    const double* p0 = part + (int64_t)blockIdx.y * DT2;
    double v = 0.0;
    for (int k = 0; k < g; ++k) v += p0[(int64_t)k * ntp * DT2 + e];
    if (t1 == t2) {
        double w = 0.0;
        const int et = row * DT + col;  // the transposed element
        for (int k = 0; k < g; ++k) w += p0[(int64_t)k * ntp * DT2 + et];
        v = 0.5 * (v + w);
    }
    out[(int64_t)r * n + c] = v;
    if (t1 != t2) out[(int64_t)c * n + r] = v;
}

// acc (n x n): entries below the diagonal from those above.
__global__ void mirror_upper_kernel(double* __restrict__ a, int64_t n) {
    const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (e >= n * n) return;
    const int64_t r = e / n, c = e % n;
    if (r > c) a[e] = a[c * n + r];
}

// a <- (a + a^T) / 2 (n x n), into b.
__global__ void sym_kernel(const double* __restrict__ a, int64_t n, double* __restrict__ b) {
    const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (e >= n * n) return;
    const int64_t r = e / n, c = e % n;
    b[e] = 0.5 * (a[e] + a[c * n + r]);
}

// p[e] = acc[e] - sum_s part[s][e] (split order)
__global__ void oo_fold_f64_kernel(const double* __restrict__ part, int splits, int64_t nn, double* __restrict__ acc) {
    const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (e >= nn) return;
    double v = 0.0;
    for (int s = 0; s < splits; ++s) v += part[(int64_t)s * nn + e];
    acc[e] -= v;
}

bool g_dens_attr = false;

fc_status dens_attrs() {
    if (g_dens_attr) return FC_OK;
    FC_CUDA(cudaFuncSetAttribute(xgemm_kernel<128, EpiDensVV, true, LdRows>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, xg::Cfg<128, true>::SMEM));
    FC_CUDA(cudaFuncSetAttribute(xgemm_kernel<128, EpiDensOO, true, LdPlanes>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, xg::Cfg<128, true>::SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    FC_CUDA(cudaFuncSetAttribute(dgemm_tn_kernel<EpiSplit>, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_SMEM));
    g_dens_attr = true;
    return FC_OK;
}

int64_t items_per_slab(const DensFx& o) {
    const int64_t lv = (o.nocc + o.g_vv - 1) / o.g_vv, lo = (o.nvir + o.g_oo - 1) / o.g_oo;
    return lv * o.ntp_vv * o.g_vv + lo * o.ntp_oo * o.g_oo;
}

}  // namespace

// ------------------------------------------------------------------ mixed --

int64_t dens_chunk_fx(int64_t nocc, int64_t nvir, int64_t cc, int64_t budget) {
    const int64_t tp = (nvir + 15) / 16 * 16;
    const int64_t per = 6 * nocc * tp * tp;  // slab bytes per occupied orbital of the column chunk
    int64_t c = std::max<int64_t>(1, budget / std::max<int64_t>(per, 1));
    return std::min(c, cc);
}

fc_status dens_fx_alloc(int64_t nocc, int64_t nvir, int64_t tp, int64_t cc, cudaStream_t st, DensFx* o) {
    FC_TRY(dens_attrs());
    const Context& c = ctx();
    o->nocc = nocc;
    o->nvir = nvir;
    o->tp = tp;
    o->rows = nocc * tp;
    if (3 * o->rows > INT32_MAX || cc * tp > INT32_MAX / 2)
        return fail(FC_ERR_LAYOUT, "MP2 densities: amplitude slab beyond the int8 kernels' range");
    const int64_t ld = cc * tp;
    const int nv = (int)((nvir + DT - 1) / DT), no = (int)((nocc + DT - 1) / DT);
    o->ntp_vv = nv * (nv + 1) / 2;
    o->ntp_oo = no * (no + 1) / 2;
    o->g_vv = (int)std::max<int64_t>(1, std::min<int64_t>(nocc, c.sm_count / o->ntp_vv));
    o->g_oo = (int)std::max<int64_t>(1, std::min<int64_t>(nvir, c.sm_count / o->ntp_oo));
    void *vs, *vp;
    const size_t slab = (size_t)3 * o->rows * ld;
    FC_TRY(ws_get(WS_DSLAB, 2 * slab, &vs));
    o->ts = (int8_t*)vs;
    o->as = o->ts + slab;
    const size_t nvv = (size_t)o->ntp_vv * o->g_vv * DT2, noo = (size_t)o->ntp_oo * o->g_oo * DT2;
    const size_t nitems = (size_t)items_per_slab(*o);
    const size_t nt = (size_t)nocc * nvir;
    FC_TRY(ws_get(WS_DPART, (2 * o->rows + 2 * nt + nvv + noo) * 8 + nitems * sizeof(int4), &vp));
    o->tsc = (double*)vp;
    o->asc = o->tsc + o->rows;
    o->tscT = o->asc + o->rows;
    o->ascT = o->tscT + nt;
    o->part_vv = o->ascT + nt;
    o->part_oo = o->part_vv + nvv;
    o->items = (int4*)(o->part_oo + noo);
    FC_CUDA(cudaMemsetAsync(o->part_vv, 0, (nvv + noo) * 8, st));
    return FC_OK;
}

fc_status dens_fx_block(const DensFx& o, float* blk, int64_t r0, int64_t nr, int64_t nk, cudaStream_t st,
                        int64_t* nl) {
    const int64_t ld = nk * o.tp, rows = nr * o.tp;
    FC_TRY(amp_from_tt<float>(blk, blk, ld, o.tp, nr, nk, st));
    dens_split_rows_kernel<<<(unsigned)rows, 256, 0, st>>>(blk, ld, o.rows, o.asc + r0, o.as + r0 * ld);
    *nl += 2;
    return check_launch("dens_split_rows_kernel");
}

fc_status dens_fx_slab(const DensFx& o, int64_t nk, cudaStream_t st, int* err, int64_t* nl) {
    const int64_t ld = nk * o.tp;
    const int nks = (int)((ld + 127) / 128);
    const int nv = (int)((o.nvir + DT - 1) / DT), no = (int)((o.nocc + DT - 1) / DT);
    // items: CTA s of grid g ntp + x (group g, tile pair x) takes item s + grid l,
    // l = 0 .. L-1, for i = g L + l (P_vv) or a = g L + l (P_oo)
    std::vector<int4> it;
    const int gvv = o.ntp_vv * o.g_vv, goo = o.ntp_oo * o.g_oo;
    const int64_t lv = (o.nocc + o.g_vv - 1) / o.g_vv, lo = (o.nvir + o.g_oo - 1) / o.g_oo;
    it.reserve((size_t)items_per_slab(o));
    for (int64_t l = 0; l < lv; ++l)
        for (int s = 0; s < gvv; ++s) {
            const int g = s / o.ntp_vv;
            int t1, t2;
            tile_pair(s % o.ntp_vv, nv, &t1, &t2);
            const int64_t i = g * lv + l;
            const int64_t r = std::min(i, o.nocc - 1) * o.tp;
            it.push_back(make_int4((int)(r + t1 * DT), (int)(r + t2 * DT), 0, i < o.nocc ? nks : 0));
        }
    const size_t nvv_items = it.size();
    for (int64_t l = 0; l < lo; ++l)
        for (int s = 0; s < goo; ++s) {
            const int g = s / o.ntp_oo;
            int t1, t2;
            tile_pair(s % o.ntp_oo, no, &t1, &t2);
            const int64_t a = g * lo + l;
            it.push_back(make_int4(t1, t2, (int)std::min(a, o.nvir - 1), a < o.nvir ? nks : 0));
        }
    FC_CUDA(cudaMemcpyAsync(o.items, it.data(), it.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    CUtensorMap ta, tt, pa, pt;
    FC_TRY(make_tmap_i8_2d(&ta, o.as, ld, 3 * o.rows, ld, 128, 128));
    FC_TRY(make_tmap_i8_2d(&tt, o.ts, ld, 3 * o.rows, ld, 128, 128));
    FC_TRY(make_tmap_i8_3d(&pa, o.as, ld, o.tp, 3 * o.nocc, ld, o.tp * ld, 128, 128));
    FC_TRY(make_tmap_i8_3d(&pt, o.ts, ld, o.tp, 3 * o.nocc, ld, o.tp * ld, 128, 128));
    {
        XArgs a{o.items, (int64_t)nvv_items, (int)o.rows, (int)o.rows, err};
        EpiDensVV epi{o.asc, o.tsc, o.part_vv, o.tp, (int)o.nvir};
        xgemm_kernel<128, EpiDensVV, true, LdRows>
            <<<gvv, xg::Cfg<128, true>::THREADS, xg::Cfg<128, true>::SMEM, st>>>(ta, tt, a, epi);
        FC_TRY(check_launch("xgemm_kernel<P_vv>"));
    }
    {
        const int64_t nt = o.nocc * o.nvir;
        scale_t_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(o.asc, o.nocc, o.nvir, o.tp, o.ascT);
        scale_t_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(o.tsc, o.nocc, o.nvir, o.tp, o.tscT);
        *nl += 2;
        XArgs a{o.items + nvv_items, (int64_t)(it.size() - nvv_items), (int)o.nocc, (int)o.nocc, err};
        EpiDensOO epi{o.ascT, o.tscT, o.part_oo, (int)o.nocc};
        xgemm_kernel<128, EpiDensOO, true, LdPlanes>
            <<<goo, xg::Cfg<128, true>::THREADS, xg::Cfg<128, true>::SMEM, st>>>(pa, pt, a, epi);
        FC_TRY(check_launch("xgemm_kernel<P_oo>"));
    }
    *nl += 2;
    return FC_OK;
}

fc_status dens_fx_finish(const DensFx& o, const DensOut& out, cudaStream_t st, int64_t* nl) {
    const int nv = (int)((o.nvir + DT - 1) / DT), no = (int)((o.nocc + DT - 1) / DT);
    dens_fold_kernel<<<dim3(DT2 / 256, (unsigned)o.ntp_vv), 256, 0, st>>>(o.part_vv, o.ntp_vv, o.g_vv, nv,
                                                                         (int)o.nvir, out.p_vv);
    dens_fold_kernel<<<dim3(DT2 / 256, (unsigned)o.ntp_oo), 256, 0, st>>>(o.part_oo, o.ntp_oo, o.g_oo, no,
                                                                         (int)o.nocc, out.p_oo);
    *nl += 2;
    return check_launch("dens_fold_kernel");
}

// ------------------------------------------------------------------- FP64 --

int64_t dens_chunk_f64(int64_t nocc, int64_t nvir, int64_t cc, int64_t budget) {
    const int64_t per = 16 * nocc * nvir * nvir;  // t and Tt slab bytes per occupied orbital of the column
    int64_t c = std::max<int64_t>(1, budget / std::max<int64_t>(per, 1));
    return std::min(c, cc);
}

fc_status dens_f64_alloc(int64_t nocc, int64_t nvir, int64_t cc, cudaStream_t st, DensF64* o) {
    FC_TRY(dens_attrs());
    o->nocc = nocc;
    o->nvir = nvir;
    o->splits = std::max(1, ctx().sm_count);
    const size_t slab = (size_t)nocc * nvir * cc * nvir;
    void *vs, *vp;
    FC_TRY(ws_get(WS_DSLAB, 2 * slab * 8, &vs));
    o->ts = (double*)vs;
    o->as = o->ts + slab;
    const size_t nn = (size_t)nocc * nocc;
    FC_TRY(ws_get(WS_DPART, ((size_t)o->splits * nn + nn + (size_t)nvir * nvir) * 8, &vp));
    o->part_oo = (double*)vp;
    o->acc_oo = o->part_oo + (size_t)o->splits * nn;
    o->acc_vv = o->acc_oo + nn;
    FC_CUDA(cudaMemsetAsync(o->acc_oo, 0, (nn + (size_t)nvir * nvir) * 8, st));
    return FC_OK;
}

fc_status dens_f64_block(const DensF64& o, int64_t r0, int64_t nr, int64_t nk, cudaStream_t st, int64_t* nl) {
    const int64_t ld = nk * o.nvir;
    ++*nl;
    return amp_from_tt<double>(o.ts + r0 * ld, o.as + r0 * ld, ld, o.nvir, nr, nk, st);
}

fc_status dens_f64_slab(const DensF64& o, int64_t nk, cudaStream_t st, int64_t* nl) {
    const int64_t nvir = o.nvir, nocc = o.nocc, ld = nk * nvir;
    // P_vv (upper tiles): one GEMM per occupied i, accumulated in order
    const dim3 gv((unsigned)((nvir + DG_BN - 1) / DG_BN), (unsigned)((nvir + DG_BM - 1) / DG_BM), 1);
    for (int64_t i = 0; i < nocc; ++i) {
        const int64_t off = i * nvir * ld;
        EpiStore epi{o.acc_vv, nvir, 1.0, 1};
        dgemm_tn_kernel<EpiStore><<<gv, 256, DG_SMEM, st>>>(o.as + off, ld, o.ts + off, ld, (int)nvir, (int)nvir, ld,
                                                            ld, 1, epi);
    }
    FC_TRY(check_launch("dgemm_tn_kernel<P_vv>"));
    // P_oo: rows i are nvir ld contiguous doubles in both slabs
    const int64_t K = nvir * ld;
    const int64_t kps = ((K + o.splits - 1) / o.splits + DG_BK - 1) / DG_BK * DG_BK;
    const dim3 go((unsigned)((nocc + DG_BN - 1) / DG_BN), (unsigned)((nocc + DG_BM - 1) / DG_BM),
                  (unsigned)o.splits);
    EpiSplit es{o.part_oo, nocc * nocc, (int)nocc};
    FC_CUDA(cudaMemsetAsync(o.part_oo, 0, (size_t)o.splits * nocc * nocc * 8, st));
    dgemm_tn_kernel<EpiSplit><<<go, 256, DG_SMEM, st>>>(o.as, K, o.ts, K, (int)nocc, (int)nocc, K, kps, 0, es);
    FC_TRY(check_launch("dgemm_tn_kernel<P_oo>"));
    oo_fold_f64_kernel<<<(unsigned)((nocc * nocc + 255) / 256), 256, 0, st>>>(o.part_oo, o.splits, nocc * nocc,
                                                                              o.acc_oo);
    *nl += nocc + 2;
    return check_launch("oo_fold_f64_kernel");
}

fc_status dens_f64_finish(const DensF64& o, const DensOut& out, cudaStream_t st, int64_t* nl) {
    const int64_t nv2 = o.nvir * o.nvir, no2 = o.nocc * o.nocc;
    mirror_upper_kernel<<<(unsigned)((nv2 + 255) / 256), 256, 0, st>>>(o.acc_vv, o.nvir);
    FC_CUDA(cudaMemcpyAsync(out.p_vv, o.acc_vv, nv2 * 8, cudaMemcpyDeviceToDevice, st));
    sym_kernel<<<(unsigned)((no2 + 255) / 256), 256, 0, st>>>(o.acc_oo, o.nocc, out.p_oo);
    *nl += 2;
    return check_launch("mirror_upper_kernel");
}

}  // namespace fc
