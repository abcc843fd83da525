// Internal interface of the RI-MP2 kernel sets (device pointers only).
#pragma once
#include <vector>
#include "fc_internal.cuh"

namespace fc {

struct Rimp2Dev {
    const double* b_ov;     // (naux, nocc*nvir) on the device
    const double* eps_occ;  // [nocc] on the device
    const double* eps_vir;  // [nvir] on the device
    int64_t naux, nocc, nvir;
    int has_kappa;
    double kappa;
    int64_t chunk_bytes;    // amplitude-chunk budget of the gradient
    int shard = 0;          // this process's share of the occupied pairs (of nshards)
    int nshards = 1;
    // optional (mixed gradient): b_ov arrives in occupied chunks of arrive_cc
    // orbitals, chunk J complete when arrive[J] has fired; the driver prepares
    // a chunk after its event, so the upload overlaps the first chunk pairs
    const cudaEvent_t* arrive = nullptr;
    int64_t arrive_cc = 0;
};

// Occupied-pair sharding of one system over nshards processes (the same
// partition in every process; the sum over shards of each call's E, Gamma
// and dE/deps is the unsharded result).
// Energy: pairs i <= j in i-major order, shard s computes [lo, hi).
void shard_pair_range(int64_t nocc, int shard, int nshards, int64_t* lo, int64_t* hi);
// Gradient: occupied chunks of size cc, chunk pairs (I <= J) in I-major
// order; the owner of each is the shard whose share of the total pair count
// holds the chunk pair's midpoint (contiguous, balanced ranges).
std::vector<int> chunk_pair_owner(int64_t nocc, int64_t cc, int nshards);
// Chunk sizes of the two gradient drivers for an amplitude budget, capped
// with several shards so that there are at least 8 chunk pairs per shard.
int64_t grad_chunk_fx(int64_t nocc, int64_t nvir, int64_t budget, int nshards);
int64_t grad_chunk_f64(int64_t nocc, int64_t nvir, int64_t budget, int nshards);

// Where the gradient's Gamma goes as its column blocks become final: a
// pinned host array (naux x nov, row-major) and a copy stream; the block of
// occupied chunk I is final once every chunk pair (I, J >= I) has run, and is
// copied out on `stream` while later chunk pairs compute.
struct GammaSink {
    double* host;
    cudaStream_t stream;
    cudaEvent_t ready;
};

// Unrelaxed MP2 densities (device, row-major, zeroed by nobody: the
// gradient drivers write every element): p_oo (nocc x nocc), p_vv (nvir x nvir).
struct DensOut {
    double* p_oo;
    double* p_vv;
};

fc_status rimp2_energy_f64(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                           fc_stats* stats);
fc_status rimp2_grad_f64(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                         double* gamma, double* de_docc, double* de_dvir, fc_stats* stats,
                         const GammaSink* sink = nullptr, const DensOut* dens = nullptr);

// Tensor-core (tcgen05) kernel sets.  _fx: int8 integer slices with exact
// int32 accumulation (FC_PREC_MIXED).  _mixed: floating bf16 hi+lo split, 3
// products, FP32 accumulation (FC_PREC_MIXED_FAST; energy only).
fc_status rimp2_energy_mixed(const Rimp2Dev& d, int terms, cudaStream_t st, double* e_os,
                             double* e_ss, fc_stats* stats);
fc_status rimp2_energy_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                          fc_stats* stats);
fc_status rimp2_grad_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss, double* gamma,
                        double* de_docc, double* de_dvir, fc_stats* stats, const GammaSink* sink = nullptr,
                        const DensOut* dens = nullptr);

// ---- densities over amplitude slabs (rimp2_dens.cu) ----
// With densities the gradient drivers take their chunk pairs by column
// chunk K: the slab of K holds the amplitude blocks (I, K) of every occupied
// chunk I, i.e. rows (i, a) of all i and columns (k, b) of k in K, at row
// pitch tp (>= nvir) and column pitch ld = |K| tp.
//
// FC_PREC_MIXED: three int8 slices of Tt and of t per slab row.
struct DensFx {
    int64_t nocc, nvir, tp, rows;  // rows = nocc tp (slice stride of the slabs)
    int8_t* ts;                    // [3][rows][ld] slices of Tt (the adjoint's operand)
    int8_t* as;                    // [3][rows][ld] slices of t
    double* tsc;                   // [rows] row scales of ts
    double* asc;                   // [rows] row scales of as
    double* tscT;                  // [nvir][nocc] ts scales, transposed (P_oo)
    double* ascT;                  // [nvir][nocc] as scales, transposed
    double* part_vv;               // [grid_vv][128 x 128] partial P_vv tiles
    double* part_oo;               // [grid_oo][128 x 128] partial P_oo tiles
    int4* items;                   // per-slab work items (P_vv, then P_oo)
    int ntp_vv, g_vv, ntp_oo, g_oo;
};
// Largest chunk (occupied orbitals per column) whose slabs fit `budget`
// bytes (at least 1, at most cc).
int64_t dens_chunk_fx(int64_t nocc, int64_t nvir, int64_t cc, int64_t budget);
fc_status dens_fx_alloc(int64_t nocc, int64_t nvir, int64_t tp, int64_t cc, cudaStream_t st, DensFx* o);
// Block (rows r0 .. r0 + nr tp of the slab, FP32 Tt at pitch ld = nk tp):
// Tt -> t in place, then t's slices into the slab.  The Tt slices are the
// adjoint's, written into the slab by the caller.
fc_status dens_fx_block(const DensFx& o, float* blk, int64_t r0, int64_t nr, int64_t nk, cudaStream_t st,
                        int64_t* nl);
// The slab of a column chunk of nk orbitals is complete: add its P terms.
fc_status dens_fx_slab(const DensFx& o, int64_t nk, cudaStream_t st, int* err, int64_t* nl);
// Fold the partials into the outputs (after the last slab).
fc_status dens_fx_finish(const DensFx& o, const DensOut& out, cudaStream_t st, int64_t* nl);

// FC_PREC_F64: FP64 slabs of Tt and t.
struct DensF64 {
    int64_t nocc, nvir;
    double* ts;       // [nocc nvir][ld]
    double* as;       // [nocc nvir][ld]
    double* part_oo;  // [splits][nocc x nocc]
    double* acc_vv;   // [nvir x nvir] running P_vv (upper tiles)
    double* acc_oo;   // [nocc x nocc] running P_oo
    int splits;
};
int64_t dens_chunk_f64(int64_t nocc, int64_t nvir, int64_t cc, int64_t budget);
fc_status dens_f64_alloc(int64_t nocc, int64_t nvir, int64_t cc, cudaStream_t st, DensF64* o);
// Block rows r0 .. r0 + nr nvir of the Tt slab (pitch nk nvir): t into the t slab.
fc_status dens_f64_block(const DensF64& o, int64_t r0, int64_t nr, int64_t nk, cudaStream_t st, int64_t* nl);
fc_status dens_f64_slab(const DensF64& o, int64_t nk, cudaStream_t st, int64_t* nl);
fc_status dens_f64_finish(const DensF64& o, const DensOut& out, cudaStream_t st, int64_t* nl);
// Copy Gamma's columns of occupied rows [r0, r0 + nr) to the sink once `st`
// has reached this point.
fc_status gamma_sink_block(const GammaSink* sink, const double* gamma, int64_t naux, int64_t nov, int64_t nvir,
                           int64_t r0, int64_t nr, cudaStream_t st);

// One spin channel of unrestricted RI-MP2 (device pointers).
struct UmpSpin {
    const double* b_ov;     // (naux, nocc*nvir)
    const double* eps_occ;  // [nocc]
    const double* eps_vir;  // [nvir]
    int64_t nocc, nvir;
};
// Opposite-spin energy sum_{i a J B} (ia|JB)^2 / D: FP64 DMMA, or exact
// slices on tcgen05.
fc_status ump2_cross_f64(const UmpSpin& a, const UmpSpin& b, int64_t naux, cudaStream_t st, double* e_ab,
                         fc_stats* stats);
fc_status ump2_cross_fx(const UmpSpin& a, const UmpSpin& b, int64_t naux, cudaStream_t st, double* e_ab,
                        fc_stats* stats);

}  // namespace fc
