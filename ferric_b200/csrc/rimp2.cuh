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

fc_status rimp2_energy_f64(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                           fc_stats* stats);
fc_status rimp2_grad_f64(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                         double* gamma, double* de_docc, double* de_dvir, fc_stats* stats,
                         const GammaSink* sink = nullptr);

// Tensor-core (tcgen05) kernel sets.  _fx: int8 integer slices with exact
// int32 accumulation (FC_PREC_MIXED).  _mixed: floating bf16 hi+lo split, 3
// products, FP32 accumulation (FC_PREC_MIXED_FAST; energy only).
fc_status rimp2_energy_mixed(const Rimp2Dev& d, int terms, cudaStream_t st, double* e_os,
                             double* e_ss, fc_stats* stats);
fc_status rimp2_energy_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss,
                          fc_stats* stats);
fc_status rimp2_grad_fx(const Rimp2Dev& d, cudaStream_t st, double* e_os, double* e_ss, double* gamma,
                        double* de_docc, double* de_dvir, fc_stats* stats, const GammaSink* sink = nullptr);
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
