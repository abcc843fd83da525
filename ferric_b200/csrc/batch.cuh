// Internal state of a prepared RI-MP2 batch: many molecules of uneven size,
// their operands split once per run, persistent launches over all of them,
// the whole sequence captured into one CUDA graph and replayed.
#pragma once
#include <string>
#include <vector>

#include "fc_internal.cuh"

struct fc_rimp2_batch {
    int64_t nmol = 0;
    int precision = 0;
    int grad = 0;
    std::vector<void*> allocs;  // device buffers owned by the batch
    uint64_t bytes = 0;
    double* out = nullptr;      // [nmol][2] (e_os, e_ss) on the device
    int* flags = nullptr;       // [2] range, timeout
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;  // private capture stream
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t items = 0;          // pair-kernel work items (all groups)
    int64_t gemm_tiles = 0;     // adjoint-contraction tiles (all groups)
    int launches = 0;           // kernels in the graph
    int groups = 0;             // amplitude groups (gradient)
    int pair_launches = 0;      // persistent pair-kernel launches in the graph
    double flops = 0.0;         // algorithmic flops of one run
    double ms = 0.0;            // device time of the last timed replay
    std::string plan_json;      // per size bucket: the exchange choice and where it came from
};

namespace fc {
struct BatchMolIn {
    const double* b_ov;
    const double* eps_occ;
    const double* eps_vir;
    int64_t naux, nocc, nvir;
    double* gamma;
    double* de_deps_occ;
    double* de_deps_vir;
};
fc_status batch_alloc(fc_rimp2_batch* b, size_t bytes, void** out);
// Builds the batch's tables and records its launch sequence into b->graph
// (split-BF16 exact-slice kernels).  group_bytes bounds the amplitude
// workspace of one group of molecules (gradient).
// The default choice of the diagonal-tile exchange for items with nk k-steps
// (FERRIC_CUDA_XT=0/1 forces it).
int fx_exchange_choice(int nk, int grad);
// k-steps of the pair kernel over naux (its K tile).
int fx_ksteps(int64_t naux);
// plan[m] (or the default when plan is null): 1 = diagonal tiles of molecule m
// in one phase with the transpose exchanged in shared memory.
fc_status rimp2_batch_build_fx(fc_rimp2_batch* b, const std::vector<BatchMolIn>& mols, size_t group_bytes,
                               const int* plan);
}  // namespace fc
