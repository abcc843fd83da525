/*
 * ferric_cuda.h -- C ABI of libferric_cuda, the B200 (sm_100a) density-fitting
 * contraction library that sits behind ferric's device hooks.
 *
 * Plain pointers, sizes and status codes only.  Every array is row-major
 * (C order, as ndarray stores it) and contiguous.  Functions without a `_dev`
 * suffix take HOST arrays and do their own host<->device copies (the
 * reference hooks are host-array APIs); `_dev` variants take device pointers
 * and a `cudaStream_t` passed as `void*` (NULL = the library's own stream) and
 * return once the work is enqueued.
 *
 * No function falls back to the CPU.  A non-zero status means "not done":
 * the caller keeps the reference's decline-to-CPU behaviour
 * (ferric-mp2/src/rimp2_gpu.rs:105-179, ferric-scf/src/df_j_gpu.rs:622-676).
 * fc_last_error() gives the message of the calling thread's last failure.
 */
#ifndef FERRIC_CUDA_H
#define FERRIC_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1..8 mirror GpuError (ferric-core/src/gpu/device.rs:16-36). */
typedef int32_t fc_status;
#define FC_OK             0
#define FC_ERR_DRIVER     1  /* GpuError::DriverLibrary: CUDA driver unusable      */
#define FC_ERR_BLAS       2  /* GpuError::BlasLibrary (reserved; no BLAS is used) */
#define FC_ERR_DEVICE     3  /* GpuError::Device: no such device / not sm_100      */
#define FC_ERR_POOL_FULL  4  /* GpuError::PoolFull: request exceeds the pool cap   */
#define FC_ERR_LAYOUT     5  /* GpuError::Layout: bad shape, size or overflow      */
#define FC_ERR_CUDA       6  /* GpuError::Cuda: a CUDA call failed                 */
#define FC_ERR_KERNEL     7  /* GpuError::Kernel: kernel image or launch refused   */
#define FC_ERR_RANGE      8  /* GpuError::F32Range: operand outside the mixed range*/
#define FC_ERR_TIMEOUT    9  /* a bounded device wait ran out                      */
#define FC_ERR_INVALID   10  /* null pointer, bad enum, library not initialised   */

/* Arithmetic of the contraction kernels. */
#define FC_PREC_F64        0  /* all-FP64 "plain" kernels: the drop-in             */
#define FC_PREC_MIXED      1  /* exact integer slices: each operand row scaled by  */
                              /* a power of two and split into integer slices      */
                              /* whose tensor-core products sum in accumulators    */
                              /* that never round.  RI-MP2 pair kernel: 4 int8     */
                              /* slices, the 10 products of level <= 3 in 4 int32  */
                              /* sums (tcgen05 kind::i8), (ia|ia) of the i == j    */
                              /* blocks in FP64; adjoint: 3 int8 slices, 6         */
                              /* products; DF-K and the MP2 densities: 3 int8      */
                              /* slices, int32 sums; dressing, Imat: 3 bf16        */
                              /* slices, FP32 sums drained to FP64 before they     */
                              /* could round                                       */
#define FC_PREC_MIXED_FAST 2  /* split-BF16 hi+lo, 3 products, FP32 accumulation   */
                              /* (energy only; ~1e-5 relative, accumulation-bound) */

/* Storage layout of the 3-index tensor handed to fc_dfjk_create. */
#define FC_LAYOUT_SQUARE        0  /* (naux, n, n), symmetric in (mu, nu)          */
#define FC_LAYOUT_PACKED_LOWER  1  /* (naux, n(n+1)/2), rows (mu, nu <= mu)        */

/* Mixed DF-J keeps B as FP32 (the reference's f32 RI-J tier,
 * ferric-scf/src/df_j.rs:33-91) with FP64 accumulation: half the bytes of the
 * bandwidth-bound passes. */

/* Per-call record (the reference's gpu::stats counters, per call). */
typedef struct fc_stats {
    double   kernel_ms;    /* device time of the contraction kernels (CUDA events) */
    double   flops;        /* algorithmic flops of the call                       */
    uint64_t h2d_bytes;    /* host->device bytes copied by the call               */
    uint64_t d2h_bytes;    /* device->host bytes copied by the call               */
    int32_t  precision;    /* FC_PREC_* that ran                                  */
    int32_t  launches;     /* kernels launched by the call                        */
    int32_t  tile_m;       /* tile of the dominant kernel                         */
    int32_t  tile_n;
    int32_t  k_panel;      /* FP64 flush interval of mixed kernels (0 = none)     */
    int32_t  main_launches;/* launches of the dominant kernel                      */
    double   main_ms;      /* device time of the dominant kernel, all its launches */
    double   main_flops;   /* algorithmic flops done by the dominant kernel        */
    double   main_bytes;   /* algorithmic bytes moved by the dominant kernel       */
    int32_t  aux_launches; /* launches of the second kernel (RI-MP2 gradient: the  */
    int32_t  reserved_;    /* adjoint contraction Gamma += 4 B Tt^T), 0 if none    */
    double   aux_ms;       /* its device time, all its launches (CUDA events)      */
    double   aux_flops;    /* its algorithmic flops                                */
    double   aux_bytes;    /* its algorithmic bytes                                */
} fc_stats;

/* ---- library ------------------------------------------------------------ */

/* Select `device` (ordinal) and cap the library's device allocations at
 * `pool_bytes` (0 = no cap).  Replaces gpu::install/decide + DevicePool
 * (ferric-core/src/gpu/mod.rs:110-373, ferric-core/src/gpu/pool.rs:1-30).
 * Idempotent for the same device. */
fc_status   fc_init(int32_t device, uint64_t pool_bytes);
/* Free every cached workspace of the library.  Handles stay valid. */
fc_status   fc_release_workspace(void);
/* Bytes currently held by the library on the device (workspaces + handles). */
uint64_t    fc_pool_used(void);
/* Copy the calling thread's last error message into buf (NUL-terminated);
 * returns the full message length. */
size_t      fc_last_error(char* buf, size_t len);
const char* fc_version(void);

/* ---- RI-MP2 ---------------------------------------------------------------
 * b_ov: (naux, nocc*nvir), column i*nvir + a, dressed B_Q,ia.
 * eps_occ[nocc], eps_vir[nvir]: active occupied / virtual orbital energies
 * (the reference's eps[first_occ + i], eps[nocc_total + a]).
 *
 * Replaces try_spin_components_on_device (ferric-mp2/src/rimp2_gpu.rs:105-170)
 * and the CPU pair loop (ferric-mp2/src/rimp2.rs:1399-1544).
 * has_kappa != 0 applies the kappa damping (1 - exp(kappa*D))^2
 * (rimp2.rs:1425-1437); it is FP64 only, as mixed_energy_operator allows mixed
 * only without kappa (rimp2.rs:1293-1300).  e_os/e_ss are host scalars. */
fc_status fc_rimp2_energy(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                          const double* eps_occ, const double* eps_vir,
                          int32_t has_kappa, double kappa, int32_t precision,
                          double* e_os, double* e_ss, fc_stats* stats);
fc_status fc_rimp2_energy_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                              const double* eps_occ, const double* eps_vir,
                              int32_t has_kappa, double kappa, int32_t precision,
                              double* e_os, double* e_ss, void* stream, fc_stats* stats);

/* Energy plus its adjoint: gamma[P, ia] = dE/dB[P, ia] (naux x nocc*nvir,
 * = 4 x_ov of ferric-mp2/src/zvector.rs:651-703, rimp2.rs:1832-1836),
 * de_docc[i] = dE/d eps_occ[i] and de_dvir[a] = dE/d eps_vir[a]
 * (= 2 diag(P_oo), 2 diag(P_vv) of ferric-mp2/src/oo_rimp2.rs:1170-1300).
 * E = E_os + E_ss.  No amplitudes are stored: occupied-pair blocks are
 * recomputed.  In the host form, page-locked b_ov and gamma let the copies
 * overlap the compute (b_ov goes up in occupied chunks as FC_PREC_MIXED
 * needs them, gamma comes down in column blocks as they are final);
 * pageable buffers are copied before and after.  In the _dev form
 * e_os/e_ss are host scalars and the call synchronises its stream before
 * returning. */
fc_status fc_rimp2_energy_grad(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                               const double* eps_occ, const double* eps_vir, int32_t precision,
                               double* e_os, double* e_ss, double* gamma,
                               double* de_docc, double* de_dvir, fc_stats* stats);
fc_status fc_rimp2_energy_grad_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                   const double* eps_occ, const double* eps_vir, int32_t precision,
                                   double* e_os, double* e_ss, double* gamma,
                                   double* de_docc, double* de_dvir, void* stream,
                                   fc_stats* stats);

/* The gradient call plus the full unrelaxed MP2 densities the reference's
 * gradient chain takes (build_mp2_density, ferric-mp2/src/oo_rimp2.rs:
 * 1170-1300; Mp2Intermediates::from_ri_densities, ferric-mp2/src/rimp2.rs:
 * 1841-1883, with x_ov = gamma / 4):
 *   p_oo[i*nocc + j] = -sum_kab t_ik^ab (2 t_jk^ab - t_jk^ba)   (nocc x nocc)
 *   p_vv[a*nvir + b] =  sum_ijc t_ij^ac (2 t_ij^bc - t_ij^cb)   (nvir x nvir)
 * row-major and symmetric.  The chunk pairs run by column chunk and each
 * column's amplitude blocks are held as one slab (FC_PREC_MIXED: int8 slices
 * of t and 2t - t^T, 6 B per element, at most four chunk budgets;
 * FC_PREC_F64: 16 B per element).  FC_PREC_MIXED runs each chunk pair once
 * and keeps the blocks above the diagonal in FP32 until their column (at
 * most eight chunk budgets, else -- or with FERRIC_CUDA_DENS_STORE=0 -- the
 * chunk pairs off the diagonal run once per column, as in FC_PREC_F64).
 * Slabs and kept blocks are library workspace: they stay allocated for the
 * next call until fc_release_workspace.  Otherwise as fc_rimp2_energy_grad /
 * _dev (gamma, de_docc, de_dvir as there). */
fc_status fc_rimp2_energy_grad_dens(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                    const double* eps_occ, const double* eps_vir, int32_t precision,
                                    double* e_os, double* e_ss, double* gamma, double* de_docc,
                                    double* de_dvir, double* p_oo, double* p_vv, fc_stats* stats);
fc_status fc_rimp2_energy_grad_dens_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                        const double* eps_occ, const double* eps_vir, int32_t precision,
                                        double* e_os, double* e_ss, double* gamma, double* de_docc,
                                        double* de_dvir, double* p_oo, double* p_vv, void* stream,
                                        fc_stats* stats);

/* One system over nshards processes (one GPU each), partitioned by occupied
 * pairs.  The reference's MPI RI-MP2 (ferric-mp2/src/mpi_rimp2.rs:16-43)
 * cuts aux bands and all-reduces per-i intermediates; here every process
 * holds all of B_ov and takes a balanced share of the pairs, so the only
 * collectives are on the results.  Each call returns this shard's partial
 * sums: e_os, e_ss, gamma (all naux x nocc*nvir entries, zero outside this
 * shard's contributions), de_docc, de_dvir; their sum over the shards is the
 * unsharded result (FP64: to summation order; FC_PREC_MIXED: the amplitude
 * blocks are split at their own row scales, as with a smaller chunk budget).
 * The caller adds them with its collectives (all-reduce of the scalars and
 * dE/deps, reduce-scatter of gamma by aux rows).  No counterpart in the
 * reference, which has no occupied-pair partition. */
fc_status fc_rimp2_energy_shard_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                    const double* eps_occ, const double* eps_vir, int32_t has_kappa,
                                    double kappa, int32_t precision, int32_t shard, int32_t nshards,
                                    double* e_os, double* e_ss, void* stream, fc_stats* stats);
fc_status fc_rimp2_energy_grad_shard_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                         const double* eps_occ, const double* eps_vir, int32_t precision,
                                         int32_t shard, int32_t nshards, double* e_os, double* e_ss,
                                         double* gamma, double* de_docc, double* de_dvir, void* stream,
                                         fc_stats* stats);
/* The occupied pairs (i <= j, as (i, j) int32 pairs into ij[2 * cap]) that
 * shard `shard` of `nshards` computes in the energy (grad = 0) or energy +
 * gradient (grad = 1) call under the current chunk budget.  Host only: needs
 * no device and no fc_init.  *npairs receives the count (ij may be NULL to
 * query it). */
fc_status fc_rimp2_shard_pairs(int64_t nocc, int64_t nvir, int32_t precision, int32_t grad, int32_t shard,
                               int32_t nshards, int32_t* ij, int64_t cap, int64_t* npairs);

/* Unrestricted RI-MP2 energy components (alpha-alpha, beta-beta,
 * alpha-beta), the device part of u_ri_mp2: same_spin_block_energy and
 * opposite_spin_block_energy (ferric-mp2/src/u_rimp2.rs:693-753), with the
 * reference's device path try_u_{same,opposite}_spin_on_device
 * (ferric-mp2/src/rimp2_gpu.rs:884-1038).  b_a (naux, nocc_a*nvir_a) and
 * b_b (naux, nocc_b*nvir_b) share naux; SCS/SOS weights are applied by the
 * caller (e_corr = c_os e_ab + c_ss (e_aa + e_bb)).  FC_PREC_F64 or
 * FC_PREC_MIXED (exact slices). */
fc_status fc_ump2_energy(const double* b_a, int64_t nocc_a, int64_t nvir_a, const double* eps_occ_a,
                         const double* eps_vir_a, const double* b_b, int64_t nocc_b, int64_t nvir_b,
                         const double* eps_occ_b, const double* eps_vir_b, int64_t naux, int32_t precision,
                         double* e_aa, double* e_bb, double* e_ab, fc_stats* stats);
fc_status fc_ump2_energy_dev(const double* b_a, int64_t nocc_a, int64_t nvir_a, const double* eps_occ_a,
                             const double* eps_vir_a, const double* b_b, int64_t nocc_b, int64_t nvir_b,
                             const double* eps_occ_b, const double* eps_vir_b, int64_t naux, int32_t precision,
                             double* e_aa, double* e_bb, double* e_ab, void* stream, fc_stats* stats);

/* RI Lagrangian Imat (nmo x nmo, row-major), the first consumer of the
 * RI-MP2 adjoint in the analytic gradient (build_imat_ri / imat_fill_rows,
 * ferric-mp2/src/zvector.rs:735-832):
 *   Imat[q, fo + i] = -2 sum_{P,a} x_ov[P, i*nvir + a] b_full[P, q, fo + nocc + a]
 *   Imat[q, fo + nocc + a] = -2 sum_{P,i} x_ov[P, i*nvir + a] b_full[P, q, fo + i]
 * with x_ov = Gamma / 4 (naux, nocc*nvir) and b_full the dressed MO 3-index
 * tensor (naux, nmo, nmo); fo = first_occ, frozen-core columns zero.
 * FC_PREC_F64 or FC_PREC_MIXED (exact slices, k-panel FP64 flush). */
fc_status fc_rimp2_imat(const double* x_ov, const double* b_full, int64_t naux, int64_t nmo, int64_t nocc,
                        int64_t nvir, int64_t first_occ, int32_t precision, double* imat, fc_stats* stats);
fc_status fc_rimp2_imat_dev(const double* x_ov, const double* b_full, int64_t naux, int64_t nmo, int64_t nocc,
                            int64_t nvir, int64_t first_occ, int32_t precision, double* imat, void* stream,
                            fc_stats* stats);

/* The GEMM-shaped part of the RI 3c/2c integral response of the RI-MP2
 * gradient, for one channel of weight w (integral_response_gradient_3c2c /
 * ri_response_gradient_channels, ferric-mp2/src/gradient.rs:559-887; w = 2
 * closed shell, 1 per spin):
 *   y_ov     = V^{-1/2 T} x_ov                          (naux x nov)
 *   gamma_2c = -w (V^{-1/2 T} b_ov) y_ov^T               (naux x naux)
 *   g3c[P]   = w (G_P + G_P^T), G_P = C_occ Y_P C_vir^T  (nbf x nbf)
 * Y_P = row P of y_ov as nocc x nvir; v_inv_sqrt (naux x naux), c_occ
 * (nbf x nocc), c_vir (nbf x nvir), all row-major FP64.  g3c is produced for
 * the aux slab [p0, p0 + np) (np x nbf x nbf), as the reference builds it per
 * aux shell for the derivative integrals, which stay with the caller.  FP64
 * throughout (DMMA).  The _dev forms take device pointers and synchronise
 * their stream before returning; the host form of _3c uploads only the rows
 * [p0, p0 + np) of y_ov. */
fc_status fc_rimp2_response_2c(const double* x_ov, const double* b_ov, const double* v_inv_sqrt, int64_t naux,
                               int64_t nov, double weight, double* y_ov, double* gamma_2c, fc_stats* stats);
fc_status fc_rimp2_response_2c_dev(const double* x_ov, const double* b_ov, const double* v_inv_sqrt, int64_t naux,
                                   int64_t nov, double weight, double* y_ov, double* gamma_2c, void* stream,
                                   fc_stats* stats);
fc_status fc_rimp2_response_3c(const double* y_ov, const double* c_occ, const double* c_vir, int64_t naux,
                               int64_t nocc, int64_t nvir, int64_t nbf, int64_t p0, int64_t np, double weight,
                               double* g3c, fc_stats* stats);
fc_status fc_rimp2_response_3c_dev(const double* y_ov, const double* c_occ, const double* c_vir, int64_t naux,
                                   int64_t nocc, int64_t nvir, int64_t nbf, int64_t p0, int64_t np, double weight,
                                   double* g3c, void* stream, fc_stats* stats);

/* FP64 RI-MP2 energy that allocates no device memory.  No counterpart in the
 * reference: it is for callers that cannot call cudaMalloc -- callers whose
 * device memory belongs to another allocator (ferric's device-pool ledger
 * charges every byte to a reservation and refuses past it; a framework's
 * caching allocator may hold nearly all of the device) and inner loops that
 * must not take cudaMalloc/cudaFree's implicit device synchronisation.
 * Arguments are device pointers as in fc_rimp2_energy_dev; e_os/e_ss are host
 * scalars; the call synchronises `stream` (NULL = the legacy default stream)
 * and does not need fc_init.  Its scratch is a fixed 4 MiB array inside the
 * library, held by every device that loads the library until the process
 * exits; problems needing more (about 262,000 tiles of 64 x 64 virtual
 * indices, i.e. nocc(nocc+1)/2 * T(T+1)/2 with T = ceil(nvir/64)) are refused with
 * FC_ERR_LAYOUT.  The first call on a device looks up the array's device
 * address and sets the kernel's shared-memory limit; make that first call
 * before any stream capture.  All calls on a device share the one array
 * (each call writes every byte it later reads, so earlier contents do not
 * matter), so two calls that overlapped on the GPU would race on it.  The
 * function rules that out within a process: it holds one process-wide lock
 * from its first launch until its stream has finished, so calls from
 * different threads or streams run one after another, and calls on
 * different devices also queue behind each other.  Separate processes each
 * have their own copy of the array. */
fc_status fc_rimp2_energy_noalloc(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                  const double* eps_occ, const double* eps_vir,
                                  int32_t has_kappa, double kappa,
                                  double* e_os, double* e_ss, void* stream);

/* ---- Batched RI-MP2 --------------------------------------------------------
 * Many molecules of uneven size (naux, nocc, nvir) in one CUDA graph.  The
 * reference has no batched entry point: its callers loop over
 * spin_components (ferric-mp2/src/rimp2.rs:1445-1544) and the adjoint
 * (rimp2.rs:1832-1836) one molecule at a time; this replaces that loop.
 * All pointers of a descriptor are device pointers and stay valid (and at
 * the same address) for the life of the batch; their contents may change
 * between replays.  gamma (naux x nocc*nvir), de_deps_occ [nocc] and
 * de_deps_vir [nvir] are all set (energy + gradient) or all NULL (energy
 * only), the same for every molecule.  Only FC_PREC_MIXED (exact integer
 * slices) is batched; FP64 is one fc_rimp2_energy_grad_dev call per
 * molecule.  create splits nothing yet: it sizes and allocates the batch's
 * buffers, builds its work tables and records the launch sequence (split
 * kernels, persistent pair and adjoint kernels over all molecules' tiles,
 * reductions) into a graph; replay enqueues that graph on `stream` (NULL =
 * the batch's own stream); energies waits for the last replay and returns
 * its per-molecule e_os, e_ss (host arrays of nmol).  The amplitudes of the
 * gradient are held for a group of molecules at a time; the environment
 * variable FERRIC_CUDA_BATCH_GROUP_BYTES bounds that workspace (default
 * 16 GiB).  A batch is used by one thread at a time. */
typedef struct fc_mol_desc {
    const double* b_ov;      /* (naux, nocc*nvir), column i*nvir + a */
    const double* eps_occ;   /* [nocc] */
    const double* eps_vir;   /* [nvir] */
    int64_t naux, nocc, nvir;
    double* gamma;           /* (naux, nocc*nvir) = dE/dB_ov, or NULL */
    double* de_deps_occ;     /* [nocc], or NULL */
    double* de_deps_vir;     /* [nvir], or NULL */
} fc_mol_desc;

typedef struct fc_rimp2_batch fc_rimp2_batch;

typedef struct fc_batch_info {
    int64_t nmol;
    int64_t items;           /* pair-kernel work items (molecule, i, j, tile pair) */
    int64_t gemm_tiles;      /* adjoint-contraction tiles */
    int32_t launches;        /* kernels recorded in the graph */
    int32_t groups;          /* amplitude groups (gradient) */
    int32_t pair_launches;   /* persistent pair-kernel launches */
    int32_t precision;
    int32_t grad;
    int32_t tile_m, tile_n, k_panel;
    double flops;            /* algorithmic flops of one replay */
    double last_ms;          /* device time of the last replay read by _energies */
    uint64_t bytes;          /* device memory held by the batch */
} fc_batch_info;

fc_status fc_rimp2_batched_create(const fc_mol_desc* mols, int64_t nmol, int32_t precision,
                                  fc_rimp2_batch** out);
fc_status fc_rimp2_batched_replay(fc_rimp2_batch* b, void* stream);
fc_status fc_rimp2_batched_energies(fc_rimp2_batch* b, double* e_os, double* e_ss);
fc_status fc_rimp2_batched_info(const fc_rimp2_batch* b, fc_batch_info* info);
/* The batch's schedule per size bucket, as a JSON array (NUL-terminated
 * into buf, returns the full length): bucket key ("grad"/"energy", virtual
 * tiles of 128, k-steps of 64), molecules, tile shape, the diagonal-tile
 * exchange choice and its source ("tuned": measured by the autotuner when
 * FERRIC_CUDA_AUTOTUNE=1, or read from FERRIC_CUDA_AUTOTUNE_CACHE;
 * "default"; "forced" by FERRIC_CUDA_XT), with the measured times. */
size_t fc_rimp2_batched_plan(const fc_rimp2_batch* b, char* buf, size_t len);
fc_status fc_rimp2_batched_destroy(fc_rimp2_batch* b);
/* create + replay + energies + destroy. */
fc_status fc_rimp2_batched(const fc_mol_desc* mols, int64_t nmol, int32_t precision,
                           double* e_os, double* e_ss);

/* ---- MO transform and metric dressing (the step before the RI-MP2 path) -----
 * B[P, l*nright + r] = sum_Q M[P, Q] (Q|lr),
 * (Q|lr) = sum_{mu nu} C_left[mu, l] (Q|mu nu) C_right[nu, r]
 * (stream_dressed_mo_band, ferric-mp2/src/rimp2.rs:648-737; with C_left = C_occ
 * and C_right = C_vir, B is the B_ov of the RI-MP2 entry points).  eri3:
 * (naux, n, n) row-major, symmetric in (mu, nu); m: (naux, naux) row-major
 * (V^-1/2 or L^-1); c_left (n x nleft), c_right (n x nright) row-major;
 * b: (naux, nleft*nright).  FC_PREC_F64: FP64 throughout; FC_PREC_MIXED:
 * the two half transforms in FP64 and the dressing GEMM (2 naux^2 nleft
 * nright flops, the dominant term) as exact-slice split-BF16 on the tensor
 * cores.  The host variant copies eri3 in aux chunks. */
fc_status fc_mo_dress(const double* eri3, int64_t naux, int64_t n, const double* m,
                      const double* c_left, int64_t nleft, const double* c_right, int64_t nright,
                      int32_t precision, double* b, fc_stats* stats);
fc_status fc_mo_dress_dev(const double* eri3, int64_t naux, int64_t n, const double* m,
                          const double* c_left, int64_t nleft, const double* c_right, int64_t nright,
                          int32_t precision, double* b, void* stream, fc_stats* stats);

/* ---- DF-JK ----------------------------------------------------------------
 * A handle owns the device copy of the 3-index tensor for the lifetime of a
 * builder (the reference's per-builder DeviceSlot, ferric-scf/src/df_j_gpu.rs:1-5,
 * df_k_gpu.rs:1-4).  Without a metric the tensor is taken as dressed,
 * B = L^-1 (P|mn), and J = B^T (B . D).  A handle is used by one thread at a
 * time. */
typedef struct fc_dfjk fc_dfjk;

fc_status fc_dfjk_create(const double* b, int64_t naux, int64_t n, int32_t layout,
                         int32_t precision, fc_dfjk** out);
fc_status fc_dfjk_create_dev(const double* b, int64_t naux, int64_t n, int32_t layout,
                             int32_t precision, void* stream, fc_dfjk** out);
/* Raw (P|mn) form: l = lower Cholesky factor of the metric V = L L^T
 * (naux x naux, row-major); each J build then solves V c = d on the device
 * (DfJ::solve_metric, ferric-scf/src/df_j.rs:931). */
fc_status fc_dfj_set_metric_chol(fc_dfjk* h, const double* l);
/* J = sum_P B_P c_P, c = V^-1 d, d_P = <B_P, D>  (JBuilder::build,
 * ferric-scf/src/fock.rs:10-19; df_j.rs:1459-1572).  d, j: n x n. */
fc_status fc_dfj_build(fc_dfjk* h, const double* d, double* j, fc_stats* stats);
fc_status fc_dfj_build_dev(fc_dfjk* h, const double* d, double* j, void* stream,
                           fc_stats* stats);
/* K = sum_Q (B_Q C)(B_Q C)^T for c_occ (n x nocc); no occupation factor
 * (KBuilder::build_from_occ, ferric-scf/src/fock.rs:22-52;
 * df_k.rs:1409-1520).  FC_LAYOUT_SQUARE handles only. */
fc_status fc_dfk_build_occ(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k,
                           fc_stats* stats);
fc_status fc_dfk_build_occ_dev(fc_dfjk* h, const double* c_occ, int64_t nocc, double* k,
                               void* stream, fc_stats* stats);
/* J and K of one occupied-orbital matrix in one call (square handles):
 * K exactly as fc_dfk_build_occ, and j = J(C_occ C_occ^T), the density of
 * build_from_occ with no occupation factor.  J's first pass d_P =
 * <B_P, C C^T> = sum_mu (B_P C)[mu, :] . C[mu, :] is read off the K stage's
 * W = B C, so B is read once for K's stage 1 and once for J's second pass
 * (instead of two passes for J); the metric solve (fc_dfj_set_metric_chol)
 * applies as in fc_dfj_build; J's second pass runs on the library's side
 * stream, overlapping the rest of DF-K, and the call's stream waits for it
 * before the call returns.  No counterpart in the reference, whose RHF
 * calls JBuilder::build(D) and KBuilder::build_from_occ(C_occ) with
 * D = 2 C_occ C_occ^T (ferric-scf/src/rhf.rs:3164-3178): J(D) = 2 j here.
 * stats: kernel_ms/flops of the whole call, main_* of the K stages, aux_*
 * of J's second pass. */
fc_status fc_dfjk_build_occ(fc_dfjk* h, const double* c_occ, int64_t nocc, double* j, double* k,
                            fc_stats* stats);
fc_status fc_dfjk_build_occ_dev(fc_dfjk* h, const double* c_occ, int64_t nocc, double* j, double* k,
                                void* stream, fc_stats* stats);
/* Precision of the handle's next builds: FC_PREC_F64 always works (the FP64
 * tensor stays resident beside the mixed copy); the handle's creation
 * precision switches back.  This is how the SCF precision ladder
 * (ferric-scf/src/jk_ladder.rs:312-430) publishes its per-build decision. */
fc_status fc_dfjk_set_precision(fc_dfjk* h, int32_t precision);
fc_status fc_dfjk_destroy(fc_dfjk* h);

/* Self-check: out[k] = the mixed pair epilogue's FP64 reciprocal of d[k]
 * (host arrays, n <= 2^31), evaluated on the device: an FP32 seed refined by
 * the third-order Newton-Raphson step, which the tests hold to the
 * correctly rounded 1 / d (CUDA's FP64 division) within 1 ulp. */
fc_status fc_check_recip(const double* d, int64_t n, double* out);

#ifdef __cplusplus
}
#endif
#endif /* FERRIC_CUDA_H */
