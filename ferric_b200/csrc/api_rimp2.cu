// extern "C" RI-MP2 entry points: argument checks, host<->device staging and
// precision dispatch.  Replaces the reference's device hook
// try_spin_components_on_device / spin_components_on_device
// (ferric-mp2/src/rimp2_gpu.rs:105-471) and the host gradient intermediates
// x_ov / P (ferric-mp2/src/zvector.rs:651-703, oo_rimp2.rs:1170-1300).
#include <algorithm>
#include "fc_internal.cuh"
#include "rimp2.cuh"

#include <cmath>
#include <cstdlib>

using namespace fc;

namespace {

fc_status check_shapes(const void* b_ov, int64_t naux, int64_t nocc, int64_t nvir, const void* eo,
                       const void* ev, int32_t precision, int32_t has_kappa, double kappa,
                       const void* e_os, const void* e_ss) {
    if (!e_os || !e_ss) return fail(FC_ERR_INVALID, "RI-MP2: null output pointer");
    if (naux < 0 || nocc < 0 || nvir < 0) return fail(FC_ERR_LAYOUT, "RI-MP2: negative dimension");
    int64_t nov, nb;
    if (!mul_ok(nocc, nvir, &nov) || !mul_ok(nov, naux, &nb) || !mul_ok(nb, 8, &nb))
        return fail(FC_ERR_LAYOUT, "RI-MP2: naux*nocc*nvir overflows");
    if (nocc > 1 << 20 || nvir > 1 << 24) return fail(FC_ERR_LAYOUT, "RI-MP2: nocc/nvir out of range");
    if (nov && naux && (!b_ov || !eo || !ev)) return fail(FC_ERR_INVALID, "RI-MP2: null input pointer");
    if (precision < FC_PREC_F64 || precision > FC_PREC_MIXED_FAST)
        return fail(FC_ERR_INVALID, "RI-MP2: unknown precision " + std::to_string(precision));
    if (has_kappa && precision != FC_PREC_F64)
        return fail(FC_ERR_INVALID,
                    "RI-MP2: kappa damping runs in FP64 only (mixed is defined without kappa)");
    if (has_kappa && !(std::isfinite(kappa) && kappa > 0.0))
        return fail(FC_ERR_INVALID, "RI-MP2: kappa must be finite and > 0");
    return FC_OK;
}

// The context's copy stream and event for Gamma blocks (created once).
fc_status copy_stream(cudaStream_t* s, cudaEvent_t* e) {
    static cudaStream_t cs = nullptr;
    static cudaEvent_t ce = nullptr;
    if (!cs) {
        FC_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        FC_CUDA(cudaEventCreateWithFlags(&ce, cudaEventDisableTiming));
    }
    *s = cs;
    *e = ce;
    return FC_OK;
}

// Stream and per-chunk events of the chunked upload of b_ov (host API).
fc_status upload_stream(cudaStream_t* s, std::vector<cudaEvent_t>** evs, size_t n) {
    static cudaStream_t us = nullptr;
    static std::vector<cudaEvent_t> ev;
    if (!us) FC_CUDA(cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking));
    while (ev.size() < n) {
        cudaEvent_t e;
        FC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev.push_back(e);
    }
    *s = us;
    *evs = &ev;
    return FC_OK;
}

int64_t chunk_budget() {
    int64_t b = int64_t(8) << 30;
    if (const char* s = std::getenv("FERRIC_CUDA_CHUNK_BYTES")) {
        long long v = std::atoll(s);
        if (v > 0) b = v;
    }
    Context& c = ctx();
    if (c.pool_cap) {
        int64_t left = (int64_t)c.pool_cap - (int64_t)(ws_bytes() + c.handle_bytes);
        if (left / 2 < b) b = left / 2 > 0 ? left / 2 : 1;
    }
    return b;
}

fc_status energy_dispatch(const Rimp2Dev& d, int32_t precision, cudaStream_t st, double* e_os,
                          double* e_ss, fc_stats* stats) {
    if (precision == FC_PREC_F64) return rimp2_energy_f64(d, st, e_os, e_ss, stats);
    if (precision == FC_PREC_MIXED) return rimp2_energy_fx(d, st, e_os, e_ss, stats);
    return rimp2_energy_mixed(d, 2, st, e_os, e_ss, stats);
}

fc_status grad_dispatch(const Rimp2Dev& d, int32_t precision, cudaStream_t st, double* e_os,
                        double* e_ss, double* gamma, double* de_docc, double* de_dvir,
                        fc_stats* stats, const GammaSink* sink = nullptr, const DensOut* dens = nullptr) {
    if (precision == FC_PREC_F64)
        return rimp2_grad_f64(d, st, e_os, e_ss, gamma, de_docc, de_dvir, stats, sink, dens);
    if (precision == FC_PREC_MIXED)
        return rimp2_grad_fx(d, st, e_os, e_ss, gamma, de_docc, de_dvir, stats, sink, dens);
    return fail(FC_ERR_KERNEL, "FC_PREC_MIXED_FAST has no adjoint kernel; use FC_PREC_MIXED");
}

}  // namespace

namespace fc {

void shard_pair_range(int64_t nocc, int shard, int nshards, int64_t* lo, int64_t* hi) {
    const int64_t np = nocc * (nocc + 1) / 2;
    *lo = np * shard / nshards;
    *hi = np * (shard + 1) / nshards;
}

std::vector<int> chunk_pair_owner(int64_t nocc, int64_t cc, int nshards) {
    const int64_t nch = (nocc + cc - 1) / cc;
    std::vector<int64_t> w;
    for (int64_t I = 0; I < nch; ++I)
        for (int64_t J = I; J < nch; ++J) {
            const int64_t ni = std::min(cc, nocc - I * cc), nj = std::min(cc, nocc - J * cc);
            w.push_back(I == J ? ni * (ni + 1) / 2 : ni * nj);
        }
    int64_t total = 0;
    for (int64_t x : w) total += x;
    std::vector<int> own(w.size());
    int64_t pre = 0;
    for (size_t x = 0; x < w.size(); ++x) {
        // midpoint 2 pre + w of the chunk pair, on a scale of 2 total
        const int64_t s = (int64_t)nshards * (2 * pre + w[x]) / (2 * total);
        own[x] = (int)std::min<int64_t>(s, nshards - 1);
        pre += w[x];
    }
    return own;
}

static int64_t shard_cap(int64_t nocc, int64_t cc, int nshards) {
    if (nshards <= 1) return cc;
    int64_t n = 1;
    while (n * (n + 1) / 2 < 8 * (int64_t)nshards) ++n;  // chunks for >= 8 chunk pairs per shard
    const int64_t cap = std::max<int64_t>(1, nocc / n);
    return std::min(cc, cap);
}

int64_t grad_chunk_fx(int64_t nocc, int64_t nvir, int64_t budget, int nshards) {
    const int64_t tp = (nvir + 15) / 16 * 16;
    const int64_t per_c2 = tp * tp * (4 + 4 + 3) + 1024 * tp;  // two FP32 amplitude blocks, int8 slices
    int64_t cc = 1;
    while (cc < nocc && (cc + 1) * (cc + 1) * per_c2 <= budget) ++cc;
    return shard_cap(nocc, cc, nshards);
}

int64_t grad_chunk_f64(int64_t nocc, int64_t nvir, int64_t budget, int nshards) {
    int64_t cc = 1;
    while (cc < nocc && 2 * (cc + 1) * nvir * (cc + 1) * nvir * 8 <= budget) ++cc;
    return shard_cap(nocc, cc, nshards);
}

fc_status gamma_sink_block(const GammaSink* sink, const double* gamma, int64_t naux, int64_t nov, int64_t nvir,
                           int64_t r0, int64_t nr, cudaStream_t st) {
    FC_CUDA(cudaEventRecord(sink->ready, st));
    FC_CUDA(cudaStreamWaitEvent(sink->stream, sink->ready, 0));
    FC_CUDA(cudaMemcpy2DAsync(sink->host + r0 * nvir, nov * 8, gamma + r0 * nvir, nov * 8, nr * nvir * 8, naux,
                              cudaMemcpyDeviceToHost, sink->stream));
    return FC_OK;
}

}  // namespace fc

extern "C" {

fc_status fc_rimp2_energy_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                              const double* eps_occ, const double* eps_vir, int32_t has_kappa,
                              double kappa, int32_t precision, double* e_os, double* e_ss,
                              void* stream, fc_stats* stats) {
    FC_TRY(check_shapes(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, has_kappa, kappa, e_os, e_ss));
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    if (naux == 0 || nocc == 0 || nvir == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        return FC_OK;
    }
    Rimp2Dev d{b_ov, eps_occ, eps_vir, naux, nocc, nvir, has_kappa, kappa, chunk_budget()};
    return energy_dispatch(d, precision, pick_stream(stream), e_os, e_ss, stats);
}

fc_status fc_rimp2_energy(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                          const double* eps_occ, const double* eps_vir, int32_t has_kappa,
                          double kappa, int32_t precision, double* e_os, double* e_ss,
                          fc_stats* stats) {
    FC_TRY(check_shapes(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, has_kappa, kappa, e_os, e_ss));
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    if (naux == 0 || nocc == 0 || nvir == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        return FC_OK;
    }
    cudaStream_t st = ctx().stream;
    const size_t nb = (size_t)naux * nocc * nvir * sizeof(double);
    void *db, *de;
    FC_TRY(ws_get(WS_B, nb, &db));
    FC_TRY(ws_get(WS_EPS, (nocc + nvir) * sizeof(double), &de));
    FC_CUDA(cudaMemcpyAsync(db, b_ov, nb, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync(de, eps_occ, nocc * sizeof(double), cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync((double*)de + nocc, eps_vir, nvir * sizeof(double), cudaMemcpyHostToDevice, st));
    Rimp2Dev d{(const double*)db, (const double*)de, (const double*)de + nocc, naux, nocc, nvir,
               has_kappa, kappa, chunk_budget()};
    FC_TRY(energy_dispatch(d, precision, st, e_os, e_ss, stats));
    if (stats) stats->h2d_bytes += nb + (nocc + nvir) * sizeof(double);
    return FC_OK;
}

static fc_status grad_dev_impl(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                               const double* eps_occ, const double* eps_vir, int32_t precision, double* e_os,
                               double* e_ss, double* gamma, double* de_docc, double* de_dvir, double* p_oo,
                               double* p_vv, bool dens, void* stream, fc_stats* stats) {
    FC_TRY(check_shapes(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, 0, 0.0, e_os, e_ss));
    if (naux && nocc && nvir && (!gamma || !de_docc || !de_dvir))
        return fail(FC_ERR_INVALID, "RI-MP2 gradient: null output pointer");
    if (dens && ((nocc && !p_oo) || (nvir && !p_vv)))
        return fail(FC_ERR_INVALID, "RI-MP2 densities: null output pointer");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = pick_stream(stream);
    if (naux == 0 || nocc == 0 || nvir == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        if (gamma && naux * nocc * nvir) FC_CUDA(cudaMemsetAsync(gamma, 0, naux * nocc * nvir * 8, st));
        if (de_docc && nocc) FC_CUDA(cudaMemsetAsync(de_docc, 0, nocc * 8, st));
        if (de_dvir && nvir) FC_CUDA(cudaMemsetAsync(de_dvir, 0, nvir * 8, st));
        if (dens && nocc) FC_CUDA(cudaMemsetAsync(p_oo, 0, nocc * nocc * 8, st));
        if (dens && nvir) FC_CUDA(cudaMemsetAsync(p_vv, 0, nvir * nvir * 8, st));
        FC_CUDA(cudaStreamSynchronize(st));
        return FC_OK;
    }
    Rimp2Dev d{b_ov, eps_occ, eps_vir, naux, nocc, nvir, 0, 0.0, chunk_budget()};
    const DensOut dn{p_oo, p_vv};
    return grad_dispatch(d, precision, st, e_os, e_ss, gamma, de_docc, de_dvir, stats, nullptr,
                         dens ? &dn : nullptr);
}

fc_status fc_rimp2_energy_grad_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                   const double* eps_occ, const double* eps_vir, int32_t precision,
                                   double* e_os, double* e_ss, double* gamma, double* de_docc,
                                   double* de_dvir, void* stream, fc_stats* stats) {
    return grad_dev_impl(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, e_os, e_ss, gamma, de_docc, de_dvir,
                         nullptr, nullptr, false, stream, stats);
}

fc_status fc_rimp2_energy_grad_dens_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                        const double* eps_occ, const double* eps_vir, int32_t precision,
                                        double* e_os, double* e_ss, double* gamma, double* de_docc,
                                        double* de_dvir, double* p_oo, double* p_vv, void* stream,
                                        fc_stats* stats) {
    return grad_dev_impl(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, e_os, e_ss, gamma, de_docc, de_dvir,
                         p_oo, p_vv, true, stream, stats);
}

fc_status fc_rimp2_energy_shard_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                    const double* eps_occ, const double* eps_vir, int32_t has_kappa,
                                    double kappa, int32_t precision, int32_t shard, int32_t nshards,
                                    double* e_os, double* e_ss, void* stream, fc_stats* stats) {
    FC_TRY(check_shapes(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, has_kappa, kappa, e_os, e_ss));
    if (nshards < 1 || shard < 0 || shard >= nshards) return fail(FC_ERR_INVALID, "RI-MP2 shard: bad shard index");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    if (naux == 0 || nocc == 0 || nvir == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        return FC_OK;
    }
    Rimp2Dev d{b_ov, eps_occ, eps_vir, naux, nocc, nvir, has_kappa, kappa, chunk_budget(), shard, nshards};
    return energy_dispatch(d, precision, pick_stream(stream), e_os, e_ss, stats);
}

fc_status fc_rimp2_energy_grad_shard_dev(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                         const double* eps_occ, const double* eps_vir, int32_t precision,
                                         int32_t shard, int32_t nshards, double* e_os, double* e_ss,
                                         double* gamma, double* de_docc, double* de_dvir, void* stream,
                                         fc_stats* stats) {
    if (nshards < 1 || shard < 0 || shard >= nshards) return fail(FC_ERR_INVALID, "RI-MP2 shard: bad shard index");
    if (precision != FC_PREC_F64 && precision != FC_PREC_MIXED)
        return fail(FC_ERR_KERNEL, "RI-MP2 shard: the adjoint runs in FC_PREC_F64 or FC_PREC_MIXED");
    FC_TRY(check_shapes(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, 0, 0.0, e_os, e_ss));
    if (naux && nocc && nvir && (!gamma || !de_docc || !de_dvir))
        return fail(FC_ERR_INVALID, "RI-MP2 gradient: null output pointer");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = pick_stream(stream);
    if (naux == 0 || nocc == 0 || nvir == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        if (gamma && naux * nocc * nvir) FC_CUDA(cudaMemsetAsync(gamma, 0, naux * nocc * nvir * 8, st));
        if (de_docc && nocc) FC_CUDA(cudaMemsetAsync(de_docc, 0, nocc * 8, st));
        if (de_dvir && nvir) FC_CUDA(cudaMemsetAsync(de_dvir, 0, nvir * 8, st));
        FC_CUDA(cudaStreamSynchronize(st));
        return FC_OK;
    }
    Rimp2Dev d{b_ov, eps_occ, eps_vir, naux, nocc, nvir, 0, 0.0, chunk_budget(), shard, nshards};
    return grad_dispatch(d, precision, st, e_os, e_ss, gamma, de_docc, de_dvir, stats);
}

fc_status fc_rimp2_shard_pairs(int64_t nocc, int64_t nvir, int32_t precision, int32_t grad, int32_t shard,
                               int32_t nshards, int32_t* ij, int64_t cap, int64_t* npairs) {
    if (nocc < 0 || nvir < 1 || nshards < 1 || shard < 0 || shard >= nshards || !npairs)
        return fail(FC_ERR_INVALID, "fc_rimp2_shard_pairs: bad arguments");
    if (precision != FC_PREC_F64 && precision != FC_PREC_MIXED && !(precision == FC_PREC_MIXED_FAST && !grad))
        return fail(FC_ERR_INVALID, "fc_rimp2_shard_pairs: bad precision");
    std::vector<std::pair<int32_t, int32_t>> out;
    if (!grad) {
        int64_t lo, hi;
        shard_pair_range(nocc, shard, nshards, &lo, &hi);
        for (int64_t i = 0, k = 0; i < nocc; ++i)
            for (int64_t j = i; j < nocc; ++j, ++k)
                if (k >= lo && k < hi) out.emplace_back((int32_t)i, (int32_t)j);
    } else if (nocc > 0) {
        const int64_t budget = chunk_budget();
        const int64_t cc = precision == FC_PREC_F64 ? grad_chunk_f64(nocc, nvir, budget, nshards)
                                                    : grad_chunk_fx(nocc, nvir, budget, nshards);
        const std::vector<int> own = chunk_pair_owner(nocc, cc, nshards);
        const int64_t nch = (nocc + cc - 1) / cc;
        size_t x = 0;
        for (int64_t I = 0; I < nch; ++I)
            for (int64_t J = I; J < nch; ++J, ++x) {
                if (own[x] != shard) continue;
                for (int64_t i = I * cc; i < std::min(nocc, (I + 1) * cc); ++i)
                    for (int64_t j = (I == J ? i : J * cc); j < std::min(nocc, (J + 1) * cc); ++j)
                        out.emplace_back((int32_t)i, (int32_t)j);
            }
    }
    *npairs = (int64_t)out.size();
    if (ij) {
        if (cap < (int64_t)out.size()) return fail(FC_ERR_LAYOUT, "fc_rimp2_shard_pairs: output too small");
        for (size_t k = 0; k < out.size(); ++k) {
            ij[2 * k] = out[k].first;
            ij[2 * k + 1] = out[k].second;
        }
    }
    return FC_OK;
}

static fc_status grad_host_impl(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                const double* eps_occ, const double* eps_vir, int32_t precision, double* e_os,
                                double* e_ss, double* gamma, double* de_docc, double* de_dvir, double* p_oo,
                                double* p_vv, bool dens, fc_stats* stats) {
    FC_TRY(check_shapes(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, 0, 0.0, e_os, e_ss));
    if (naux && nocc && nvir && (!gamma || !de_docc || !de_dvir))
        return fail(FC_ERR_INVALID, "RI-MP2 gradient: null output pointer");
    if (dens && ((nocc && !p_oo) || (nvir && !p_vv)))
        return fail(FC_ERR_INVALID, "RI-MP2 densities: null output pointer");
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    const size_t nel = (size_t)naux * nocc * nvir;
    if (nel == 0) {
        *e_os = 0.0;
        *e_ss = 0.0;
        for (size_t k = 0; gamma && k < nel; ++k) gamma[k] = 0.0;
        for (int64_t k = 0; de_docc && k < nocc; ++k) de_docc[k] = 0.0;
        for (int64_t k = 0; de_dvir && k < nvir; ++k) de_dvir[k] = 0.0;
        for (int64_t k = 0; dens && k < nocc * nocc; ++k) p_oo[k] = 0.0;
        for (int64_t k = 0; dens && k < nvir * nvir; ++k) p_vv[k] = 0.0;
        return FC_OK;
    }
    cudaStream_t st = ctx().stream;
    void *db, *de, *dg, *dd;
    FC_TRY(ws_get(WS_B, nel * 8, &db));
    FC_TRY(ws_get(WS_EPS, (nocc + nvir) * 8, &de));
    FC_TRY(ws_get(WS_GAMMA, nel * 8, &dg));
    const size_t np2 = dens ? (size_t)(nocc * nocc + nvir * nvir) : 0;  // P_oo, P_vv after dE/deps
    FC_TRY(ws_get(WS_HOSTOUT, ((nocc + nvir) + np2) * 8, &dd));
    Rimp2Dev d{(const double*)db, (const double*)de, (const double*)de + nocc, naux, nocc, nvir,
               0, 0.0, chunk_budget()};
    // A pinned b_ov is uploaded in the gradient's occupied chunks on a copy
    // stream: the mixed driver prepares each chunk once it has arrived, so all
    // but the first chunk's copy overlap the first chunk pairs.  Otherwise one
    // copy on the compute stream.
    cudaPointerAttributes pb{};
    const bool b_pinned = cudaPointerGetAttributes(&pb, b_ov) == cudaSuccess && pb.type == cudaMemoryTypeHost;
    cudaGetLastError();
    cudaStream_t us = nullptr;
    if (b_pinned && precision == FC_PREC_MIXED) {
        std::vector<cudaEvent_t>* evs = nullptr;
        const int64_t cc = grad_chunk_fx(nocc, nvir, d.chunk_bytes, 1);
        const int64_t nch = (nocc + cc - 1) / cc;
        FC_TRY(upload_stream(&us, &evs, (size_t)nch));
        // the upload may start once earlier work on the compute stream is done
        FC_CUDA(cudaEventRecord((*evs)[0], st));
        FC_CUDA(cudaStreamWaitEvent(us, (*evs)[0], 0));
        const int64_t nov = nocc * nvir;
        for (int64_t J = 0; J < nch; ++J) {
            const int64_t o0 = J * cc, no = std::min(cc, nocc - o0);
            FC_CUDA(cudaMemcpy2DAsync((double*)db + o0 * nvir, nov * 8, b_ov + o0 * nvir, nov * 8, no * nvir * 8,
                                      naux, cudaMemcpyHostToDevice, us));
            FC_CUDA(cudaEventRecord((*evs)[J], us));
        }
        d.arrive = evs->data();
        d.arrive_cc = cc;
    } else {
        FC_CUDA(cudaMemcpyAsync(db, b_ov, nel * 8, cudaMemcpyHostToDevice, st));
    }
    FC_CUDA(cudaMemcpyAsync(de, eps_occ, nocc * 8, cudaMemcpyHostToDevice, st));
    FC_CUDA(cudaMemcpyAsync((double*)de + nocc, eps_vir, nvir * 8, cudaMemcpyHostToDevice, st));
    // A pinned Gamma receives its column blocks while the gradient still runs
    // (a pageable one is copied at the end: an async copy from pageable memory
    // would hold the host thread that issues the kernels).
    cudaPointerAttributes pa{};
    const bool pinned = cudaPointerGetAttributes(&pa, gamma) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    Context& c = ctx();
    GammaSink sink{gamma, nullptr, nullptr};
    if (pinned && precision != FC_PREC_MIXED_FAST) {
        FC_TRY(copy_stream(&sink.stream, &sink.ready));
    }
    double* dp = (double*)dd + nocc + nvir;
    const DensOut dn{dp, dp + nocc * nocc};
    const fc_status gs = grad_dispatch(d, precision, st, e_os, e_ss, (double*)dg, (double*)dd, (double*)dd + nocc,
                                       stats, sink.stream ? &sink : nullptr, dens ? &dn : nullptr);
    // the caller may reuse b_ov once this returns, also after an error
    if (us) FC_CUDA(cudaStreamSynchronize(us));
    if (gs != FC_OK) return gs;
    if (!sink.stream) FC_CUDA(cudaMemcpyAsync(gamma, dg, nel * 8, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(de_docc, dd, nocc * 8, cudaMemcpyDeviceToHost, st));
    FC_CUDA(cudaMemcpyAsync(de_dvir, (double*)dd + nocc, nvir * 8, cudaMemcpyDeviceToHost, st));
    if (dens) {
        FC_CUDA(cudaMemcpyAsync(p_oo, dn.p_oo, nocc * nocc * 8, cudaMemcpyDeviceToHost, st));
        FC_CUDA(cudaMemcpyAsync(p_vv, dn.p_vv, nvir * nvir * 8, cudaMemcpyDeviceToHost, st));
    }
    FC_CUDA(cudaStreamSynchronize(st));
    if (sink.stream) FC_CUDA(cudaStreamSynchronize(sink.stream));
    (void)c;
    if (stats) {
        stats->h2d_bytes += nel * 8 + (nocc + nvir) * 8;
        stats->d2h_bytes += nel * 8 + (nocc + nvir + np2) * 8;
    }
    return FC_OK;
}

fc_status fc_rimp2_energy_grad(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                               const double* eps_occ, const double* eps_vir, int32_t precision,
                               double* e_os, double* e_ss, double* gamma, double* de_docc,
                               double* de_dvir, fc_stats* stats) {
    return grad_host_impl(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, e_os, e_ss, gamma, de_docc, de_dvir,
                          nullptr, nullptr, false, stats);
}

fc_status fc_rimp2_energy_grad_dens(const double* b_ov, int64_t naux, int64_t nocc, int64_t nvir,
                                    const double* eps_occ, const double* eps_vir, int32_t precision,
                                    double* e_os, double* e_ss, double* gamma, double* de_docc,
                                    double* de_dvir, double* p_oo, double* p_vv, fc_stats* stats) {
    return grad_host_impl(b_ov, naux, nocc, nvir, eps_occ, eps_vir, precision, e_os, e_ss, gamma, de_docc, de_dvir,
                          p_oo, p_vv, true, stats);
}

}  // extern "C"

namespace {

// Unrestricted RI-MP2 energy components (u_rimp2.rs:693-753): same-spin from
// the closed-shell kernels (E_ss of one spin's B = 2 E_sigma-sigma, the
// pair sum of same_spin_block_energy), opposite-spin from the cross kernels.
fc_status ump2_dispatch(const UmpSpin& a, const UmpSpin& b, int64_t naux, int32_t precision, cudaStream_t st,
                        double* e_aa, double* e_bb, double* e_ab, fc_stats* stats) {
    *e_aa = *e_bb = *e_ab = 0.0;
    if (naux == 0) return FC_OK;
    const UmpSpin* sp[2] = {&a, &b};
    double* out[2] = {e_aa, e_bb};
    for (int k = 0; k < 2; ++k) {
        const UmpSpin& x = *sp[k];
        if (x.nocc < 2 || x.nvir == 0) continue;  // one occupied orbital: no same-spin pair
        Rimp2Dev d{x.b_ov, x.eps_occ, x.eps_vir, naux, x.nocc, x.nvir, 0, 0.0, chunk_budget()};
        double os = 0.0, ss = 0.0;
        fc_stats st1{};
        FC_TRY(energy_dispatch(d, precision, st, &os, &ss, stats ? &st1 : nullptr));
        *out[k] = 0.5 * ss;
        if (stats) {
            stats->main_ms += st1.main_ms;
            stats->main_flops += st1.main_flops;
            stats->main_launches += st1.main_launches;
            stats->launches += st1.launches;
        }
    }
    if (a.nocc && a.nvir && b.nocc && b.nvir) {
        if (precision == FC_PREC_F64) FC_TRY(ump2_cross_f64(a, b, naux, st, e_ab, stats));
        else FC_TRY(ump2_cross_fx(a, b, naux, st, e_ab, stats));
    }
    if (stats) stats->precision = precision == FC_PREC_F64 ? FC_PREC_F64 : FC_PREC_MIXED;
    return FC_OK;
}

fc_status ump2_checks(int64_t naux, int64_t noa, int64_t nva, int64_t nob, int64_t nvb, int32_t precision,
                      const void* ba, const void* bb, const void* e1, const void* e2, const void* e3) {
    if (!e1 || !e2 || !e3) return fail(FC_ERR_INVALID, "U-RI-MP2: null output pointer");
    if (precision != FC_PREC_F64 && precision != FC_PREC_MIXED)
        return fail(FC_ERR_INVALID, "U-RI-MP2: precision is FC_PREC_F64 or FC_PREC_MIXED");
    FC_TRY(check_shapes(ba, naux, noa, nva, ba, ba, FC_PREC_F64, 0, 0.0, e1, e2));
    FC_TRY(check_shapes(bb, naux, nob, nvb, bb, bb, FC_PREC_F64, 0, 0.0, e1, e2));
    return FC_OK;
}

}  // namespace

extern "C" {

fc_status fc_ump2_energy_dev(const double* b_a, int64_t nocc_a, int64_t nvir_a, const double* eps_occ_a,
                             const double* eps_vir_a, const double* b_b, int64_t nocc_b, int64_t nvir_b,
                             const double* eps_occ_b, const double* eps_vir_b, int64_t naux, int32_t precision,
                             double* e_aa, double* e_bb, double* e_ab, void* stream, fc_stats* stats) {
    FC_TRY(ump2_checks(naux, nocc_a, nvir_a, nocc_b, nvir_b, precision, b_a, b_b, e_aa, e_bb, e_ab));
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    UmpSpin a{b_a, eps_occ_a, eps_vir_a, nocc_a, nvir_a}, b{b_b, eps_occ_b, eps_vir_b, nocc_b, nvir_b};
    return ump2_dispatch(a, b, naux, precision, pick_stream(stream), e_aa, e_bb, e_ab, stats);
}

fc_status fc_ump2_energy(const double* b_a, int64_t nocc_a, int64_t nvir_a, const double* eps_occ_a,
                         const double* eps_vir_a, const double* b_b, int64_t nocc_b, int64_t nvir_b,
                         const double* eps_occ_b, const double* eps_vir_b, int64_t naux, int32_t precision,
                         double* e_aa, double* e_bb, double* e_ab, fc_stats* stats) {
    FC_TRY(ump2_checks(naux, nocc_a, nvir_a, nocc_b, nvir_b, precision, b_a, b_b, e_aa, e_bb, e_ab));
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    if (stats) *stats = fc_stats{};
    cudaStream_t st = ctx().stream;
    const size_t na = (size_t)naux * nocc_a * nvir_a * 8, nb = (size_t)naux * nocc_b * nvir_b * 8;
    void *da, *db, *ea, *eb;
    FC_TRY(ws_get(WS_B, na, &da));
    FC_TRY(ws_get(WS_GAMMA, nb, &db));
    FC_TRY(ws_get(WS_EPS, (nocc_a + nvir_a) * 8, &ea));
    FC_TRY(ws_get(WS_HOSTOUT, (nocc_b + nvir_b) * 8, &eb));
    if (na) FC_CUDA(cudaMemcpyAsync(da, b_a, na, cudaMemcpyHostToDevice, st));
    if (nb) FC_CUDA(cudaMemcpyAsync(db, b_b, nb, cudaMemcpyHostToDevice, st));
    if (nocc_a) FC_CUDA(cudaMemcpyAsync(ea, eps_occ_a, nocc_a * 8, cudaMemcpyHostToDevice, st));
    if (nvir_a) FC_CUDA(cudaMemcpyAsync((double*)ea + nocc_a, eps_vir_a, nvir_a * 8, cudaMemcpyHostToDevice, st));
    if (nocc_b) FC_CUDA(cudaMemcpyAsync(eb, eps_occ_b, nocc_b * 8, cudaMemcpyHostToDevice, st));
    if (nvir_b) FC_CUDA(cudaMemcpyAsync((double*)eb + nocc_b, eps_vir_b, nvir_b * 8, cudaMemcpyHostToDevice, st));
    UmpSpin a{(const double*)da, (const double*)ea, (const double*)ea + nocc_a, nocc_a, nvir_a};
    UmpSpin b{(const double*)db, (const double*)eb, (const double*)eb + nocc_b, nocc_b, nvir_b};
    FC_TRY(ump2_dispatch(a, b, naux, precision, st, e_aa, e_bb, e_ab, stats));
    FC_CUDA(cudaStreamSynchronize(st));
    if (stats) stats->h2d_bytes += na + nb + (nocc_a + nvir_a + nocc_b + nvir_b) * 8;
    return FC_OK;
}

}  // extern "C"
