// Batched RI-MP2 (many molecules of uneven size in one CUDA graph): the C ABI.
//
// The reference computes one molecule per call (ferric-mp2/src/rimp2.rs:
// 1445-1544 for the energy, rimp2.rs:1832-1836 for the adjoint); a batch of
// molecules is a loop over that call.  Here the loop becomes persistent
// kernels over the (molecule, pair, tile) items of all molecules, recorded
// once into a CUDA graph and replayed.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "batch.cuh"

namespace fc {

fc_status batch_alloc(fc_rimp2_batch* b, size_t bytes, void** out) {
    bytes = (bytes + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    FC_TRY(pool_reserve(bytes));
    void* p = nullptr;
    FC_CUDA(cudaMalloc(&p, bytes));
    b->allocs.push_back(p);
    b->bytes += bytes;
    ctx().handle_bytes += bytes;
    *out = p;
    return FC_OK;
}

namespace {

void batch_free(fc_rimp2_batch* b) {
    Context& c = ctx();
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void* p : b->allocs) cudaFree(p);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    c.handle_bytes -= b->bytes < c.handle_bytes ? b->bytes : c.handle_bytes;
    delete b;
}

// ------------------------------------------------------------ autotuner --
//
// Per size bucket (gradient or energy, virtual tiles of 128, k-steps of the pair kernel's K tile, 128)
// the one schedule choice that is not fixed by the shapes: diagonal tiles in
// one tensor-core phase with the transpose exchanged in shared memory, or in
// two phases.  Which wins depends on the bucket (the exchange shortens the
// MMA work and lengthens the epilogue), so it is measured: the first batch
// that meets an untuned bucket with FERRIC_CUDA_AUTOTUNE=1 times both
// choices on a trial sub-batch of up to 16 of its molecules (graph replays,
// CUDA events) and keeps the faster.  Decisions live for the process and, with
// FERRIC_CUDA_AUTOTUNE_CACHE=<file>, in a JSON file read at first use and
// rewritten after each new decision.  Without either the built-in default
// (fx_exchange_choice) applies.
struct Tuned {
    int choice;
    double ms0, ms1;
};
std::map<std::string, Tuned> g_tune;
bool g_tune_loaded = false;

std::string bucket_key(int grad, int64_t nt, int64_t nk) {
    return std::string(grad ? "grad" : "energy") + "_t" + std::to_string(nt) + "_k" + std::to_string(nk);
}

void load_tune_cache() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("FERRIC_CUDA_AUTOTUNE_CACHE");
    if (!path || !*path) return;
    std::ifstream f(path);
    if (!f) return;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string t = ss.str();
    // entries: "key": {"exchange": c, "ms_two_phase": a, "ms_exchange": b}
    size_t pos = 0;
    while ((pos = t.find('"', pos)) != std::string::npos) {
        const size_t e = t.find('"', pos + 1);
        if (e == std::string::npos) break;
        const std::string key = t.substr(pos + 1, e - pos - 1);
        pos = e + 1;
        if (key.rfind("grad_", 0) != 0 && key.rfind("energy_", 0) != 0) continue;
        const size_t c = t.find("\"exchange\":", pos);
        const size_t a = t.find("\"ms_two_phase\":", pos);
        const size_t b = t.find("\"ms_exchange\":", pos);
        if (c == std::string::npos || a == std::string::npos || b == std::string::npos) break;
        Tuned v;
        v.choice = std::atoi(t.c_str() + c + 11) != 0;
        v.ms0 = std::atof(t.c_str() + a + 15);
        v.ms1 = std::atof(t.c_str() + b + 14);
        g_tune[key] = v;
        pos = std::max(b, std::max(a, c)) + 1;
    }
}

void save_tune_cache() {
    const char* path = std::getenv("FERRIC_CUDA_AUTOTUNE_CACHE");
    if (!path || !*path) return;
    std::ofstream f(path);
    if (!f) return;
    f << "{\n";
    size_t k = 0;
    for (const auto& kv : g_tune) {
        f << "  \"" << kv.first << "\": {\"exchange\": " << kv.second.choice << ", \"ms_two_phase\": "
          << kv.second.ms0 << ", \"ms_exchange\": " << kv.second.ms1 << "}" << (++k < g_tune.size() ? ",\n" : "\n");
    }
    f << "}\n";
}

bool autotune_on() {
    const char* e = std::getenv("FERRIC_CUDA_AUTOTUNE");
    return e && e[0] == '1';
}

size_t group_budget();

// Device time of one replay of a batch of `sub` with every molecule on `xt`
// (best of 3 after a warm-up replay).
fc_status time_choice(const std::vector<BatchMolIn>& sub, int grad, int xt, double* ms) {
    fc_rimp2_batch* t = new fc_rimp2_batch();
    t->nmol = (int64_t)sub.size();
    t->precision = FC_PREC_MIXED;
    t->grad = grad;
    auto done = [&](fc_status s) {
        batch_free(t);
        return s;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&t->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&t->ev1);
    if (e != cudaSuccess) return done(cuda_fail(e, "autotune: stream/events"));
    void *vo, *vf;
    fc_status s = batch_alloc(t, (size_t)t->nmol * 16, &vo);
    if (s == FC_OK) s = batch_alloc(t, 256, &vf);
    if (s != FC_OK) return done(s);
    t->out = (double*)vo;
    t->flags = (int*)vf;
    std::vector<int> plan(sub.size(), xt);
    s = rimp2_batch_build_fx(t, sub, group_budget(), plan.data());
    if (s != FC_OK) return done(s);
    double best = 1e300;
    for (int r = 0; r < 4; ++r) {
        e = cudaEventRecord(t->ev0, t->stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(t->exec, t->stream);
        if (e == cudaSuccess) e = cudaEventRecord(t->ev1, t->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(t->ev1);
        if (e != cudaSuccess) return done(cuda_fail(e, "autotune: replay"));
        float x = 0.f;
        cudaEventElapsedTime(&x, t->ev0, t->ev1);
        if (r > 0) best = std::min(best, (double)x);
    }
    int hf[2];
    e = cudaMemcpy(hf, t->flags, sizeof(hf), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return done(cuda_fail(e, "autotune: flags"));
    if (hf[0]) return done(fail(FC_ERR_RANGE, "batched RI-MP2: a B_ov has a non-finite element"));
    if (hf[1]) return done(fail(FC_ERR_TIMEOUT, "batched RI-MP2 autotune: a pipeline wait ran out"));
    *ms = best;
    return done(FC_OK);
}

// The exchange choice of every molecule, tuning buckets first met here when
// asked to; b->plan_json records the buckets.
fc_status make_plan(fc_rimp2_batch* b, const std::vector<BatchMolIn>& in, std::vector<int>* plan) {
    load_tune_cache();
    const int grad = b->grad;
    const char* forced = std::getenv("FERRIC_CUDA_XT");
    const bool is_forced = forced && (forced[0] == '0' || forced[0] == '1');
    std::map<std::string, std::vector<int64_t>> members;
    std::vector<std::string> keys(in.size());
    std::vector<int64_t> nks(in.size());
    for (size_t m = 0; m < in.size(); ++m) {
        const int64_t nt = (in[m].nvir + 127) / 128, nk = fx_ksteps(in[m].naux);
        keys[m] = bucket_key(grad, nt, nk);
        nks[m] = nk;
        members[keys[m]].push_back((int64_t)m);
    }
    bool tuned_new = false;
    std::string js = "[";
    for (const auto& kv : members) {
        const std::string& key = kv.first;
        const int64_t nk = nks[kv.second[0]];
        int choice;
        const char* src;
        double ms0 = -1.0, ms1 = -1.0;
        auto it = g_tune.find(key);
        if (is_forced) {
            choice = forced[0] == '1';
            src = "forced";
        } else if (it != g_tune.end()) {
            choice = it->second.choice;
            ms0 = it->second.ms0;
            ms1 = it->second.ms1;
            src = "tuned";
        } else if (autotune_on()) {
            std::vector<BatchMolIn> sub;
            for (size_t q = 0; q < kv.second.size() && q < 16; ++q) sub.push_back(in[kv.second[q]]);
            FC_TRY(time_choice(sub, grad, 0, &ms0));
            FC_TRY(time_choice(sub, grad, 1, &ms1));
            choice = ms1 < ms0 ? 1 : 0;
            g_tune[key] = Tuned{choice, ms0, ms1};
            tuned_new = true;
            src = "tuned";
        } else {
            choice = fx_exchange_choice((int)nk, grad);
            src = "default";
        }
        for (int64_t m : kv.second) (*plan)[m] = choice;
        if (js.size() > 1) js += ", ";
        js += "{\"bucket\": \"" + key + "\", \"molecules\": " + std::to_string(kv.second.size()) +
              ", \"tile_m\": 128, \"tile_n\": 128, \"k_panel\": 64, \"exchange\": " + std::to_string(choice) +
              ", \"source\": \"" + src + "\", \"ms_two_phase\": " + std::to_string(ms0) +
              ", \"ms_exchange\": " + std::to_string(ms1) + "}";
    }
    js += "]";
    b->plan_json = js;
    if (tuned_new) save_tune_cache();
    return FC_OK;
}

size_t group_budget() {
    const char* e = std::getenv("FERRIC_CUDA_BATCH_GROUP_BYTES");
    if (e && *e) {
        const long long v = std::atoll(e);
        if (v > 0) return (size_t)v;
    }
    return (size_t)16 << 30;
}

}  // namespace
}  // namespace fc

using namespace fc;

extern "C" {

fc_status fc_rimp2_batched_create(const fc_mol_desc* mols, int64_t nmol, int32_t precision, fc_rimp2_batch** out) {
    if (!mols || !out || nmol <= 0) return fail(FC_ERR_INVALID, "fc_rimp2_batched_create: null argument or empty batch");
    *out = nullptr;
    if (precision != FC_PREC_MIXED)
        return fail(FC_ERR_KERNEL,
                    "fc_rimp2_batched_create: the batched launch runs the exact integer-slice kernels "
                    "(FC_PREC_MIXED) only; call fc_rimp2_energy_grad_dev per molecule for FP64");
    if (nmol > (1 << 30)) return fail(FC_ERR_LAYOUT, "fc_rimp2_batched_create: too many molecules");
    int with_grad = -1;
    std::vector<BatchMolIn> in((size_t)nmol);
    for (int64_t m = 0; m < nmol; ++m) {
        const fc_mol_desc& d = mols[m];
        const std::string at = " (molecule " + std::to_string(m) + ")";
        if (!d.b_ov || !d.eps_occ || !d.eps_vir) return fail(FC_ERR_INVALID, "fc_rimp2_batched_create: null input" + at);
        if (d.naux <= 0 || d.nocc <= 0 || d.nvir <= 0 || d.nocc > 32767 || d.nvir > (1 << 22) ||
            d.naux > (1 << 24) || d.nocc * d.nvir > (int64_t)1 << 31)
            return fail(FC_ERR_LAYOUT, "fc_rimp2_batched_create: bad shape" + at);
        const int g = (d.gamma && d.de_deps_occ && d.de_deps_vir) ? 1 : 0;
        if (!g && (d.gamma || d.de_deps_occ || d.de_deps_vir))
            return fail(FC_ERR_INVALID, "fc_rimp2_batched_create: gamma, de_deps_occ and de_deps_vir are all set "
                                        "(energy + gradient) or all null (energy)" + at);
        if (with_grad >= 0 && g != with_grad)
            return fail(FC_ERR_INVALID, "fc_rimp2_batched_create: every molecule of a batch asks for the gradient, "
                                        "or none does" + at);
        with_grad = g;
        in[m] = BatchMolIn{d.b_ov, d.eps_occ, d.eps_vir, d.naux, d.nocc, d.nvir, d.gamma, d.de_deps_occ,
                           d.de_deps_vir};
    }
    FC_TRY(require_init());
    std::lock_guard<std::mutex> lk(ctx().mu);
    fc_rimp2_batch* b = new fc_rimp2_batch();
    b->nmol = nmol;
    b->precision = precision;
    b->grad = with_grad;
    auto bail = [&](fc_status s) {
        batch_free(b);
        return s;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) return bail(cuda_fail(e, "fc_rimp2_batched_create: stream/events"));
    void *vout, *vflags;
    fc_status s = batch_alloc(b, (size_t)nmol * 16, &vout);
    if (s == FC_OK) s = batch_alloc(b, 256, &vflags);
    if (s != FC_OK) return bail(s);
    b->out = (double*)vout;
    b->flags = (int*)vflags;
    std::vector<int> plan(in.size(), 0);
    s = make_plan(b, in, &plan);
    if (s != FC_OK) return bail(s);
    s = rimp2_batch_build_fx(b, in, group_budget(), plan.data());
    if (s != FC_OK) return bail(s);
    *out = b;
    return FC_OK;
}

fc_status fc_rimp2_batched_replay(fc_rimp2_batch* b, void* stream) {
    if (!b || !b->exec) return fail(FC_ERR_INVALID, "fc_rimp2_batched_replay: null batch");
    FC_TRY(require_init());
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    FC_CUDA(cudaEventRecord(b->ev0, st));
    FC_CUDA(cudaGraphLaunch(b->exec, st));
    FC_CUDA(cudaEventRecord(b->ev1, st));
    return FC_OK;
}

fc_status fc_rimp2_batched_energies(fc_rimp2_batch* b, double* e_os, double* e_ss) {
    if (!b || !e_os || !e_ss) return fail(FC_ERR_INVALID, "fc_rimp2_batched_energies: null argument");
    FC_TRY(require_init());
    FC_CUDA(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) b->ms = ms;
    std::vector<double> h((size_t)b->nmol * 2);
    int hf[2];
    FC_CUDA(cudaMemcpy(h.data(), b->out, h.size() * 8, cudaMemcpyDeviceToHost));
    FC_CUDA(cudaMemcpy(hf, b->flags, sizeof(hf), cudaMemcpyDeviceToHost));
    if (hf[0]) return fail(FC_ERR_RANGE, "batched RI-MP2: a B_ov has a non-finite element");
    if (hf[1]) return fail(FC_ERR_TIMEOUT, "batched RI-MP2: a pipeline wait ran out");
    for (int64_t m = 0; m < b->nmol; ++m) {
        e_os[m] = h[2 * m];
        e_ss[m] = h[2 * m + 1];
    }
    return FC_OK;
}

fc_status fc_rimp2_batched_info(const fc_rimp2_batch* b, fc_batch_info* info) {
    if (!b || !info) return fail(FC_ERR_INVALID, "fc_rimp2_batched_info: null argument");
    fc_batch_info r{};
    r.nmol = b->nmol;
    r.items = b->items;
    r.gemm_tiles = b->gemm_tiles;
    r.launches = b->launches;
    r.groups = b->groups;
    r.pair_launches = b->pair_launches;
    r.precision = b->precision;
    r.grad = b->grad;
    r.tile_m = 128;
    r.tile_n = 128;
    r.k_panel = 64;
    r.flops = b->flops;
    r.last_ms = b->ms;
    r.bytes = b->bytes;
    *info = r;
    return FC_OK;
}

size_t fc_rimp2_batched_plan(const fc_rimp2_batch* b, char* buf, size_t len) {
    if (!b) return 0;
    const std::string& s = b->plan_json;
    if (buf && len) {
        const size_t n = s.size() < len - 1 ? s.size() : len - 1;
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return s.size();
}

fc_status fc_rimp2_batched_destroy(fc_rimp2_batch* b) {
    if (!b) return FC_OK;
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.device >= 0) cudaSetDevice(c.device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaDeviceSynchronize();
    batch_free(b);
    return FC_OK;
}

fc_status fc_rimp2_batched(const fc_mol_desc* mols, int64_t nmol, int32_t precision, double* e_os,
                           double* e_ss) {
    fc_rimp2_batch* b = nullptr;
    FC_TRY(fc_rimp2_batched_create(mols, nmol, precision, &b));
    fc_status s = fc_rimp2_batched_replay(b, nullptr);
    if (s == FC_OK) s = fc_rimp2_batched_energies(b, e_os, e_ss);
    fc_rimp2_batched_destroy(b);
    return s;
}

}  // extern "C"
