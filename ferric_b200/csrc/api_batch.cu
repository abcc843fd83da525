// Batched RI-MP2 (many molecules of uneven size in one CUDA graph): the C ABI.
//
// The reference computes one molecule per call (ferric-mp2/src/rimp2.rs:
// 1445-1544 for the energy, rimp2.rs:1832-1836 for the adjoint); a batch of
// molecules is a loop over that call.  Here the loop becomes persistent
// kernels over the (molecule, pair, tile) items of all molecules, recorded
// once into a CUDA graph and replayed.
#include <cstdlib>
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
                    "fc_rimp2_batched_create: the batched launch runs the split-BF16 exact-slice kernels "
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
    s = rimp2_batch_build_fx(b, in, group_budget());
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
