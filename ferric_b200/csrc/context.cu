// Library context: device binding, pool cap, cached workspaces, errors.
// Mirrors the reference's GPU backend state (ferric-core/src/gpu/mod.rs:110-373:
// install/decide/status; ferric-core/src/gpu/pool.rs:1-30: the pool ledger).
#include "fc_internal.cuh"

#include <cstring>

namespace fc {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

fc_status fail(fc_status code, const std::string& msg) {
    set_error(msg);
    return code;
}

fc_status cuda_fail(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                    cudaGetErrorString(e) + ")";
    // A device without an sm_100a image reports "no kernel image".
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction)
        return fail(FC_ERR_KERNEL, m);
    if (e == cudaErrorMemoryAllocation) return fail(FC_ERR_POOL_FULL, m);
    return fail(FC_ERR_CUDA, m);
}

fc_status check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fc_status s = cuda_fail(e, what);
        return s == FC_ERR_CUDA ? fail(FC_ERR_KERNEL, g_last_error) : s;
    }
    return FC_OK;
}

Context& ctx() {
    static Context c;
    return c;
}

fc_status require_init() {
    if (ctx().device < 0) return fail(FC_ERR_INVALID, "libferric_cuda: fc_init was not called");
    FC_CUDA(cudaSetDevice(ctx().device));
    return FC_OK;
}

uint64_t ws_bytes() {
    uint64_t t = 0;
    for (auto& w : ctx().ws) t += w.bytes;
    return t;
}

fc_status pool_reserve(uint64_t bytes) {
    Context& c = ctx();
    if (c.pool_cap && ws_bytes() + c.handle_bytes + bytes > c.pool_cap)
        return fail(FC_ERR_POOL_FULL,
                    "device pool full: need " + std::to_string(bytes) + " B, held " +
                        std::to_string(ws_bytes() + c.handle_bytes) + " B of cap " +
                        std::to_string(c.pool_cap) + " B");
    return FC_OK;
}

fc_status ws_get(int slot, size_t bytes, void** out) {
    Context& c = ctx();
    bytes = (bytes + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    Workspace& w = c.ws[slot];
    if (w.bytes < bytes) {
        uint64_t others = ws_bytes() - w.bytes + c.handle_bytes;
        if (c.pool_cap && others + bytes > c.pool_cap)
            return fail(FC_ERR_POOL_FULL, "device pool full: workspace of " +
                                              std::to_string(bytes) + " B over cap " +
                                              std::to_string(c.pool_cap) + " B");
        if (w.ptr) {
            // The previous user of the slot may still be queued on a stream.
            FC_CUDA(cudaDeviceSynchronize());
            FC_CUDA(cudaFree(w.ptr));
            w.ptr = nullptr;
            w.bytes = 0;
        }
        FC_CUDA(cudaMalloc(&w.ptr, bytes));
        w.bytes = bytes;
    }
    *out = w.ptr;
    return FC_OK;
}

fc_status timing_events(int n, cudaEvent_t** out) {
    Context& c = ctx();
    while ((int)c.evs.size() < 2 * n) {
        cudaEvent_t e;
        FC_CUDA(cudaEventCreate(&e));
        c.evs.push_back(e);
    }
    *out = c.evs.data();
    return FC_OK;
}

fc_status timing_sum(int n, double* ms) {
    Context& c = ctx();
    double t = 0.0;
    if (n > 0) FC_CUDA(cudaEventSynchronize(c.evs[2 * n - 1]));
    for (int k = 0; k < n; ++k) {
        float x = 0.f;
        FC_CUDA(cudaEventElapsedTime(&x, c.evs[2 * k], c.evs[2 * k + 1]));
        t += x;
    }
    *ms = t;
    return FC_OK;
}

fc_status timing_events2(int n, cudaEvent_t** out) {
    Context& c = ctx();
    while ((int)c.evs2.size() < 2 * n) {
        cudaEvent_t e;
        FC_CUDA(cudaEventCreate(&e));
        c.evs2.push_back(e);
    }
    *out = c.evs2.data();
    return FC_OK;
}

fc_status timing_sum2(int n, double* ms) {
    Context& c = ctx();
    double t = 0.0;
    if (n > 0) FC_CUDA(cudaEventSynchronize(c.evs2[2 * n - 1]));
    for (int k = 0; k < n; ++k) {
        float x = 0.f;
        FC_CUDA(cudaEventElapsedTime(&x, c.evs2[2 * k], c.evs2[2 * k + 1]));
        t += x;
    }
    *ms = t;
    return FC_OK;
}

cudaStream_t pick_stream(void* s) { return s ? static_cast<cudaStream_t>(s) : ctx().stream; }

bool mul_ok(int64_t a, int64_t b, int64_t* out) {
    if (a < 0 || b < 0) return false;
    if (a != 0 && b > INT64_MAX / a) return false;
    *out = a * b;
    return true;
}

}  // namespace fc

using namespace fc;

extern "C" {

fc_status fc_init(int32_t device, uint64_t pool_bytes) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return fail(FC_ERR_DRIVER, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    if (device < 0 || device >= n)
        return fail(FC_ERR_DEVICE, "device ordinal " + std::to_string(device) + " not present (" +
                                       std::to_string(n) + " visible)");
    cudaDeviceProp p;
    FC_CUDA(cudaGetDeviceProperties(&p, device));
    if (p.major != 10)
        return fail(FC_ERR_DEVICE, std::string("libferric_cuda is built for sm_100a; device is ") +
                                       p.name + " sm_" + std::to_string(p.major * 10 + p.minor));
    if (c.device == device) {
        c.pool_cap = pool_bytes;
        return FC_OK;
    }
    if (c.device >= 0) return fail(FC_ERR_INVALID, "libferric_cuda is already bound to another device");
    FC_CUDA(cudaSetDevice(device));
    FC_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    FC_CUDA(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
    FC_CUDA(cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming));
    FC_CUDA(cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming));
    FC_CUDA(cudaEventCreate(&c.ev0));
    FC_CUDA(cudaEventCreate(&c.ev1));
    c.sm_count = p.multiProcessorCount;
    c.device = device;
    c.pool_cap = pool_bytes;
    return FC_OK;
}

fc_status fc_release_workspace(void) {
    Context& c = ctx();
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.device < 0) return FC_OK;
    FC_CUDA(cudaSetDevice(c.device));
    FC_CUDA(cudaDeviceSynchronize());
    for (auto& w : c.ws) {
        if (w.ptr) FC_CUDA(cudaFree(w.ptr));
        w.ptr = nullptr;
        w.bytes = 0;
    }
    return FC_OK;
}

uint64_t fc_pool_used(void) { return ws_bytes() + ctx().handle_bytes; }

size_t fc_last_error(char* buf, size_t len) {
    const std::string& m = g_last_error;
    if (buf && len) {
        size_t k = m.size() < len - 1 ? m.size() : len - 1;
        std::memcpy(buf, m.data(), k);
        buf[k] = 0;
    }
    return m.size();
}

const char* fc_version(void) { return "ferric_cuda 0.1.0 (sm_100a)"; }

}  // extern "C"
