// Internal plumbing of libferric_cuda: status/error handling, the per-device
// context with its workspace pool, and small device helpers shared by the
// kernels (compensated FP64 sums, deterministic block reductions).
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ferric_cuda.h"

namespace fc {

// ---------------------------------------------------------------- errors --

void set_error(const std::string& msg);
fc_status fail(fc_status code, const std::string& msg);
fc_status cuda_fail(cudaError_t e, const char* what);

#define FC_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return ::fc::cuda_fail(e_, #call);       \
    } while (0)

#define FC_TRY(expr)                                                    \
    do {                                                                \
        fc_status s_ = (expr);                                          \
        if (s_ != FC_OK) return s_;                                     \
    } while (0)

// A launch error is reported as FC_ERR_KERNEL (image missing / refused).
fc_status check_launch(const char* what);

// Kernel attributes (cudaFuncSetAttribute) belong to the device that is
// current when they are set: a setter runs once per device, tracked in
// `done` (one bit per device; devices past 63 set them on every call).
inline bool attrs_needed(const std::atomic<uint64_t>& done, uint64_t* bit) {
    int dev = 0;
    *bit = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
    *bit = 1ull << dev;
    return !(done.load() & *bit);
}

// ---------------------------------------------------------- the context --

// One device per process (the reference also binds one ordinal,
// ferric-core/src/gpu/device.rs:50-64).  Workspaces are cached and grown on
// demand; every byte held counts against the pool cap.
struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// Each slot has one owner per call path, so no call frees memory another
// part of the same call still uses.
enum WsSlot {
    WS_B = 0,      // host API: uploaded B_ov, or D/J, C/K staging
    WS_EPS,        // host API: orbital energies
    WS_GAMMA,      // host API: gamma
    WS_HOSTOUT,    // host API: dE/deps outputs
    WS_PAIRS,      // pair tables (+ Q-row scales of the adjoint split)
    WS_PART,       // per-tile partials
    WS_OUT,        // small results and error flags
    WS_T,          // amplitude chunk (FP64 or FP32) + row scales
    WS_TS,         // amplitude chunk slices
    WS_SPLIT,      // integer-slice pair operands
    WS_SPLIT2,     // integer-slice adjoint operand (Q rows)
    WS_SCALE,      // column maxima + operand-row scales
    WS_MISC,       // DF-J weights / d_P, DF-K C^T
    WS_PSCR,       // pair kernel: FP64 X / Y tiles of each CTA
    WS_JD,         // fused DF-JK: d_P and J's pass-2 partials
    WS_DSLAB,      // MP2 densities: amplitude slabs (t and Tt)
    WS_DPART,      // MP2 densities: row scales, partial tiles, work items
    WS_DSTORE,     // MP2 densities: FP32 amplitude blocks kept for a later column chunk
    WS_COUNT
};

struct Context {
    int device = -1;
    uint64_t pool_cap = 0;
    uint64_t handle_bytes = 0;  // held by DF-JK handles
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;   // a call's second stream (work that overlaps its main stream)
    cudaEvent_t fork = nullptr, join = nullptr;
    int sm_count = 0;
    std::mutex mu;
    Workspace ws[WS_COUNT];
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> evs;   // per-launch timing pairs of the dominant kernel
    std::vector<cudaEvent_t> evs2;  // per-launch timing pairs of the second kernel
};

Context& ctx();
fc_status require_init();
uint64_t ws_bytes();
// Workspace slot `slot` with at least `bytes` (16-byte rounded); refuses with
// FC_ERR_POOL_FULL before allocating when the cap would be exceeded.
fc_status ws_get(int slot, size_t bytes, void** out);
fc_status pool_reserve(uint64_t bytes);  // handle allocation check
cudaStream_t pick_stream(void* s);
// At least 2*n timing events (created on first use, kept by the context).
fc_status timing_events(int n, cudaEvent_t** out);
// Sum of elapsed times of the n event pairs (waits for the last one).
fc_status timing_sum(int n, double* ms);
// The same pool for a call's second timed kernel.
fc_status timing_events2(int n, cudaEvent_t** out);
fc_status timing_sum2(int n, double* ms);

// Overflow-checked size products.
bool mul_ok(int64_t a, int64_t b, int64_t* out);

// ------------------------------------------------------- device helpers --

// Neumaier compensated accumulator (sum + running correction).
struct KSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

__device__ __forceinline__ double warp_sum(double v) {
    // Fixed butterfly order: identical bits run to run.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum of one double per thread (blockDim.x multiple of
// 32, <= 1024).  Every thread gets the result.
__device__ __forceinline__ double block_sum(double v, double* sh /* >= 32 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (warp == 0) {
        t = lane < nw ? sh[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) sh[0] = t;
    }
    __syncthreads();
    t = sh[0];
    __syncthreads();
    return t;
}

}  // namespace fc
