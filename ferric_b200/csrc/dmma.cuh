// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) building blocks and cp.async
// staging used by the all-FP64 "plain" kernel set.
//
// Fragment layout of mma.m8n8k4.row.col.f64 (PTX ISA, "Matrix fragments for
// mma.m8n8k4 with .f64"): with g = lane / 4 and t = lane % 4, a thread holds
// A[g][t], B[t][g] and C[g][2t], C[g][2t+1].
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace fc {

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile(
        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 8-byte asynchronous copy global -> shared; zero-fills when !valid (no bytes
// are read from src then, but src must still be a mapped address).
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(n));
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(n));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

}  // namespace fc
