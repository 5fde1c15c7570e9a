// Asynchronous global -> shared copies (cp.async, sm_80+ and sm_100a).  A copy
// with `valid` false writes zero, which is how halo cells that the reference
// never writes (edges and corners) are filled.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lenia {

__device__ __forceinline__ void cp_async_f32(float *smem_dst, const float *gmem_src, bool valid)
{
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem_dst);
    const int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(gmem_src), "r"(n) : "memory");
}

__device__ __forceinline__ void cp_async_f64(void *smem_dst, const void *gmem_src, bool valid)
{
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem_dst);
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(gmem_src), "r"(n) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Bulk prefetch of [p, p + bytes) into L2, issued by one thread; only the
// 16-byte-aligned interior of the range is requested (the bulk copy engine
// wants both the address and the size in whole 16-byte units), so nothing
// outside the range is touched.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes)
{
    const uintptr_t a = ((uintptr_t)p + 15) & ~(uintptr_t)15;
    const uintptr_t b = ((uintptr_t)p + bytes) & ~(uintptr_t)15;
    if (b <= a) return;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a), "r"((uint32_t)(b - a)) : "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace lenia
