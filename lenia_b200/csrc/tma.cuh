// Tensor-memory-accelerator (TMA) tile loads with an mbarrier, for sm_100a.
//
// A tile is copied from global to shared memory by one thread with
// cp.async.bulk.tensor; the copy signals an mbarrier with its byte count and
// the block waits on the barrier's phase.  Tensor maps are encoded on the host
// (encode_tensor_map) and passed to kernels as __grid_constant__ parameters.
// Loads only (no multicast): a load may start at negative or out-of-range
// coordinates and reads zeros there; its x coordinate must be a multiple of
// 16 bytes (4 floats).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lenia {

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the asynchronous proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later asynchronous-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Waits until the barrier's phase `parity` has completed, at most `limit`
// polls; returns false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned limit)
{
    const uint32_t a = smem_addr(bar);
    for (unsigned i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Poll limit of the wait for a copy still in flight after a block gave up on
// it (the block must not exit while the copy can still write its shared
// memory).
constexpr unsigned kDrainPolls = 1u << 24;

// Block-wide wait for a tile copy: each thread polls at most `polls` times;
// true when every thread saw the phase complete.  Called by every thread of
// the block; the result is the same in all of them.
__device__ __forceinline__ bool block_wait(uint64_t *bar, unsigned parity, unsigned polls)
{
    const bool ok = mbar_wait(bar, parity, polls);
    return __syncthreads_or(!ok) == 0;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_addr(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int x, int y, int z, int w,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(smem_addr(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_addr(bar))
        : "memory");
}

// Asks L2 for a tile (no shared memory, no barrier): a later tma_load_4d of
// the same box then reads L2 instead of DRAM.
__device__ __forceinline__ void tma_prefetch_4d(const CUtensorMap *map, int x, int y, int z, int w)
{
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];\n" ::"l"((uint64_t)map),
                 "r"(x), "r"(y), "r"(z), "r"(w)
                 : "memory");
}

// Host: encodes a tiled float32 tensor map over a dense array of `rank`
// dimensions (dims[0] fastest) with a box of `box` elements per dimension,
// zero fill out of bounds.  Returns cudaErrorInvalidValue when the driver
// rejects the description.
cudaError_t encode_tensor_map(CUtensorMap *map, const float *base, int rank, const unsigned long long *dims,
                              const unsigned *box);

// Host: the same for elements of driver type `dtype` (a CUtensorMapDataType)
// and `elem_bytes` bytes each.
cudaError_t encode_tensor_map_typed(CUtensorMap *map, const void *base, int dtype, int elem_bytes, int rank,
                                    const unsigned long long *dims, const unsigned *box);

// Host: the same with explicit byte strides of dimensions 1..rank-1
// (strides[i] is the stride of dimension i + 1; each a multiple of 16), so
// that dims[0] may be shorter than the row pitch: reads past dims[0] then
// return zero.
cudaError_t encode_tensor_map_strided(CUtensorMap *map, const void *base, int dtype, int rank,
                                      const unsigned long long *dims, const unsigned long long *strides,
                                      const unsigned *box);

}  // namespace lenia
