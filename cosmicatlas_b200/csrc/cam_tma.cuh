// Tensor-memory-accelerator (TMA) staging for sm_100a: tiled bulk copies
// between global memory and shared memory described by a CUtensorMap, with
// completion tracked on shared-memory mbarriers.
//
// Loads never use cluster multicast: every tensor map here covers this GPU's
// own memory, and each CTA fetches its own tiles.
//
// Every wait on an mbarrier is bounded by the global timer; a wait that runs
// out reports failure instead of spinning on, so a copy that never lands
// cannot hang the GPU (the kernel then sets an error word and returns).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cam {
namespace tma {

// Upper bound of one mbarrier wait, in ns of %globaltimer.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the initialised mbarriers visible to the async proxy (TMA).
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits until the phase of `parity` has completed; false if that took
// longer than kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > kWaitLimitNs) return false;
    return true;
}

// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (TMA) reads of them.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 4D tiled load global -> shared, completing on `bar` (complete_tx bytes).
__device__ __forceinline__ void load_4d(void *smem_dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                        uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// 4D tiled store shared -> global (bulk group of this thread).
__device__ __forceinline__ void store_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3, const void *smem_src)
{
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(smem_src))
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// This thread's bulk stores have finished reading their shared memory.
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// This thread's bulk stores are complete.
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace tma

// Host: a 4D tiled tensor map of FP32 or FP64 scalars (dims[0] innermost,
// strides in bytes of dims 1..3), no swizzle, no interleave.  Returns false
// if the driver entry point is unavailable or refuses the map; callers then
// use their non-TMA kernels.
bool make_tensor_map_4d(CUtensorMap *map, bool fp64, void *base, const uint64_t dims[4], const uint64_t strides[3],
                        const uint32_t box[4]);

}  // namespace cam
