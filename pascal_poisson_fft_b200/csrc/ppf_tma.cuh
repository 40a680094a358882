// ppf_tma.cuh -- tensor-memory-access (TMA) tile and bulk loads into shared
// memory with completion on an mbarrier (sm_100a PTX), and the host-side
// encoding of their tensor maps.  Loads only, never with cluster multicast:
// every source is this GPU's own memory.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ppf {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// make the initialised barriers visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// non-blocking: has the phase with the given parity completed?
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// one poll of the phase with the given parity (the instruction itself may
// suspend the thread for a while before it reports "not yet")
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// one poll that may suspend the thread for up to `ns` nanoseconds while the
// phase is incomplete (it resumes as soon as the phase completes)
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, unsigned parity, unsigned ns)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}
// bounded wait: false if the phase did not complete within `limit` polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long limit)
{
    for (long q = 0; q < limit; ++q)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// bounded wait of polls that sleep up to `ns` each: false after `limit` polls
__device__ __forceinline__ bool mbar_wait_sleep_bounded(uint64_t* bar, unsigned parity, unsigned ns, long limit)
{
    for (long q = 0; q < limit; ++q)
        if (mbar_try_wait_sleep(bar, parity, ns)) return true;
    return false;
}

// L2 eviction priorities for the loads: evict_last for data read again
// soon, evict_first for data read for the last time
__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}

// The 2-D box at element coordinates (x, y) of the map into shared memory
// at dst (128-byte aligned); its bytes complete on bar.  x times the element
// size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar,
                                            uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3}], [%4], %5;\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// `bytes` (a multiple of 16) from global src to shared dst, both 16-byte
// aligned, completing on bar (a bulk copy of consecutive bytes)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Order this CTA's earlier generic-proxy accesses of shared memory before
// the asynchronous proxy's writes that follow (a buffer refilled by TMA).
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda); a map of a row-major 2-D array of FP32 values:
// `inner` values per row, `rows` rows, `row_bytes` apart, boxes of
// box_inner x box_rows values, zero fill outside.  false: not encodable.
bool tma_map_2d_f32(CUtensorMap* map, void* base, unsigned long long inner, unsigned long long rows,
                    unsigned long long row_bytes, unsigned box_inner, unsigned box_rows);

}  // namespace ppf
