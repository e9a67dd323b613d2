// TMA (cp.async.bulk.tensor) tile loads and mbarrier helpers for sm_100a, local memory only.
//
// Every wait on an mbarrier is bounded: after kWaitLimit polls the waiting thread records
// QPD_DEVERR_TIMEOUT in the context's device status word and gives up, so a load that never
// completes ends the kernel with an error the host can read instead of hanging the GPU.
// No load here uses cluster multicast; every tensor map covers this GPU's own memory.
#pragma once

#include <cuda.h>

#include "qpd_common.cuh"

namespace qpd {

constexpr long long kWaitLimit = 1LL << 24;  // try_wait polls (each may suspend briefly): seconds, not forever
constexpr int QPD_DEVERR_TIMEOUT = 1;
constexpr int QPD_DEVERR_ALIGN = 2;  // dynamic shared memory not 128-byte aligned: no TMA load was issued

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Per-thread asynchronous copy of one BYTES-sized (4, 8 or 16) value from global to shared memory;
// completion is waited for by the issuing thread only (cp.async groups), nothing spins.
template <int BYTES> __device__ __forceinline__ void cp_async(void* dst, const void* src) {
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async copies 4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's committed groups are still in flight.
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make the initialised barriers visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Order this thread's earlier generic-proxy shared-memory accesses before later async-proxy ones.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of bar, at most `limit` polls; false (and the status word set) when it
// gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status, long long limit = kWaitLimit) {
    for (long long it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    if (status) atomicExch(status, QPD_DEVERR_TIMEOUT);
    return false;
}

// 3-D tiled load of the box at (c0, c1, c2) into shared memory, completing on bar.
// c0 is the innermost coordinate; callers keep c0 * element size a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// 1-D bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned), completing on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace qpd
