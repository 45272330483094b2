// Tensor-memory-accelerator (TMA) tile loads into shared memory, completed on an
// mbarrier, with bounded waits.  No multicast form is used anywhere.
//
// Rules the callers keep: the innermost box coordinate times the element size is
// a multiple of 16 bytes (negative or out-of-range coordinates are allowed and
// read as zeros); the shared-memory destination is 128-byte aligned; one thread
// arms the barrier with the total byte count of the loads it then issues.
//
// Every wait gives up after kWaitCycles SM clocks (about two seconds) and
// reports failure; callers record it in a device flag the host reads and return
// only after waiting (again bounded) for their loads still in flight.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace fpm {
namespace tma {

constexpr long long kWaitCycles = 1ll << 32;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// makes initialised barriers visible to the TMA unit (async proxy)
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders the block's earlier generic-proxy shared-memory accesses (after a block
// barrier) before a following TMA write into the same shared memory
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// 3-D tile load (x innermost) of the box the tensor map describes
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                        uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// 1-D bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from
// global into shared memory, counted on bar (armed by the caller with expect_tx)
__device__ __forceinline__ void load_1d(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Starts bringing `bytes` (a multiple of 16; src 16-byte aligned) from global memory into
// L2 without a destination or completion: a later copy of the same range reads L2.
__device__ __forceinline__ void prefetch_l2(const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity to complete; false after `limit` SM clocks.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          long long limit = kWaitCycles) {
    const long long t0 = clock64();
    while (!mbar_test(bar, parity)) {
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

}  // namespace tma
}  // namespace fpm
