// Shared-memory ring primitives of the ring-fed H.v kernels: mbarriers, bounded waits and TMA
// bulk copies (cp.async.bulk, no multicast) global -> shared.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace nvb {
namespace ring {

constexpr int WAIT_LIMIT = 1 << 22;  // polls before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// arrive on bar when pred holds (a predicated instruction, no branch)
__device__ __forceinline__ void mbar_arrive_if(uint64_t *bar, bool pred) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.u32 p, %1, 0;\n @p mbarrier.arrive.shared::cta.b64 _, [%0];\n}\n" ::"r"(
            smem_u32(bar)),
        "r"((unsigned)pred)
        : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on a phase; gives up (and raises the abort flag) after `limit` polls, or early
// once another thread raised it.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, volatile int *abort_flag,
                                          int limit = WAIT_LIMIT) {
    for (int i = 0; i < limit; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255) == 255 && *abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// barrier 1 among the consumer warps only (the producer warp never joins it)
__device__ __forceinline__ void consumer_sync(int n) { asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory"); }

}  // namespace ring
}  // namespace nvb
