// async_copy.cuh -- bulk global->shared copies completed on a shared-memory mbarrier
// (sm_90+ bulk-copy engine), with bounded waits.
//
// One elected thread arms the barrier with the byte count it is about to request and
// issues the copies; the CTA later waits on phase 0.  Every wait gives up after a fixed
// number of polls and reports it, so a copy that never completes cannot hang the kernel:
// the caller records a fault code in a host-mapped word and returns.
#pragma once

#include <cstdint>

namespace osc {

// Fault codes written by kernels to the context's host-mapped fault word.
constexpr unsigned FAULT_BULK_WAIT = 1u;  // a bulk copy did not complete within the poll limit

constexpr unsigned MBAR_POLL_LIMIT = 1u << 22;

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the bulk-copy (async) proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// dst (shared) and src (global) 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Polls phase `parity` of the barrier at most `limit` times (0: MBAR_POLL_LIMIT).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, unsigned limit = 0) {
    if (limit == 0) limit = MBAR_POLL_LIMIT;
    for (unsigned it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void report_fault(unsigned *fault, unsigned code) {
    if (fault) *reinterpret_cast<volatile unsigned *>(fault) = code;
}

}  // namespace osc
