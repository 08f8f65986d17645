// Bulk asynchronous copies into shared memory with mbarrier completion, and bounded waits.
// Shared by the SELL SpMV and SpMM kernels.
//
// A copy is issued by one thread: mbar_expect_tx(bar, bytes) arrives on the barrier and adds
// the bytes it waits for, then bulk_g2s copies (global -> this CTA's own shared memory only,
// untiled, no cache-hint operand; both addresses 16-byte aligned, the size a multiple of 16).
// The phase completes when all the bytes have landed; consumers wait on its parity.  Every
// wait is bounded: mbarrier.try_wait with a suspend hint, at most BULK_WAIT_TRIES tries
// (about a second), and the caller decides what to do when it gives up.
#pragma once
#include <cstdint>

namespace pava {

constexpr unsigned BULK_WAIT_HINT_NS = 20000;
constexpr int BULK_WAIT_TRIES = 1 << 16;

__device__ __forceinline__ void mbar_init(unsigned a) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
}
// after the barriers of a CTA are initialised, before any thread uses them
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned a, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
                 : "memory");
}
// the shared memory a copy will overwrite was last read by ordinary loads: order those first
__device__ __forceinline__ void proxy_fence() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes,
                                         unsigned mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}
// true when the phase of the given parity completed; false after BULK_WAIT_TRIES tries
__device__ __forceinline__ bool mbar_wait(unsigned a, unsigned parity) {
    for (int i = 0; i < BULK_WAIT_TRIES; ++i) {
        unsigned ok;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; "
            "selp.u32 %0, 1, 0, p; }"
            : "=r"(ok) : "r"(a), "r"(parity), "r"(BULK_WAIT_HINT_NS) : "memory");
        if (ok) return true;
    }
    return false;
}

}  // namespace pava
