// Shared-memory addresses, mbarriers with bounded waits and the one-dimensional
// bulk copy global -> shared memory (cp.async.bulk, no multicast), for the
// kernels that stage data asynchronously (harmonic_fast.cu) or wait for the
// tensor cores (fused_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace brp {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Initialises an mbarrier for `count` arrivals and makes the initialisation
// visible to the asynchronous proxy (bulk copies, tensor-core commits).
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrives on the barrier and adds `bytes` to the transaction count its current
// phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Poll bound of a wait that must end before a CTA may leave (its own bulk
// copies or MMAs still write its shared or tensor memory): far above any copy
// or MMA latency (at least ~0.5 s with the back-off below).
constexpr uint32_t kDrainPolls = 1u << 22;

// Waits for the phase of the given parity to complete; gives up (returns
// false) after `polls` polls (0: at once, without polling).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint32_t polls = kDrainPolls) {
    for (uint32_t it = 0; it < polls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (it >= 64) __nanosleep(128);
    }
    return false;
}

// Bulk copy of `bytes` (a multiple of 16) from 16-byte aligned global memory
// to 16-byte aligned shared memory of this CTA; completion is counted on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

}  // namespace brp
