// One-dimensional bulk copies (TMA, cp.async.bulk) from this GPU's global memory into the issuing
// CTA's shared memory, completed on an mbarrier, for the kernels that stage a per-block tile (a block's
// 512 cell words) while they process the previous one. No multicast: each copy lands in its own CTA.
// Both addresses must be 16-byte aligned and the size a multiple of 16 bytes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sdfb {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // the initialised barrier is visible to the async proxy that completes the copies
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// this thread's arrival on the barrier's current phase, announcing `bytes` of copies to complete it
__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// global -> shared bulk copy of `bytes`, counted on `bar`; prior generic accesses of the destination
// by this thread are ordered before it
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool bar_test(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity; gives up after about two seconds and returns false.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, unsigned parity) {
    if (bar_test(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (bar_test(bar, parity)) return true;
        if (clock64() - t0 > 4000000000ll) return false;
    }
}

}  // namespace sdfb
