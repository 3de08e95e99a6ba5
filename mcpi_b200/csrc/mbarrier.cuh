// Shared-memory mbarriers with bounded waits, shared by the warp-specialised
// kernels (the dense pair product in hpsi.cu, the tensor-core Gram in
// density.cu). A wait gives up after a limit in SM cycles and reports it, so
// a stuck pipeline ends its kernel with an error status instead of hanging.
#pragma once
#include <stdint.h>

namespace mcpi {

constexpr long long kWaitCycles = 4000000000LL;   // about two seconds

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}

// true once the phase of the given parity has completed; false after limit cycles
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit)
{
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n"
            ".reg .pred p;\n"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n"
            "}\n"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit) return false;
    }
}


}  // namespace mcpi
