// slc_tma.cuh -- the Tensor Memory Accelerator pieces shared by the staged
// gathers (sl_tma.cu for FP64, sl_mixed.cu for the mixed form): mbarrier
// set-up and bounded waits, and the 3-D tiled bulk tensor load (never with
// cluster multicast: a block loads only into its own shared memory).
#pragma once

#include <cuda.h>

constexpr int kTmaWaitLimit = 1 << 20;  // bounded mbarrier polls

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// Poll phase 0 of the barrier at most kTmaWaitLimit times; false on time-out.
__device__ __forceinline__ bool mbar_wait(unsigned bar)
{
    for (int it = 0; it < kTmaWaitLimit; ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(0u)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap *tm, int c0, int c1, int c2,
                                            unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"((unsigned long long)tm), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

