// Asynchronous global -> shared copies (cp.async, sm_80 and later, used here
// on sm_100a).  A gather issued this way does not hold a register or stall
// the issuing warp until cp.async.wait_all, so one thread can keep dozens of
// scattered 4/8-byte reads in flight -- the memory-level parallelism the
// permutation gathers of the cell sort need to run at HBM speed.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rmpcd {

__device__ inline unsigned smem_addr(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ inline void cp_async4(void *smem_dst, const void *gsrc)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(smem_dst)), "l"(gsrc) : "memory");
}

__device__ inline void cp_async8(void *smem_dst, const void *gsrc)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(smem_dst)), "l"(gsrc) : "memory");
}

__device__ inline void cp_async16(void *smem_dst, const void *gsrc)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem_dst)), "l"(gsrc) : "memory");
}

template <typename T>
__device__ inline void cp_async(T *smem_dst, const T *gsrc)
{
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async of 4 or 8 bytes");
    if (sizeof(T) == 4) cp_async4(smem_dst, gsrc);
    else cp_async8(smem_dst, gsrc);
}

__device__ inline void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Bulk copies (cp.async.bulk, the TMA unit's untiled form, sm_90 and later;
// no multicast) completing on a shared-memory mbarrier.  Source, destination
// and size must be multiples of 16 bytes.
__device__ inline void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// one arrival that also announces the bytes the phase's copies will deliver
__device__ inline void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(
                     smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ inline void bulk_copy_to_smem(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ inline bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}

// waits for the phase of the given parity at most `polls` times; false if
// it did not complete
__device__ inline bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, int polls)
{
    for (int i = 0; i < polls; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace rmpcd
