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

}  // namespace rmpcd
