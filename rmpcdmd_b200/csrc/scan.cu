#include "scan.cuh"

namespace rmpcd {

__device__ inline int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int w = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += w;
    }
    return v;
}

// Exclusive scan of one value per thread across a block of kScanThreads.
__device__ inline int block_excl_scan(int v, int *total)
{
    __shared__ int warp_tot[kScanThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = warp_incl_scan(v);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int t = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
        int ti = warp_incl_scan(t);
        if (lane < kScanThreads / 32) warp_tot[lane] = ti - t;
        if (lane == 31 && total) *total = ti;
    }
    __syncthreads();
    int r = warp_tot[wid] + inc - v;
    __syncthreads();
    return r;
}

__global__ void k_scan_reduce(const int *__restrict__ in, int n, int *__restrict__ block_tmp)
{
    int base = blockIdx.x * kScanTile + threadIdx.x * kScanPerThread;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPerThread; k++)
        if (base + k < n) s += in[base + k];
    __shared__ int tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) block_tmp[blockIdx.x] = tot;
}

__global__ void k_scan_top(int *block_tmp, int nb)
{
    // each thread scans a run of per = ceil(nb / kScanThreads) block totals
    int per = (nb + kScanThreads - 1) / kScanThreads;
    int b0 = threadIdx.x * per;
    int s = 0;
    for (int k = 0; k < per; k++)
        if (b0 + k < nb) s += block_tmp[b0 + k];
    int off = block_excl_scan(s, nullptr);
    for (int k = 0; k < per; k++) {
        if (b0 + k < nb) {
            int v = block_tmp[b0 + k];
            block_tmp[b0 + k] = off;
            off += v;
        }
    }
}

__global__ void k_scan_apply(int *__restrict__ in, int n, const int *__restrict__ block_tmp,
                             int *__restrict__ out, int *__restrict__ out2, int zero_in)
{
    int base = blockIdx.x * kScanTile + threadIdx.x * kScanPerThread;
    int v[kScanPerThread];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPerThread; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int off = block_excl_scan(s, nullptr) + block_tmp[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanPerThread; k++) {
        if (base + k < n) {
            out[base + k] = off;
            if (out2) out2[base + k] = off;
            if (zero_in) in[base + k] = 0;
        }
        off += v[k];
    }
}

int exclusive_scan(int *in, int *out, int *out2, int n, int *block_tmp, bool zero_in,
                   cudaStream_t s)
{
    if (n <= 0) return RMPCD_OK;
    int nb = scan_blocks_for(n);
    if (nb > 16 * kScanThreads)
        return fail(RMPCD_ERR_CAPACITY, "slot scan: %d slots above the supported maximum", n);
    k_scan_reduce<<<nb, kScanThreads, 0, s>>>(in, n, block_tmp);
    k_scan_top<<<1, kScanThreads, 0, s>>>(block_tmp, nb);
    k_scan_apply<<<nb, kScanThreads, 0, s>>>(in, n, block_tmp, out, out2, zero_in ? 1 : 0);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

}  // namespace rmpcd
