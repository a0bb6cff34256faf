#include "scan.cuh"

namespace rmpcd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRows = kScanPerThread / 4;
constexpr int kWarps = kScanThreads / 32;

__device__ inline int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int w = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += w;
    }
    return v;
}

// Sum over the block; every thread gets the result.  Ends with a barrier,
// so part can be reused.
__device__ inline int block_sum(int v, int *part)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = __reduce_add_sync(kFull, v);
    if (lane == 0) part[wid] = v;
    __syncthreads();
    int s = 0;
#pragma unroll
    for (int k = 0; k < kWarps; k++) s += part[k];
    __syncthreads();
    return s;
}

// A tile is kRows rows of int4: row k is elements [k*kScanThreads*4,
// (k+1)*kScanThreads*4), thread t holding elements 4t..4t+3 of every row, so
// each row is one coalesced 16-byte access per thread.
__device__ inline void load_tile(const int *__restrict__ in, long long tile0, int n, bool whole, int4 (&q)[kRows])
{
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        const long long e0 = tile0 + 4LL * (k * kScanThreads + threadIdx.x);
        if (whole) {
            q[k] = reinterpret_cast<const int4 *>(in + e0)[0];
        } else {
            q[k].x = e0 < n ? in[e0] : 0;
            q[k].y = e0 + 1 < n ? in[e0 + 1] : 0;
            q[k].z = e0 + 2 < n ? in[e0 + 2] : 0;
            q[k].w = e0 + 3 < n ? in[e0 + 3] : 0;
        }
    }
}

// Exclusive scan of a tile held as rows: rs[k] is the thread's sum in row k;
// ex[k] receives the tile offset of the thread's first element of row k.
__device__ inline void block_rows_scan(const int (&rs)[kRows], int (&ex)[kRows])
{
    __shared__ int warp_tot[kRows][kWarps];
    __shared__ int row_tot[kRows];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc[kRows];
#pragma unroll
    for (int k = 0; k < kRows; k++) inc[k] = warp_incl_scan(rs[k]);
    if (lane == 31) {
#pragma unroll
        for (int k = 0; k < kRows; k++) warp_tot[k][wid] = inc[k];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < kRows; k++) {
            int w = lane < kWarps ? warp_tot[k][lane] : 0;
            int wi = warp_incl_scan(w);
            if (lane < kWarps) warp_tot[k][lane] = wi - w;
            if (lane == 31) row_tot[k] = wi;
        }
    }
    __syncthreads();
    int base = 0;
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        ex[k] = base + warp_tot[k][wid] + inc[k] - rs[k];
        base += row_tot[k];
    }
}

}  // namespace

// Launch 1: the total of every tile.
__global__ void __launch_bounds__(kScanThreads) k_scan_tile_totals(const int *__restrict__ in, int n,
                                                                   int *__restrict__ tile_total)
{
    __shared__ int s_part[kWarps];
    const long long tile0 = (long long)blockIdx.x * kScanTile;
    int4 q[kRows];
    load_tile(in, tile0, n, tile0 + kScanTile <= n, q);
    int s = 0;
#pragma unroll
    for (int k = 0; k < kRows; k++) s += q[k].x + q[k].y + q[k].z + q[k].w;
    s = block_sum(s, s_part);
    if (threadIdx.x == 0) tile_total[blockIdx.x] = s;
}

// Launch 2: each block adds up the totals of the tiles before it (a few
// loads per thread, from L2) and scans its own tile.
__global__ void __launch_bounds__(kScanThreads)
    k_scan_tiles(const int *__restrict__ in, int n, const int *__restrict__ tile_total, int *__restrict__ out,
                 int *__restrict__ out2, int *__restrict__ clear)
{
    __shared__ int s_part[kWarps];
    const int tile = blockIdx.x;
    int pre = 0;
    for (int j = threadIdx.x; j < tile; j += kScanThreads) pre += tile_total[j];
    const long long tile0 = (long long)tile * kScanTile;
    const bool whole = tile0 + kScanTile <= n;
    int4 q[kRows];
    load_tile(in, tile0, n, whole, q);
    int rs[kRows], ex[kRows];
#pragma unroll
    for (int k = 0; k < kRows; k++) rs[k] = q[k].x + q[k].y + q[k].z + q[k].w;
    const int prefix = block_sum(pre, s_part);
    block_rows_scan(rs, ex);
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        const long long e0 = tile0 + 4LL * (k * kScanThreads + threadIdx.x);
        int4 o;
        o.x = prefix + ex[k];
        o.y = o.x + q[k].x;
        o.z = o.y + q[k].y;
        o.w = o.z + q[k].z;
        if (whole) {
            reinterpret_cast<int4 *>(out + e0)[0] = o;
            if (out2) reinterpret_cast<int4 *>(out2 + e0)[0] = o;
            if (clear) reinterpret_cast<int4 *>(clear + e0)[0] = make_int4(0, 0, 0, 0);
        } else {
            const int ov[4] = {o.x, o.y, o.z, o.w};
            for (int c = 0; c < 4; c++) {
                if (e0 + c < n) {
                    out[e0 + c] = ov[c];
                    if (out2) out2[e0 + c] = ov[c];
                    if (clear) clear[e0 + c] = 0;
                }
            }
        }
    }
}

int exclusive_scan(const int *in, int *out, int *out2, int n, int *tile_total, int *clear, cudaStream_t s)
{
    if (n <= 0) return RMPCD_OK;
    const int nb = scan_blocks_for(n);
    if (nb > kScanMaxTiles)
        return fail(RMPCD_ERR_CAPACITY, "slot scan: %d slots above the supported maximum", n);
    k_scan_tile_totals<<<nb, kScanThreads, 0, s>>>(in, n, tile_total);
    k_scan_tiles<<<nb, kScanThreads, 0, s>>>(in, n, tile_total, out, out2, clear);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

}  // namespace rmpcd
