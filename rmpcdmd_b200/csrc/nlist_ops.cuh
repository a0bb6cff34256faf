// Neighbor-list and Lennard-Jones bodies (src/neighbor_list.f90,
// src/interaction.f90) shared by the single-system kernels and the batched
// replica engine.
#pragma once

#include <cstring>

#include "async_copy.cuh"
#include "keys.cuh"
#include "rmpcd_common.cuh"
#include "state.cuh"

namespace rmpcd {

constexpr int kNlBlockThreads = 256;


struct LJDev {
    int n1;
    double epsilon[16], sigma[16], cut_sq[16], cut_energy[16];
};

inline LJDev lj_dev(const rmpcd_lj *lj)
{
    LJDev d;
    memset(&d, 0, sizeof(d));
    if (!lj) return d;
    d.n1 = lj->n1;
    for (int i = 0; i < 16; i++) {
        d.epsilon[i] = lj->epsilon[i];
        d.sigma[i] = lj->sigma[i];
        d.cut_sq[i] = lj->cut_sq[i];
        d.cut_energy[i] = lj->cut_energy[i];
    }
    return d;
}

// x**3 = x*(x*x), x**6 = x**3 * x**3 (gfortran's constant-power expansion)
__device__ inline double cube(double x) { return x * (x * x); }
__device__ inline double sixth(double x)
{
    double c = cube(x);
    return c * c;
}

// lj_force / lj_energy, src/interaction.f90:83-96,126-136
__device__ inline double lj_force_over_r(double r_sq, double eps, double sigma)
{
    double s6 = sixth(sigma) / cube(r_sq);
    return 24.0 * eps * s6 / r_sq * (2.0 * s6 - 1.0);
}
__device__ inline double lj_energy(double r_sq, double eps, double sigma, double ce)
{
    double s6 = sixth(sigma) / cube(r_sq);
    return 4.0 * eps * (s6 * s6 - s6) - ce;
}

__device__ inline int imod(int a, int p)
{
    int r = a % p;
    return (r != 0 && ((r < 0) != (p < 0))) ? r + p : r;
}

// Staging of a chunk's candidate cells in shared memory by bulk copies: per
// cell its particle range of x, y, z and species, rounded outward to
// multiples of 4 elements so that every copy starts and ends on a 16-byte
// boundary (the particle arrays are allocated to a multiple of 4 elements).
// kNlStageCap elements per array; a chunk with more stays on direct loads.
constexpr int kNlStageCap = 4096;
constexpr int kNlStagePolls = 1 << 16;

template <typename R>
constexpr size_t nl_stage_bytes()
{
    return (size_t)kNlStageCap * (3 * sizeof(R) + sizeof(int));
}

struct NlStage {
    unsigned char *buf;       // nl_stage_bytes<R>() of dynamic shared memory; null = direct loads
    unsigned long long *bar;  // mbarrier in shared memory
};

// exclusive scan of one int per thread over a block of kNlBlockThreads;
// *total gets the sum (shared, read after the call)
__device__ inline int nl_block_excl_scan(int v, int *warp_sum, int *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        int w = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += w;
    }
    if (lane == 31) warp_sum[wid] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < kNlBlockThreads / 32; w++) {
            int x = warp_sum[w];
            warp_sum[w] = acc;
            acc += x;
        }
        *total = acc;
    }
    __syncthreads();
    int r = warp_sum[wid] + inc - v;
    __syncthreads();
    return r;
}

// update_list, src/neighbor_list.f90:76-157: one block per colloid; stencil
// cells are processed in chunks of kNlBlockThreads, their particles enumerated in
// stencil order and compacted in order with a block scan.  With a stage,
// each chunk's cells are first brought into shared memory by bulk copies.
template <typename R>
__device__ inline void update_list_block(int i, const Grid &g, const double *cx, const double *cy, const double *cz,
                                         const int *cs, const R *sx, const R *sy, const R *sz, const int *sspec,
                                         const int *count, const int *start, const int *stencil, int n_stencil,
                                         double radiussq, const LJDev &lj, int do_lj, int Nmax, int *list,
                                         int *n_out, unsigned char *is_md, unsigned char *is_reac, unsigned *err,
                                         NlStage stage = {nullptr, nullptr})
{
    __shared__ int c_slot[kNlBlockThreads], c_start[kNlBlockThreads], c_off[kNlBlockThreads + 1];
    __shared__ int c_md[kNlBlockThreads], c_noreac[kNlBlockThreads], c_shift[kNlBlockThreads];
    __shared__ int warp_sum[kNlBlockThreads / 32];
    __shared__ int s_total, s_base, s_wtotal;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    R *st_x = nullptr, *st_y = nullptr, *st_z = nullptr;
    int *st_s = nullptr;
    bool use_stage = stage.buf != nullptr;
    unsigned phase = 0;
    bool pending = false;  // a copy phase that was given up on
    if (use_stage) {
        st_x = (R *)stage.buf;
        st_y = st_x + kNlStageCap;
        st_z = st_y + kNlStageCap;
        st_s = (int *)(st_z + kNlStageCap);
        if (t == 0) mbar_init(stage.bar, 1);
    }
    double x0 = cx[i], x1 = cy[i], x2 = cz[i];
    int si = cs[i];
    int cell[3];
    cell_coords(g, x0, x1, x2, cell);  // cartesian_indices (0-based)
    double L0 = g.L[0] * g.a, L1 = g.L[1] * g.a, L2 = g.L[2] * g.a;
    if (t == 0) s_base = 0;
    __syncthreads();
    for (int j0 = 0; j0 < n_stencil; j0 += kNlBlockThreads) {
        int j = j0 + t;
        int cnt = 0;
        if (j < n_stencil) {
            int p[3] = {imod(cell[0] + stencil[3 * j], g.L[0]), imod(cell[1] + stencil[3 * j + 1], g.L[1]),
                        imod(cell[2] + stencil[3 * j + 2], g.L[2])};
            int s = slot_of_cell(g, p);
            c_slot[t] = s;
            c_start[t] = start[s];
            cnt = count[s];
        }
        c_md[t] = 0;
        c_noreac[t] = 0;
        // exclusive scan of the candidate counts of this chunk
        int inc = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            int w = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += w;
        }
        if (lane == 31) warp_sum[wid] = inc;
        __syncthreads();
        if (t == 0) {
            int acc = 0;
            for (int w = 0; w < kNlBlockThreads / 32; w++) {
                int v = warp_sum[w];
                warp_sum[w] = acc;
                acc += v;
            }
            s_total = acc;
        }
        __syncthreads();
        c_off[t] = warp_sum[wid] + inc - cnt;
        if (t == 0) c_off[kNlBlockThreads] = s_total;
        __syncthreads();
        const int total = c_off[kNlBlockThreads];
        bool staged = false;
        if (use_stage) {
            // window of this thread's cell: [w0, w0 + wl), w0 and wl multiples of 4
            int w0 = 0, wl = 0;
            if (cnt > 0) {
                w0 = c_start[t] & ~3;
                wl = (c_start[t] - w0 + cnt + 3) & ~3;
            }
            const int woff = nl_block_excl_scan(wl, warp_sum, &s_wtotal);
            const int wtot = s_wtotal;
            if (wtot > 0 && wtot <= kNlStageCap) {
                if (t == 0) mbar_arrive_expect_tx(stage.bar, (unsigned)(wtot * (3 * sizeof(R) + sizeof(int))));
                if (wl > 0) {
                    bulk_copy_to_smem(st_x + woff, sx + w0, (unsigned)(wl * sizeof(R)), stage.bar);
                    bulk_copy_to_smem(st_y + woff, sy + w0, (unsigned)(wl * sizeof(R)), stage.bar);
                    bulk_copy_to_smem(st_z + woff, sz + w0, (unsigned)(wl * sizeof(R)), stage.bar);
                    bulk_copy_to_smem(st_s + woff, sspec + w0, (unsigned)(wl * sizeof(int)), stage.bar);
                }
                c_shift[t] = woff - w0;
                const bool ok = mbar_wait_bounded(stage.bar, phase, kNlStagePolls);
                phase ^= 1u;
                if (__syncthreads_or(!ok)) {
                    // not delivered in time: report it and keep to direct loads
                    if (t == 0) atomicOr(err, DEV_ERR_BULK_WAIT);
                    use_stage = false;
                    pending = true;
                } else {
                    staged = true;
                }
            }
        }
        for (int k0 = 0; k0 < total; k0 += kNlBlockThreads) {
            int k = k0 + t;
            int accept = 0;
            int idx = -1;
            if (k < total) {
                // stencil cell of candidate k: last cell with offset <= k
                int lo = 0, hi = kNlBlockThreads;
                while (hi - lo > 1) {
                    int mid = (lo + hi) >> 1;
                    if (c_off[mid] <= k) lo = mid;
                    else hi = mid;
                }
                const int cl = lo;
                idx = c_start[cl] + (k - c_off[cl]);
                const int q = staged ? idx + c_shift[cl] : 0;
                int s = staged ? st_s[q] : sspec[idx];
                if (s > 0) {
                    const R px = staged ? st_x[q] : sx[idx];
                    const R py = staged ? st_y[q] : sy[idx];
                    const R pz = staged ? st_z[q] : sz[idx];
                    double r0 = min_image_d(x0 - (double)px, L0);
                    double r1 = min_image_d(x1 - (double)py, L1);
                    double r2 = min_image_d(x2 - (double)pz, L2);
                    double rsq = r0 * r0 + r1 * r1 + r2 * r2;
                    if (rsq < radiussq) {
                        accept = 1;
                        c_md[cl] = 1;
                        if (do_lj && rsq <= lj.cut_sq[(s - 1) + lj.n1 * (si - 1)]) c_noreac[cl] = 1;
                    }
                }
            }
            // ordered compaction of accepted candidates
            unsigned bal = __ballot_sync(0xffffffffu, accept);
            if (lane == 0) warp_sum[wid] = __popc(bal);
            __syncthreads();
            if (t == 0) {
                int acc = 0;
                for (int w = 0; w < kNlBlockThreads / 32; w++) {
                    int v = warp_sum[w];
                    warp_sum[w] = acc;
                    acc += v;
                }
                s_total = acc;
            }
            __syncthreads();
            if (accept) {
                int pos = s_base + warp_sum[wid] + __popc(bal & ((1u << lane) - 1u));
                if (pos < Nmax) list[(size_t)i * Nmax + pos] = idx;
                else atomicOr(err, DEV_ERR_NLIST_FULL);
            }
            __syncthreads();
            if (t == 0) s_base += s_total;
            __syncthreads();
        }
        __syncthreads();
        if (j < n_stencil && c_md[t]) {
            is_md[c_slot[t]] = 1;
            if (c_noreac[t]) is_reac[c_slot[t]] = 0;
        }
        __syncthreads();
    }
    if (t == 0) n_out[i] = s_base < Nmax ? s_base : Nmax;
    // a copy phase given up on is waited for again, bounded, before the block's
    // shared memory is released; if it has not landed within that second
    // limit either, the block exits with it pending and sets its own error bit
    if (pending && !mbar_wait_bounded(stage.bar, phase ^ 1u, kNlStagePolls)) atomicOr(err, DEV_ERR_BULK_UNDRAINED);
}


// pair force of list entry q (src/neighbor_list.f90:198-219): colloid at x
// of species s1 and the entry's solvent particle
template <typename R>
__device__ inline void pair_force_entry(size_t q, const double x[3], int s1, const R *sx, const R *sy, const R *sz,
                                        const int *sspec, int *sflags, const int *list, double L0, double L1,
                                        double L2, const LJDev &lj, double *pf, double *pe, unsigned char *contrib,
                                        int *ncontrib, int *max_contrib)
{
    const int mask = (1 << MD_BIT) | (s1 == 1 ? (1 << CATALYZED_BIT) : 0);
    int idx = list[q];
    int s2 = sspec[idx];
    unsigned char c = 0;
    if (s2 > 0) {
        double d0 = min_image_d(x[0] - (double)sx[idx], L0);
        double d1 = min_image_d(x[1] - (double)sy[idx], L1);
        double d2 = min_image_d(x[2] - (double)sz[idx], L2);
        double r_sq = d0 * d0 + d1 * d1 + d2 * d2;
        int tt = (s2 - 1) + lj.n1 * (s1 - 1);
        if (r_sq <= lj.cut_sq[tt]) {
            double fr = lj_force_over_r(r_sq, lj.epsilon[tt], lj.sigma[tt]);
            pf[3 * q] = fr * d0;
            pf[3 * q + 1] = fr * d1;
            pf[3 * q + 2] = fr * d2;
            pe[q] = lj_energy(r_sq, lj.epsilon[tt], lj.sigma[tt], lj.cut_energy[tt]);
            c = 1;
            int prev = atomicAdd(ncontrib + idx, 1);
            if (prev >= 1) atomicMax(max_contrib, prev + 1);
            atomicOr(sflags + idx, mask);
        }
    }
    contrib[q] = c;
}

// solvent force - f of entry q when its particle has exactly one contribution
template <typename R>
__device__ inline void apply_single_entry(size_t q, const int *list, const unsigned char *contrib, const double *pf,
                                          const int *ncontrib, R *fx, R *fy, R *fz)
{
    if (!contrib[q]) return;
    int idx = list[q];
    if (ncontrib[idx] != 1) return;
    fx[idx] = fx[idx] - (R)pf[3 * q];
    fy[idx] = fy[idx] - (R)pf[3 * q + 1];
    fz[idx] = fz[idx] - (R)pf[3 * q + 2];
}

// Particles with several contributions must receive their subtractions in
// the reference's (colloid, entry) order.  The single-contribution pass
// collects them as 64-bit keys (particle << 32 | entry index q, with
// q = colloid * Nmax + entry increasing in that order); one block sorts the
// keys and applies each particle's run in order.  Larger lists than the block
// sorts take the colloid-by-colloid loop (apply_multi_block).
constexpr int kMultiSortMax = 4096;

template <typename R>
__device__ inline void apply_single_or_collect(size_t q, const int *list, const unsigned char *contrib,
                                               const double *pf, const int *ncontrib, R *fx, R *fy, R *fz,
                                               unsigned long long *mkeys, int *m_count)
{
    if (!contrib[q]) return;
    const int idx = list[q];
    const int nc = ncontrib[idx];
    if (nc == 1) {
        fx[idx] = fx[idx] - (R)pf[3 * q];
        fy[idx] = fy[idx] - (R)pf[3 * q + 1];
        fz[idx] = fz[idx] - (R)pf[3 * q + 2];
    } else if (nc > 1) {
        const int k = atomicAdd(m_count, 1);
        if (k < kMultiSortMax) mkeys[k] = ((unsigned long long)(unsigned)idx << 32) | (unsigned long long)q;
    }
}

// one block: sort the collected keys and apply each particle's contributions
// in (colloid, entry) order; returns false (nothing applied) when more keys
// were collected than the block sorts
template <typename R>
__device__ inline bool apply_multi_sorted_block(const unsigned long long *mkeys, int m, const double *pf, R *fx,
                                                R *fy, R *fz)
{
    __shared__ unsigned long long sk[kMultiSortMax];
    if (m > kMultiSortMax) return false;
    int n2 = 1;
    while (n2 < m) n2 <<= 1;
    for (int k = threadIdx.x; k < n2; k += blockDim.x) sk[k] = k < m ? mkeys[k] : ~0ull;
    __syncthreads();
    // bitonic sort of n2 keys (all distinct: q is unique)
    for (int size = 2; size <= n2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = threadIdx.x; k < n2; k += blockDim.x) {
                const int o = k ^ stride;
                if (o > k) {
                    const bool up = (k & size) == 0;
                    const unsigned long long a = sk[k], b = sk[o];
                    if ((a > b) == up) {
                        sk[k] = b;
                        sk[o] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const unsigned idx = (unsigned)(sk[k] >> 32);
        if (k > 0 && (unsigned)(sk[k - 1] >> 32) == idx) continue;
        for (int j = k; j < m && (unsigned)(sk[j] >> 32) == idx; j++) {
            const size_t q = (size_t)(sk[j] & 0xffffffffull);
            fx[idx] = fx[idx] - (R)pf[3 * q];
            fy[idx] = fy[idx] - (R)pf[3 * q + 1];
            fz[idx] = fz[idx] - (R)pf[3 * q + 2];
        }
    }
    __syncthreads();
    return true;
}

// particles with several contributions: colloid by colloid in order; inside
// one colloid's list entries are distinct unless the stencil wraps the box,
// in which case a single thread applies everything in order (one block)
template <typename R>
__device__ inline void apply_multi_block(const int *list, const int *n, int C, int Nmax, const unsigned char *contrib,
                                         const double *pf, const int *ncontrib, int serial, R *fx, R *fy, R *fz)
{
    for (int i = 0; i < C; i++) {
        const int ni = n[i];
        if (serial) {
            if (threadIdx.x == 0) {
                for (int e = 0; e < ni; e++) {
                    size_t q = (size_t)i * Nmax + e;
                    if (!contrib[q]) continue;
                    int idx = list[q];
                    if (ncontrib[idx] < 2) continue;
                    fx[idx] = fx[idx] - (R)pf[3 * q];
                    fy[idx] = fy[idx] - (R)pf[3 * q + 1];
                    fz[idx] = fz[idx] - (R)pf[3 * q + 2];
                }
            }
        } else {
            for (int e = threadIdx.x; e < ni; e += blockDim.x) {
                size_t q = (size_t)i * Nmax + e;
                if (!contrib[q]) continue;
                int idx = list[q];
                if (ncontrib[idx] < 2) continue;
                fx[idx] = fx[idx] - (R)pf[3 * q];
                fy[idx] = fy[idx] - (R)pf[3 * q + 1];
                fz[idx] = fz[idx] - (R)pf[3 * q + 2];
            }
        }
        __syncthreads();
    }
}

// f1 = sum of colloid i's pair forces in list order; force(:,i) += f1; the
// contributing entries are compacted in order into clist (one block).  The
// list is walked in chunks of kCollSumPer entries per thread, each thread owning
// a contiguous run of its chunk: the chunk's contributing entries are
// compacted in order and staged in shared memory by the whole block, then
// the three components are summed by three threads, each in list order, so
// every sum is the sequential one.  Every thread loads its run of the next
// chunk before the current chunk is summed, so those loads are in flight
// while the three threads add.
constexpr int kCollSumPer = 4;
constexpr int kCollSumChunk = kCollSumPer * kNlBlockThreads;

__device__ inline void colloid_sum_load(int i, int e_first, int ni, int Nmax, const unsigned char *contrib,
                                        const double *pf, unsigned &cmask, double (&f)[kCollSumPer][3])
{
    cmask = 0u;
#pragma unroll
    for (int m = 0; m < kCollSumPer; m++) {
        const int e = e_first + m;
        if (e < ni) {
            const size_t q = (size_t)i * Nmax + e;
            if (contrib[q]) {
                cmask |= 1u << m;
                f[m][0] = pf[3 * q];
                f[m][1] = pf[3 * q + 1];
                f[m][2] = pf[3 * q + 2];
            }
        }
    }
}

// (kSum = false: the compaction into clist / cn alone, the force untouched)
template <bool kSum = true>
__device__ inline void colloid_sum_block(int i, const int *n, int Nmax, const unsigned char *contrib, const double *pf,
                                         double *cfx, double *cfy, double *cfz, int *clist, int *cn)
{
    __shared__ int idxs[kCollSumChunk];
    __shared__ double vals[3][kCollSumChunk];
    __shared__ int warp_sum[kNlBlockThreads / 32];
    __shared__ int s_cnt;
    const int t = threadIdx.x;
    const int ni = n[i];
    double acc = 0;  // thread c < 3 accumulates component c
    int total = 0;
    // this thread's run of the current chunk: contributing entries and forces
    unsigned cmask;
    double f[kCollSumPer][3];
    colloid_sum_load(i, kCollSumPer * t, ni, Nmax, contrib, pf, cmask, f);
    for (int e0 = 0; e0 < ni; e0 += kCollSumChunk) {
        const int e_first = e0 + kCollSumPer * t;
        int k = nl_block_excl_scan(__popc(cmask), warp_sum, &s_cnt);
#pragma unroll
        for (int m = 0; m < kCollSumPer; m++) {
            if ((cmask >> m) & 1u) {
                idxs[k] = e_first + m;
                vals[0][k] = f[m][0];
                vals[1][k] = f[m][1];
                vals[2][k] = f[m][2];
                k++;
            }
        }
        __syncthreads();
        const int cnt = s_cnt;
        // the next chunk's run
        colloid_sum_load(i, e_first + kCollSumChunk, ni, Nmax, contrib, pf, cmask, f);
        if (kSum && t < 3) {
#pragma unroll 8
            for (int q = 0; q < cnt; q++) acc = acc + vals[t][q];
        }
        for (int q = t; q < cnt; q += kNlBlockThreads) clist[(size_t)i * Nmax + total + q] = idxs[q];
        total += cnt;
        __syncthreads();
    }
    if (t == 0) cn[i] = total;
    if (!kSum) return;
    if (t == 0) {
        cfx[i] = cfx[i] + acc;
    } else if (t == 1) {
        cfy[i] = cfy[i] + acc;
    } else if (t == 2) {
        cfz[i] = cfz[i] + acc;
    }
}

// The FP32 form's colloid force sum: f1 = the sum of colloid i's pair forces
// in FP64 by a fixed tree, force(:,i) += f1 (one block of kNlBlockThreads).
// Thread t adds the contributing entries t, t + T, t + 2T, ... (T threads) in
// that order; the threads' sums are combined by xor butterflies inside each
// warp, then the warps' sums by one more butterfly over warp numbers.  The
// order depends on the list alone, not on the grid, so every launch shape
// gives the same bits; it is not list order, which only the FP64 form keeps.
constexpr int kCollTreePer = 4;

__device__ inline void colloid_tree_block(int i, const int *n, int Nmax, const unsigned char *contrib,
                                          const double *pf, double *cfx, double *cfy, double *cfz)
{
    __shared__ double wsum[3][kNlBlockThreads / 32];
    const int ni = n[i];
    const size_t base = (size_t)i * Nmax;
    double a0 = 0, a1 = 0, a2 = 0;
    for (int e0 = threadIdx.x; e0 < ni; e0 += kCollTreePer * kNlBlockThreads) {
        double f[kCollTreePer][3];
        bool c[kCollTreePer];
#pragma unroll
        for (int u = 0; u < kCollTreePer; u++) {
            const int e = e0 + u * kNlBlockThreads;
            c[u] = e < ni && contrib[base + e];
            if (c[u]) {
                const size_t q = base + e;
                f[u][0] = pf[3 * q];
                f[u][1] = pf[3 * q + 1];
                f[u][2] = pf[3 * q + 2];
            }
        }
#pragma unroll
        for (int u = 0; u < kCollTreePer; u++)
            if (c[u]) {
                a0 = a0 + f[u][0];
                a1 = a1 + f[u][1];
                a2 = a2 + f[u][2];
            }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 = a0 + __shfl_xor_sync(0xffffffffu, a0, o);
        a1 = a1 + __shfl_xor_sync(0xffffffffu, a1, o);
        a2 = a2 + __shfl_xor_sync(0xffffffffu, a2, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        wsum[0][w] = a0;
        wsum[1][w] = a1;
        wsum[2][w] = a2;
    }
    __syncthreads();
    if (w == 0) {
        constexpr int NW = kNlBlockThreads / 32;
        double b0 = lane < NW ? wsum[0][lane] : 0.0, b1 = lane < NW ? wsum[1][lane] : 0.0,
               b2 = lane < NW ? wsum[2][lane] : 0.0;
#pragma unroll
        for (int o = NW / 2; o > 0; o >>= 1) {
            b0 = b0 + __shfl_xor_sync(0xffffffffu, b0, o);
            b1 = b1 + __shfl_xor_sync(0xffffffffu, b1, o);
            b2 = b2 + __shfl_xor_sync(0xffffffffu, b2, o);
        }
        if (lane == 0) {
            cfx[i] = cfx[i] + b0;
            cfy[i] = cfy[i] + b1;
            cfz[i] = cfz[i] + b2;
        }
    }
    // wsum is free again only once warp 0 has read it (a block may go on to
    // another colloid)
    __syncthreads();
}

// compute_force_n2 for colloid m = blockIdx.x with the pair terms evaluated
// by the whole block: term k (from colloid k != m) goes to shared memory in
// chunks and thread 0 accumulates the chunk in k order, so the sum is the
// sequential one of force_n2_one.  A term from k < m is stored negated
// (a - f and a + (-f) round alike), so the chain is one add per interacting
// colloid, with no branch between the loads of the next terms.
__device__ inline void force_n2_block(int m, const double *px, const double *py, const double *pz, const int *sp,
                                      int C, double L0, double L1, double L2, const LJDev &lj, double *fx,
                                      double *fy, double *fz)
{
    __shared__ double term[3][kNlBlockThreads];
    __shared__ unsigned char has[kNlBlockThreads];
    double a0 = 0, a1 = 0, a2 = 0;
    if (threadIdx.x == 0) {
        a0 = fx[m];
        a1 = fy[m];
        a2 = fz[m];
    }
    for (int k0 = 0; k0 < C; k0 += kNlBlockThreads) {
        const int k = k0 + threadIdx.x;
        unsigned char h = 0;
        double f0 = 0, f1 = 0, f2 = 0;
        if (k < C && k != m) {
            int i = k < m ? k : m, j = k < m ? m : k;
            double d0 = min_image_d(px[i] - px[j], L0);
            double d1 = min_image_d(py[i] - py[j], L1);
            double d2 = min_image_d(pz[i] - pz[j], L2);
            double r_sq = d0 * d0 + d1 * d1 + d2 * d2;
            int s1 = sp[i], s2 = sp[j];
            if (r_sq <= lj.cut_sq[(s1 - 1) + lj.n1 * (s2 - 1)]) {
                int tt = (s2 - 1) + lj.n1 * (s1 - 1);
                double fr = lj_force_over_r(r_sq, lj.epsilon[tt], lj.sigma[tt]);
                f0 = fr * d0;
                f1 = fr * d1;
                f2 = fr * d2;
                if (k < m) {
                    f0 = -f0;
                    f1 = -f1;
                    f2 = -f2;
                }
                h = 1;
            }
        }
        term[0][threadIdx.x] = f0;
        term[1][threadIdx.x] = f1;
        term[2][threadIdx.x] = f2;
        has[threadIdx.x] = h;
        __syncthreads();
        if (threadIdx.x == 0) {
            const int n = min(kNlBlockThreads, C - k0);
#pragma unroll 8
            for (int q = 0; q < n; q++) {
                const bool on = has[q] != 0;
                const double u0 = term[0][q], u1 = term[1][q], u2 = term[2][q];
                a0 = on ? a0 + u0 : a0;
                a1 = on ? a1 + u1 : a1;
                a2 = on ? a2 + u2 : a2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        fx[m] = a0;
        fy[m] = a1;
        fz[m] = a2;
    }
}

// compute_force_n2, src/neighbor_list.f90:227-264: colloid m receives, in the
// sequential loop order, -f(k,m) for k < m and then +f(m,j) for j > m
__device__ inline void force_n2_one(int m, const double *px, const double *py, const double *pz, const int *sp, int C,
                                    double L0, double L1, double L2, const LJDev &lj, double *fx, double *fy,
                                    double *fz)
{
    double a0 = fx[m], a1 = fy[m], a2 = fz[m];
    for (int k = 0; k < C; k++) {
        if (k == m) continue;
        int i = k < m ? k : m, j = k < m ? m : k;
        double d0 = min_image_d(px[i] - px[j], L0);
        double d1 = min_image_d(py[i] - py[j], L1);
        double d2 = min_image_d(pz[i] - pz[j], L2);
        double r_sq = d0 * d0 + d1 * d1 + d2 * d2;
        int s1 = sp[i], s2 = sp[j];
        if (r_sq <= lj.cut_sq[(s1 - 1) + lj.n1 * (s2 - 1)]) {
            int tt = (s2 - 1) + lj.n1 * (s1 - 1);
            double fr = lj_force_over_r(r_sq, lj.epsilon[tt], lj.sigma[tt]);
            double f0 = fr * d0, f1 = fr * d1, f2 = fr * d2;
            if (k < m) {
                a0 = a0 - f0;
                a1 = a1 - f1;
                a2 = a2 - f2;
            } else {
                a0 = a0 + f0;
                a1 = a1 + f1;
                a2 = a2 + f2;
            }
        }
    }
    fx[m] = a0;
    fy[m] = a1;
    fz[m] = a2;
}

}  // namespace rmpcd
