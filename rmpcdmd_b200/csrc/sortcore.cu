#include "keys.cuh"
#include "scan.cuh"
#include "sortcore.cuh"
#include "sortnet.cuh"
#include "timers.cuh"

namespace rmpcd {

constexpr int kSmallSegment = kSmallSegmentMax;

// key[i] = slot of particle i; histogram with one atomic per distinct key
// per warp (consecutive particles usually share a cell).
template <typename R>
__global__ void k_key_count(Grid g, const R *__restrict__ x, const R *__restrict__ y,
                            const R *__restrict__ z, int N, int *__restrict__ key,
                            int *__restrict__ count)
{
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < N; base += stride) {
        long long i = base + threadIdx.x;
        bool ok = i < N;
        int s = -1;
        if (ok) {
            s = slot_of(g, (double)x[i], (double)y[i], (double)z[i]);
            key[i] = s;
        }
        unsigned peers = __match_any_sync(0xffffffffu, s);
        if (ok && lane == __ffs(peers) - 1) atomicAdd(count + s, __popc(peers));
    }
}

// the same with apply_pbc (src/md.f90:202-217) done on each particle first:
// the wrapped position is the one keyed, and pos / image are written only
// for particles that wrap
template <typename R>
__global__ void k_pbc_key_count(Grid g, PView<R> v, double e0, double e1, double e2, int N,
                                int *__restrict__ key, int *__restrict__ count)
{
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < N; base += stride) {
        long long i = base + threadIdx.x;
        bool ok = i < N;
        int s = -1;
        if (ok) {
            R x = v.pos.x[i], y = v.pos.y[i], z = v.pos.z[i];
            const int jx = floor_div_edge((double)x, e0), jy = floor_div_edge((double)y, e1),
                      jz = floor_div_edge((double)z, e2);
            if (jx) {
                v.ix[i] += jx;
                x = x - (R)(jx * e0);
                v.pos.x[i] = x;
            }
            if (jy) {
                v.iy[i] += jy;
                y = y - (R)(jy * e1);
                v.pos.y[i] = y;
            }
            if (jz) {
                v.iz[i] += jz;
                z = z - (R)(jz * e2);
                v.pos.z[i] = z;
            }
            s = slot_of(g, (double)x, (double)y, (double)z);
            key[i] = s;
        }
        unsigned peers = __match_any_sync(0xffffffffu, s);
        if (ok && lane == __ffs(peers) - 1) atomicAdd(count + s, __popc(peers));
    }
}

// place every particle inside its cell; the order inside a cell is fixed
// afterwards by k_segsort.  Each warp handles kPermRounds groups of 32
// consecutive particles and issues all their cursor atomics before using any
// result, so the atomic round trips overlap.  cellmap (if given) receives the
// slot of every place: the slot of each particle of the sorted arrays.
constexpr int kPermRounds = 8;

__global__ void k_perm(const int *__restrict__ key, int N, int *__restrict__ cursor,
                       int *__restrict__ perm, int *__restrict__ cellmap)
{
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned lt = lanemask_lt();
    for (long long base = warp * 32 * kPermRounds; base < N; base += nwarps * 32 * kPermRounds) {
        int k[kPermRounds];
        unsigned peers[kPermRounds];
        int b[kPermRounds];
#pragma unroll
        for (int r = 0; r < kPermRounds; r++) {
            long long i = base + r * 32 + lane;
            k[r] = i < N ? key[i] : -1;
        }
#pragma unroll
        for (int r = 0; r < kPermRounds; r++) {
            peers[r] = __match_any_sync(0xffffffffu, k[r]);
            b[r] = 0;
            if (k[r] >= 0 && lane == __ffs(peers[r]) - 1) b[r] = atomicAdd(cursor + k[r], __popc(peers[r]));
        }
#pragma unroll
        for (int r = 0; r < kPermRounds; r++) {
            int bb = __shfl_sync(0xffffffffu, b[r], __ffs(peers[r]) - 1);
            if (k[r] >= 0) {
                const int place = bb + __popc(peers[r] & lt);
                perm[place] = (int)(base + r * 32 + lane);
                if (cellmap) cellmap[place] = k[r];
            }
        }
    }
}

// ascending insertion sort of short segments; long ones are queued
__global__ void k_segsort_small(const int *__restrict__ start, const int *__restrict__ count,
                                int S, int *__restrict__ perm, int *__restrict__ big,
                                int *__restrict__ n_big)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        int n = count[s];
        if (n <= 1) continue;
        if (n > kSmallSegment) {
            int q = atomicAdd(n_big, 1);
            big[q] = s;
            continue;
        }
        sort_segment(perm + start[s], n);
    }
}

__device__ inline int lower_bound_int(const int *a, int n, int v)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// one block per long segment: bottom-up merge sort of distinct values, every
// element placed by its rank in the partner run; tmp is scratch of the same
// extent as the segment
__global__ void k_segsort_big(const int *__restrict__ start, const int *__restrict__ count,
                              const int *__restrict__ big, const int *__restrict__ n_big,
                              int *__restrict__ perm, int *__restrict__ tmp)
{
    for (int q = blockIdx.x; q < *n_big; q += gridDim.x) {
        int s = big[q];
        int n = count[s];
        int *a = perm + start[s];
        int *b = tmp + start[s];
        int *src = a, *dst = b;
        for (int w = 1; w < n; w <<= 1) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                int run = i / w;
                int r0 = run * w;
                int v = src[i];
                int pos;
                if ((run & 1) == 0) {
                    int p0 = r0 + w;
                    int pn = min(w, max(0, n - p0));
                    pos = r0 + (i - r0) + lower_bound_int(src + p0, pn, v);
                } else {
                    int p0 = r0 - w;
                    pos = p0 + (i - r0) + lower_bound_int(src + p0, w, v);
                }
                dst[pos] = v;
            }
            __syncthreads();
            int *t = src;
            src = dst;
            dst = t;
        }
        if (src != a)
            for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = src[i];
        __syncthreads();
    }
}

// gated != 0: a particle with neither MD nor PAST_MD set is known to have
// zero force and force_old, so those are written as zeros without a read
template <typename R>
__global__ void k_gather(PView<R> s, PView<R> d, const int *__restrict__ perm, int N,
                         int with_force, int with_force_old, int gated)
{
    const int fmask = (1 << MD_BIT) | (1 << PAST_MD_BIT);
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < N;
         j += (long long)gridDim.x * blockDim.x) {
        const int i = perm[j];
        // all loads first: twelve independent gathers in flight per thread
        R px = s.pos.x[i], py = s.pos.y[i], pz = s.pos.z[i];
        R vx = s.vel.x[i], vy = s.vel.y[i], vz = s.vel.z[i];
        int ix = s.ix[i], iy = s.iy[i], iz = s.iz[i];
        int id = s.id[i], sp = s.species[i], fl = s.flags[i];
        d.pos.x[j] = px;
        d.pos.y[j] = py;
        d.pos.z[j] = pz;
        d.vel.x[j] = vx;
        d.vel.y[j] = vy;
        d.vel.z[j] = vz;
        d.ix[j] = ix;
        d.iy[j] = iy;
        d.iz[j] = iz;
        d.id[j] = id;
        d.species[j] = sp;
        d.flags[j] = fl;
        const bool live = !gated || (fl & fmask);
        if (with_force) {
            d.force.x[j] = live ? s.force.x[i] : (R)0;
            d.force.y[j] = live ? s.force.y[i] : (R)0;
            d.force.z[j] = live ? s.force.z[i] : (R)0;
        }
        if (with_force_old) {
            d.force_old.x[j] = live ? s.force_old.x[i] : (R)0;
            d.force_old.y[j] = live ? s.force_old.y[i] : (R)0;
            d.force_old.z[j] = live ? s.force_old.z[i] : (R)0;
        }
    }
}

template <typename R>
static int count_and_scan_t(rmpcd_cells *c, rmpcd_particles *p)
{
    cudaStream_t st = stream();
    RMPCD_CUDA_TRY(cudaMemsetAsync(c->count, 0, (size_t)c->S * sizeof(int), st));
    PView<R> v = cur<R>(p);
    if (p->N > 0)
        k_key_count<R><<<grid_for(p->N, 256), 256, 0, st>>>(grid_of(c), v.pos.x, v.pos.y, v.pos.z,
                                                           p->N, p->key, c->count);
    RMPCD_CHECK_LAUNCH();
    return exclusive_scan(c->count, c->start, c->cursor, c->S, c->scan_tmp, nullptr, st);
}

int count_and_scan(rmpcd_cells *c, rmpcd_particles *p, bool)
{
    if (p->precision == RMPCD_FP32) return count_and_scan_t<float>(c, p);
    return count_and_scan_t<double>(c, p);
}

int build_perm_unsorted(rmpcd_cells *c, rmpcd_particles *p, int *cellmap)
{
    if (p->N == 0) return RMPCD_OK;
    k_perm<<<grid_for(p->N, 256), 256, 0, stream()>>>(p->key, p->N, c->cursor, p->perm, cellmap);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int build_perm(rmpcd_cells *c, rmpcd_particles *p, int *cellmap)
{
    int rc = build_perm_unsorted(c, p, cellmap);
    if (rc) return rc;
    return sort_perm_segments(c, p);
}

int sort_perm_segments(rmpcd_cells *c, rmpcd_particles *p)
{
    cudaStream_t st = stream();
    if (p->N == 0) return RMPCD_OK;
    // big-segment queue lives in cursor[] (free once perm is built) plus a counter
    int *n_big = p->d_ints;
    RMPCD_CUDA_TRY(cudaMemsetAsync(n_big, 0, sizeof(int), st));
    k_segsort_small<<<grid_full(c->S, 256), 256, 0, st>>>(c->start, c->count, c->S, p->perm,
                                                         c->cursor, n_big);
    k_segsort_big<<<64, 512, 0, st>>>(c->start, c->count, c->cursor, n_big, p->perm, p->key);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

template <typename R>
static int gather_t(rmpcd_particles *p, bool gated = false)
{
    if (p->N > 0) {
        k_gather<R><<<grid_for(p->N, 256), 256, 0, stream()>>>(
            cur<R>(p), alt<R>(p), p->perm, p->N, p->force_zero ? 0 : 1, p->force_old_zero ? 0 : 1, gated ? 1 : 0);
        RMPCD_CHECK_LAUNCH();
    }
    p->cur = 1 - p->cur;
    // fields that were not gathered are all zero: keep the live pointer on the
    // (zero) previous arrays
    for (int k = 0; k < 3; k++) {
        if (p->force_zero) {
            void *t = p->force[p->cur][k];
            p->force[p->cur][k] = p->force[1 - p->cur][k];
            p->force[1 - p->cur][k] = t;
        }
        if (p->force_old_zero) {
            void *t = p->force_old[p->cur][k];
            p->force_old[p->cur][k] = p->force_old[1 - p->cur][k];
            p->force_old[1 - p->cur][k] = t;
        }
    }
    return RMPCD_OK;
}

void launch_segsort_big(const int *start, const int *count, const int *big, const int *n_big, int *perm,
                        int *tmp, cudaStream_t st)
{
    k_segsort_big<<<64, 512, 0, st>>>(start, count, big, n_big, perm, tmp);
}

int gather_all(rmpcd_particles *p)
{
    if (p->precision == RMPCD_FP32) return gather_t<float>(p);
    return gather_t<double>(p);
}

template <typename R>
static int sort_keyed_flagged_t(rmpcd_cells *c, rmpcd_particles *p, int *cellmap)
{
    {
        PhaseTimer t("count");
        int rc = exclusive_scan(c->count, c->start, c->cursor, c->S, c->scan_tmp, nullptr, stream());
        if (rc) return rc;
    }
    PhaseTimer t("sort");
    int rc = build_perm(c, p, cellmap);
    if (rc) return rc;
    return gather_t<R>(p, true);
}

int sort_keyed_flagged(rmpcd_cells *c, rmpcd_particles *p, int *cellmap)
{
    if (p->precision == RMPCD_FP32) return sort_keyed_flagged_t<float>(c, p, cellmap);
    return sort_keyed_flagged_t<double>(c, p, cellmap);
}

template <typename R>
static int sort_particles_flagged_t(rmpcd_cells *c, rmpcd_particles *p, const double edges[3])
{
    {
        PhaseTimer t("count");
        cudaStream_t st = stream();
        RMPCD_CUDA_TRY(cudaMemsetAsync(c->count, 0, (size_t)c->S * sizeof(int), st));
        if (p->N > 0)
            k_pbc_key_count<R><<<grid_for(p->N, 256), 256, 0, st>>>(grid_of(c), cur<R>(p), edges[0], edges[1],
                                                                   edges[2], p->N, p->key, c->count);
        RMPCD_CHECK_LAUNCH();
    }
    return sort_keyed_flagged_t<R>(c, p, nullptr);
}

int sort_particles_flagged(rmpcd_cells *c, rmpcd_particles *p, const double edges[3])
{
    if (p->precision == RMPCD_FP32) return sort_particles_flagged_t<float>(c, p, edges);
    return sort_particles_flagged_t<double>(c, p, edges);
}

// cell_system_t%sort_particles (src/cell_system.f90:131-151): the positions
// of `from` scattered into the positions of `to` through the starts of the
// last count_particles.  Before any scatter, one pass keys the positions and
// checks that they give exactly the counts on record and that every cell's
// range lies inside [0, N); a mismatch is an argument error and nothing is
// written.  The order inside a cell is ascending source index (the
// reference's single-thread order); afterwards every start has advanced by
// its cell's count, as the reference's scatter cursor leaves cell_start.
template <typename R>
__global__ void k_key_check(Grid g, const R *__restrict__ x, const R *__restrict__ y, const R *__restrict__ z,
                            int N, int *__restrict__ key, int *__restrict__ hist)
{
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < N; base += stride) {
        long long i = base + threadIdx.x;
        bool ok = i < N;
        int s = -1;
        if (ok) {
            s = slot_of(g, (double)x[i], (double)y[i], (double)z[i]);
            key[i] = s;
        }
        unsigned peers = __match_any_sync(0xffffffffu, s);
        if (ok && lane == __ffs(peers) - 1) atomicAdd(hist + s, __popc(peers));
    }
}

__global__ void k_counts_agree(const int *__restrict__ hist, const int *__restrict__ count,
                               const int *__restrict__ start, int S, int N, int *__restrict__ bad)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        const int n = count[s], a = start[s];
        if (hist[s] != n || n < 0 || a < 0 || (long long)a + n > N) atomicOr(bad, 1);
    }
}

template <typename R>
__global__ void k_gather_pos(Vec3<R> src, Vec3<R> dst, const int *__restrict__ perm, int N)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < N; j += stride) {
        const int i = perm[j];
        dst.x[j] = src.x[i];
        dst.y[j] = src.y[i];
        dst.z[j] = src.z[i];
    }
}

__global__ void k_advance_starts(int *__restrict__ start, const int *__restrict__ count, int S)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) start[s] += count[s];
}

template <typename R>
static int sort_positions_t(rmpcd_cells *c, const rmpcd_particles *from, rmpcd_particles *to)
{
    cudaStream_t st = stream();
    const int N = from->N;
    int *bad = to->d_ints;
    // the cursors are free until the scatter: they hold the check's histogram
    RMPCD_CUDA_TRY(cudaMemsetAsync(c->cursor, 0, (size_t)c->S * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    PView<R> s = cur<R>(from);
    if (N > 0)
        k_key_check<R><<<grid_for(N, 256), 256, 0, st>>>(grid_of(c), s.pos.x, s.pos.y, s.pos.z, N, to->key,
                                                         c->cursor);
    k_counts_agree<<<grid_for(c->S, 256), 256, 0, st>>>(c->cursor, c->count, c->start, c->S, N, bad);
    RMPCD_CHECK_LAUNCH();
    int h_bad = 0;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    RMPCD_CUDA_TRY(cudaStreamSynchronize(st));
    if (h_bad)
        return fail(RMPCD_ERR_INVALID,
                    "sort_particles: the cell counts and starts are not those of these positions "
                    "(call count_particles on them first)");
    if (N > 0) {
        RMPCD_CUDA_TRY(cudaMemcpyAsync(c->cursor, c->start, (size_t)c->S * sizeof(int), cudaMemcpyDeviceToDevice, st));
        int rc = build_perm(c, to);
        if (rc) return rc;
        k_gather_pos<R><<<grid_for(N, 256), 256, 0, st>>>(s.pos, cur<R>(to).pos, to->perm, N);
    }
    k_advance_starts<<<grid_for(c->S, 256), 256, 0, st>>>(c->start, c->count, c->S);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int sort_positions(rmpcd_cells *c, const rmpcd_particles *from, rmpcd_particles *to)
{
    if (from->precision == RMPCD_FP32) return sort_positions_t<float>(c, from, to);
    return sort_positions_t<double>(c, from, to);
}

int sort_particles(rmpcd_cells *c, rmpcd_particles *p)
{
    int rc;
    {
        PhaseTimer t("count");
        rc = count_and_scan(c, p, true);
        if (rc) return rc;
    }
    PhaseTimer t("sort");
    rc = build_perm(c, p);
    if (rc) return rc;
    return gather_all(p);
}

}  // namespace rmpcd
