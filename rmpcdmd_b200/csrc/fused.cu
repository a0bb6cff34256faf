// The bulk-fluid interval as one fused pass per interval (plus a slot scan
// and a key scatter), replacing the loop of test/setup_bulk_decay.f90:112-121:
//
//     simple_mpcd_step -> mpcd_stream_periodic(tau) -> random_shift -> sort
//
// Layout: inside the schedule each particle is one packed record
//     6 reals  pos(3) vel(3)        then
//     6 ints   image(3) id species flags
// (48 B in FP32 = three 16-byte chunks, 72 B in FP64 = nine 8-byte chunks),
// so the permutation gather moves whole records instead of twelve separate
// 4/8-byte fields; the SoA arrays of the API are converted on entry and
// rebuilt by the final gather.
//
// Data flow of interval i (grid G_i, next grid G_{i+1}):
//   P1  k_bulk_interval  one block per tile of consecutive Hilbert slots of
//       G_i.  The tile's particles are a contiguous range in G_i order; the
//       block loads the range's source indices (perm), sorts each cell's
//       indices ascending (the reference's stable scatter order), gathers
//       the records into shared memory with cp.async (scattered reads kept in
//       flight without stalling), performs the SRD rotation of each cell in
//       place, streams each particle, wraps it, keys it in G_{i+1}, counts
//       it, and copies the tile's records out with coalesced 16/8-byte stores.
//   P2  slot scan of the G_{i+1} counts (starts and scatter cursors).
//   P3  k_perm: perm[place] = j for every particle j of the new arrays.
// The records written by P1 hold exactly the reference's arrays after
// simple_mpcd_step and mpcd_stream_periodic; the sort into G_{i+1} is
// completed by the gather of the next P1 (or by the final gather).
//
// HBM traffic of P1 per particle: perm 4 + record read + record write +
// key 4 (104 B in FP32, 152 B in FP64), plus 12 B per slot.
#include <cmath>

#include "async_copy.cuh"
#include "cellops.cuh"
#include "keys.cuh"
#include "rng.cuh"
#include "scan.cuh"
#include "sortcore.cuh"
#include "timers.cuh"

namespace rmpcd {

constexpr int kFusedThreads = 256;

template <typename R>
struct RecT {
    static constexpr int kBytes = 6 * (int)sizeof(R) + 6 * 4;  // 48 or 72
    static constexpr int kChunk = sizeof(R) == 4 ? 16 : 8;     // copy granule
    static constexpr int kChunks = kBytes / kChunk;            // 3 or 9
    static constexpr int kIntBase = 6 * (int)sizeof(R) / 4;    // first int word
};

// record field access (rec points at the first byte of one record)
template <typename R>
__device__ __host__ inline R *rec_real(unsigned char *rec) { return (R *)rec; }
template <typename R>
__device__ __host__ inline int *rec_int(unsigned char *rec) { return (int *)rec + RecT<R>::kIntBase; }

// cells per block and staged-particle capacity; the capacity is ~7 standard
// deviations above the mean occupancy of a tile at density 10, and an
// over-full tile takes the global-memory path
template <typename R>
struct FusedCfg;
template <>
struct FusedCfg<float> {
    static constexpr int kSlots = 128;
    static constexpr int kCap = 1792;
};
template <>
struct FusedCfg<double> {
    static constexpr int kSlots = 96;
    static constexpr int kCap = 1408;
};

template <typename R>
struct FusedArgs {
    const unsigned char *in;  // records in pre-gather order
    unsigned char *out;       // records in G_i order (written)
    int *perm;                // G_i place -> record index in `in`; null = identity
    const int *count;         // G_i
    const int *start;         // G_i (0-based)
    int S;
    int N;
    int *count_next;          // G_{i+1} histogram (accumulated)
    int *key_out;             // G_{i+1} slot of out[j]
    Grid g_next;
    double e0, e1, e2;        // edges
    R dt;
    double sin_a, cos_a;
    uint64_t seed, step;
    const double *axes;
};

__device__ inline void sort_small(int *a, int n)
{
    for (int i = 1; i < n; i++) {
        int v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) {
            a[j + 1] = a[j];
            j--;
        }
        a[j + 1] = v;
    }
}

// SRD of one cell of n consecutive records (src/mpcd.f90:127-178)
template <typename R>
__device__ inline void srd_cell(unsigned char *rec0, int n, int slot, const FusedArgs<R> &A)
{
    constexpr int B = RecT<R>::kBytes;
    int n_eff = 0;
    CellSum<R> sx, sy, sz;
    for (int k = 0; k < n; k++) {
        unsigned char *r = rec0 + (size_t)k * B;
        if (rec_int<R>(r)[4] > 0) {
            R *v = rec_real<R>(r) + 3;
            sx.add(v[0]);
            sy.add(v[1]);
            sz.add(v[2]);
            n_eff++;
        }
    }
    if (n_eff <= 1) return;
    R lv[3] = {sx.value() / n_eff, sy.value() / n_eff, sz.value() / n_eff};
    double n0, n1, n2;
    if (A.axes) {
        n0 = A.axes[3 * (size_t)slot];
        n1 = A.axes[3 * (size_t)slot + 1];
        n2 = A.axes[3 * (size_t)slot + 2];
    } else {
        rng::sphere(A.seed, A.step, (uint32_t)slot, n0, n1, n2);
    }
    Rot o = srd_matrix(n0, n1, n2, A.sin_a, A.cos_a);
    for (int k = 0; k < n; k++) {
        R *v = rec_real<R>(rec0 + (size_t)k * B) + 3;
        R x = v[0], y = v[1], z = v[2];
        srd_rotate(x, y, z, lv, o);
        v[0] = x;
        v[1] = y;
        v[2] = z;
    }
}

// stream the particle of record r in place (mpcd_stream_periodic) and
// return its slot in G_{i+1}
template <typename R>
__device__ inline int stream_values(const FusedArgs<R> &A, R &x, R &y, R &z, R vx, R vy, R vz, int &ix, int &iy,
                                    int &iz)
{
    x = x + vx * A.dt;
    y = y + vy * A.dt;
    z = z + vz * A.dt;
    int jx = floor_div_edge((double)x, A.e0), jy = floor_div_edge((double)y, A.e1),
        jz = floor_div_edge((double)z, A.e2);
    if (jx) x = x - (R)(jx * A.e0);
    if (jy) y = y - (R)(jy * A.e1);
    if (jz) z = z - (R)(jz * A.e2);
    ix += jx;
    iy += jy;
    iz += jz;
    return slot_of(A.g_next, (double)x, (double)y, (double)z);
}

template <typename R>
__device__ inline int stream_rec(const FusedArgs<R> &A, unsigned char *r)
{
    if constexpr (sizeof(R) == 4) {
        // three 16-byte shared-memory accesses per record (bank-conflict free)
        int4 *q = (int4 *)r;
        int4 a = q[0], b = q[1], c = q[2];
        float x = __int_as_float(a.x), y = __int_as_float(a.y), z = __int_as_float(a.z);
        float vx = __int_as_float(a.w), vy = __int_as_float(b.x), vz = __int_as_float(b.y);
        int ix = b.z, iy = b.w, iz = c.x;
        int key = stream_values<R>(A, x, y, z, vx, vy, vz, ix, iy, iz);
        q[0] = make_int4(__float_as_int(x), __float_as_int(y), __float_as_int(z), a.w);
        q[1] = make_int4(b.x, b.y, ix, iy);
        c.x = iz;
        q[2] = c;
        return key;
    } else {
        R *f = rec_real<R>(r);
        int *w = rec_int<R>(r);
        R x = f[0], y = f[1], z = f[2];
        int ix = w[0], iy = w[1], iz = w[2];
        int key = stream_values<R>(A, x, y, z, f[3], f[4], f[5], ix, iy, iz);
        f[0] = x;
        f[1] = y;
        f[2] = z;
        w[0] = ix;
        w[1] = iy;
        w[2] = iz;
        return key;
    }
}

template <typename R>
constexpr size_t fused_smem()
{
    return (size_t)FusedCfg<R>::kCap * (RecT<R>::kBytes + sizeof(int));
}

template <typename R>
__device__ inline void copy_chunk(unsigned char *dst, const unsigned char *src)
{
    if (RecT<R>::kChunk == 16) *(int4 *)dst = *(const int4 *)src;
    else *(long long *)dst = *(const long long *)src;
}

template <typename R>
__global__ void __launch_bounds__(kFusedThreads) k_bulk_interval(FusedArgs<R> A)
{
    constexpr int SL = FusedCfg<R>::kSlots;
    constexpr int CAP = FusedCfg<R>::kCap;
    constexpr int B = RecT<R>::kBytes;
    constexpr int CH = RecT<R>::kChunk;
    constexpr int NCH = RecT<R>::kChunks;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char *s_rec = smem;
    int *s_perm = (int *)(smem + (size_t)CAP * B);

    const int t = threadIdx.x;
    const int lane = t & 31;
    const int s0 = blockIdx.x * SL;
    const int slot = s0 + t;
    const int last = min(s0 + SL, A.S) - 1;
    int my_n = 0, my_a = 0;
    if (t < SL && slot < A.S) {
        my_n = A.count[slot];
        my_a = A.start[slot];
    }
    const int a0 = A.start[s0];
    const int np = A.start[last] + A.count[last] - a0;

    if (np <= CAP) {
        // ---- staged path ----
        if (A.perm) {
            for (int j = t; j < np; j += kFusedThreads) s_perm[j] = A.perm[a0 + j];
        } else {
            for (int j = t; j < np; j += kFusedThreads) s_perm[j] = a0 + j;
        }
        __syncthreads();
        if (A.perm && my_n > 1) sort_small(s_perm + (my_a - a0), my_n);
        __syncthreads();
        // gather: consecutive threads fetch consecutive chunks of one record
        for (int q = t; q < np * NCH; q += kFusedThreads) {
            int j = q / NCH, c = q - j * NCH;
            const unsigned char *src = A.in + (size_t)s_perm[j] * B + c * CH;
            if (CH == 16) cp_async16(s_rec + (size_t)j * B + c * CH, src);
            else cp_async8(s_rec + (size_t)j * B + c * CH, src);
        }
        cp_async_wait_all();
        __syncthreads();
        if (my_n > 1) srd_cell<R>(s_rec + (size_t)(my_a - a0) * B, my_n, slot, A);
        __syncthreads();
        for (int jb = 0; jb < np; jb += kFusedThreads) {
            int j = jb + t;
            bool ok = j < np;
            int key = -1;
            if (ok) {
                key = stream_rec<R>(A, s_rec + (size_t)j * B);
                A.key_out[a0 + j] = key;
            }
            unsigned peers = __match_any_sync(0xffffffffu, key);
            if (ok && lane == __ffs(peers) - 1) atomicAdd(A.count_next + key, __popc(peers));
        }
        __syncthreads();
        // coalesced copy-out of the tile
        unsigned char *dst = A.out + (size_t)a0 * B;
        for (int q = t; q < np * NCH; q += kFusedThreads) copy_chunk<R>(dst + (size_t)q * CH, s_rec + (size_t)q * CH);
    } else {
        // ---- over-full tile (dense cells): the same steps in global memory ----
        if (A.perm && my_n > 1) sort_small(A.perm + my_a, my_n);
        __syncthreads();
        if (my_n > 0) {
            for (int k = 0; k < my_n; k++) {
                int src = A.perm ? A.perm[my_a + k] : my_a + k;
                for (int c = 0; c < NCH; c++)
                    copy_chunk<R>(A.out + (size_t)(my_a + k) * B + c * CH, A.in + (size_t)src * B + c * CH);
            }
            if (my_n > 1) srd_cell<R>(A.out + (size_t)my_a * B, my_n, slot, A);
        }
        __syncthreads();
        for (int jb = 0; jb < np; jb += kFusedThreads) {
            int j = a0 + jb + t;
            bool ok = jb + t < np;
            int key = -1;
            if (ok) {
                key = stream_rec<R>(A, A.out + (size_t)j * B);
                A.key_out[j] = key;
            }
            unsigned peers = __match_any_sync(0xffffffffu, key);
            if (ok && lane == __ffs(peers) - 1) atomicAdd(A.count_next + key, __popc(peers));
        }
    }
}

// SoA (API layout) -> records, in place order
template <typename R>
__global__ void k_soa_to_rec(PView<R> v, unsigned char *rec, int N)
{
    constexpr int B = RecT<R>::kBytes;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        unsigned char *r = rec + (size_t)i * B;
        R *f = rec_real<R>(r);
        int *w = rec_int<R>(r);
        f[0] = v.pos.x[i];
        f[1] = v.pos.y[i];
        f[2] = v.pos.z[i];
        f[3] = v.vel.x[i];
        f[4] = v.vel.y[i];
        f[5] = v.vel.z[i];
        w[0] = v.ix[i];
        w[1] = v.iy[i];
        w[2] = v.iz[i];
        w[3] = v.id[i];
        w[4] = v.species[i];
        w[5] = v.flags[i];
    }
}

// final gather: records through perm -> SoA (API layout)
template <typename R>
__global__ void k_rec_gather_to_soa(const unsigned char *rec, const int *perm, PView<R> d, int N)
{
    constexpr int B = RecT<R>::kBytes;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < N;
         j += (long long)gridDim.x * blockDim.x) {
        const unsigned char *r = rec + (size_t)perm[j] * B;
        const R *f = (const R *)r;
        const int *w = (const int *)r + RecT<R>::kIntBase;
        R px = f[0], py = f[1], pz = f[2], vx = f[3], vy = f[4], vz = f[5];
        int ix = w[0], iy = w[1], iz = w[2], id = w[3], sp = w[4], fl = w[5];
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
    }
}

template <typename R>
static int ensure_records(rmpcd_particles *p)
{
    size_t need = (size_t)p->N * RecT<R>::kBytes + 64;
    if (p->rec_bytes >= need && p->rec[0] && p->rec[1]) return RMPCD_OK;
    cudaStreamSynchronize(stream());
    cudaFree(p->rec[0]);
    cudaFree(p->rec[1]);
    p->rec[0] = p->rec[1] = nullptr;
    p->rec_bytes = 0;
    RMPCD_CUDA_TRY(cudaMalloc(&p->rec[0], need));
    RMPCD_CUDA_TRY(cudaMalloc(&p->rec[1], need));
    p->rec_bytes = need;
    return RMPCD_OK;
}

template <typename R>
static int bulk_run_fused(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r, double tau, int has_alpha,
                          double alpha, int n_intervals)
{
    cudaStream_t st = stream();
    static bool attr_set[2] = {false, false};
    if (!attr_set[sizeof(R) == 8]) {
        RMPCD_CUDA_TRY(cudaFuncSetAttribute(k_bulk_interval<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)fused_smem<R>()));
        attr_set[sizeof(R) == 8] = true;
    }
    int rc = ensure_records<R>(p);
    if (rc) return rc;
    double sin_a = 1, cos_a = 0;
    if (has_alpha) {
        sin_a = sin(alpha);
        cos_a = cos(alpha);
    }
    {
        PhaseTimer t("pack");
        k_soa_to_rec<R><<<grid_for(p->N, 256), 256, 0, st>>>(cur<R>(p), p->rec[0], p->N);
        RMPCD_CHECK_LAUNCH();
    }
    int rb = 0;  // record buffer holding the current arrays
    const int nblocks = (c->S + FusedCfg<R>::kSlots - 1) / FusedCfg<R>::kSlots;
    int *perm = nullptr;  // identity for the first interval (data sorted on entry)
    for (int it = 0; it < n_intervals; it++) {
        uint64_t step_c = r->step;
        uint64_t step_s = r->step + 1;
        r->step += 2;
        double u0, u1, u2, u3;
        rng::uniform2(r->seed, step_s, 0, rng::SHIFT, 0, u0, u1);
        rng::uniform2(r->seed, step_s, 1, rng::SHIFT, 0, u2, u3);
        FusedArgs<R> A;
        A.in = p->rec[rb];
        A.out = p->rec[1 - rb];
        A.perm = perm;
        A.count = c->count;
        A.start = c->start;
        A.S = c->S;
        A.N = p->N;
        A.count_next = c->count_next;
        A.key_out = p->key;
        A.g_next = grid_of(c);
        A.g_next.origin[0] = u0 - 1;
        A.g_next.origin[1] = u1 - 1;
        A.g_next.origin[2] = u2 - 1;
        A.e0 = c->edges[0];
        A.e1 = c->edges[1];
        A.e2 = c->edges[2];
        A.dt = (R)tau;
        A.sin_a = sin_a;
        A.cos_a = cos_a;
        A.seed = r->seed;
        A.step = step_c;
        A.axes = c->axes;
        {
            PhaseTimer t("interval_fused");
            k_bulk_interval<R><<<nblocks, kFusedThreads, fused_smem<R>(), st>>>(A);
            RMPCD_CHECK_LAUNCH();
        }
        rb = 1 - rb;
        for (int k = 0; k < 3; k++) c->origin[k] = A.g_next.origin[k];
        // the G_i arrays are consumed: the G_{i+1} counts become current
        {
            PhaseTimer t("scan");
            int *tmp = c->count;
            c->count = c->count_next;
            c->count_next = tmp;
            rc = exclusive_scan(c->count, c->start, c->cursor, c->S, c->scan_tmp, false, st);
            if (rc) return rc;
            RMPCD_CUDA_TRY(cudaMemsetAsync(c->count_next, 0, (size_t)c->S * sizeof(int), st));
        }
        {
            PhaseTimer t("perm");
            rc = build_perm_unsorted(c, p);
            if (rc) return rc;
        }
        perm = p->perm;
    }
    // complete the last sort: order each cell, gather the records into the
    // API arrays (which become current)
    PhaseTimer t("sort");
    rc = sort_perm_segments(c, p);
    if (rc) return rc;
    k_rec_gather_to_soa<R><<<grid_for(p->N, 256), 256, 0, st>>>(p->rec[rb], p->perm, alt<R>(p), p->N);
    RMPCD_CHECK_LAUNCH();
    p->cur = 1 - p->cur;
    return RMPCD_OK;
}

}  // namespace rmpcd

using namespace rmpcd;

extern "C" int rmpcd_bulk_run(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r, double tau, int has_alpha,
                              double alpha, int n_intervals)
{
    RMPCD_ARG(p && c && r, "null argument");
    RMPCD_ARG(n_intervals >= 0, "n_intervals must be >= 0");
    if (p->N == 0 || n_intervals == 0) {
        r->step += 2 * (uint64_t)n_intervals;
        return RMPCD_OK;
    }
    if (c->has_walls)
        return fail(RMPCD_ERR_INVALID, "rmpcd_bulk_run: the bulk schedule is periodic (no walls)");
    if (!p->force_zero || !p->force_old_zero) {
        // forces are carried by the sort: run the unfused sequence
        for (int it = 0; it < n_intervals; it++) {
            int rc = rmpcd_simple_mpcd_step(p, c, r, has_alpha, alpha, 0, 0.0, 1);
            if (!rc) rc = rmpcd_mpcd_stream_periodic(p, c, tau);
            if (!rc) rc = rmpcd_cells_random_shift(c, r);
            if (!rc) rc = rmpcd_particles_sort(p, c);
            if (rc) return rc;
        }
        return RMPCD_OK;
    }
    if (p->precision == RMPCD_FP32) return bulk_run_fused<float>(p, c, r, tau, has_alpha, alpha, n_intervals);
    return bulk_run_fused<double>(p, c, r, tau, has_alpha, alpha, n_intervals);
}
