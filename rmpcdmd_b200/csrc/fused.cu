// The bulk-fluid interval as one fused pass per interval (plus a slot scan
// and a key scatter), replacing the loop of test/setup_bulk_decay.f90:112-121:
//
//     simple_mpcd_step -> mpcd_stream_periodic(tau) -> random_shift -> sort
//
// Data flow of interval i (grid G_i, next grid G_{i+1}):
//   P1  k_bulk_interval  one block per 256 consecutive Hilbert slots of G_i.
//       The block's particle range is contiguous in G_i order; it loads the
//       range's source indices (perm), sorts each cell's indices ascending
//       (the reference's stable scatter order), gathers velocities and
//       species into shared memory, performs the SRD rotation of every cell
//       in place, then streams each particle, wraps it, computes its slot in
//       G_{i+1}, counts it, and writes the whole particle record in G_i order.
//   P2  slot scan of the G_{i+1} counts (starts and scatter cursors).
//   P3  k_perm: perm[place] = j for every particle j of the new arrays.
// The arrays written by P1 are exactly the reference's arrays after
// simple_mpcd_step and mpcd_stream_periodic; the sort into G_{i+1} is
// completed by the gather of the next P1 (or by a final gather).
//
// HBM traffic of P1 per particle: perm 4 + vel 3R + species 4 + pos 3R +
// image 12 + flags 4 + id 4 read, the same record + key 4 written.
#include <cmath>

#include "cellops.cuh"
#include "keys.cuh"
#include "rng.cuh"
#include "scan.cuh"
#include "sortcore.cuh"
#include "timers.cuh"

namespace rmpcd {

constexpr int kFusedSlots = 256;  // cells (and threads) per block
constexpr int kFusedCap = 3072;   // particles staged in shared memory per block

template <typename R>
struct FusedArgs {
    PView<R> in;        // particle arrays in pre-gather order
    PView<R> out;       // particle arrays in G_i order (written)
    int *perm;          // G_i place -> index into `in`; null = identity
    const int *count;   // G_i
    const int *start;   // G_i (0-based)
    int S;
    int N;
    int *count_next;    // G_{i+1} histogram (accumulated)
    int *key_out;       // G_{i+1} slot of out[j]
    Grid g_next;
    double e0, e1, e2;  // edges
    R dt;
    double sin_a, cos_a;
    uint64_t seed, step;
    const double *axes;
};

template <typename R>
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

// SRD of one cell whose velocities sit at vx[0..n) (src/mpcd.f90:127-178)
template <typename R>
__device__ inline void srd_cell(R *vx, R *vy, R *vz, const int *sp, int n, int slot,
                                const FusedArgs<R> &A)
{
    int n_eff = 0;
    CellSum<R> sx, sy, sz;
    for (int k = 0; k < n; k++) {
        if (sp[k] > 0) {
            sx.add(vx[k]);
            sy.add(vy[k]);
            sz.add(vz[k]);
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
        R x = vx[k], y = vy[k], z = vz[k];
        srd_rotate(x, y, z, lv, o);
        vx[k] = x;
        vy[k] = y;
        vz[k] = z;
    }
}

// stream particle `src` with velocity v, write it at place j, key + count it
template <typename R>
__device__ inline int stream_write(const FusedArgs<R> &A, int j, int src, R vx, R vy, R vz, int sp)
{
    R x = A.in.pos.x[src] + vx * A.dt;
    R y = A.in.pos.y[src] + vy * A.dt;
    R z = A.in.pos.z[src] + vz * A.dt;
    int jx = ifloor((double)x / A.e0), jy = ifloor((double)y / A.e1), jz = ifloor((double)z / A.e2);
    x = x - (R)(jx * A.e0);
    y = y - (R)(jy * A.e1);
    z = z - (R)(jz * A.e2);
    A.out.pos.x[j] = x;
    A.out.pos.y[j] = y;
    A.out.pos.z[j] = z;
    A.out.vel.x[j] = vx;
    A.out.vel.y[j] = vy;
    A.out.vel.z[j] = vz;
    A.out.ix[j] = A.in.ix[src] + jx;
    A.out.iy[j] = A.in.iy[src] + jy;
    A.out.iz[j] = A.in.iz[src] + jz;
    A.out.species[j] = sp;
    A.out.flags[j] = A.in.flags[src];
    A.out.id[j] = A.in.id[src];
    int key = slot_of(A.g_next, (double)x, (double)y, (double)z);
    A.key_out[j] = key;
    return key;
}

template <typename R>
__global__ void __launch_bounds__(kFusedSlots) k_bulk_interval(FusedArgs<R> A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    R *s_vx = (R *)smem;
    R *s_vy = s_vx + kFusedCap;
    R *s_vz = s_vy + kFusedCap;
    int *s_perm = (int *)(s_vz + kFusedCap);
    int *s_sp = s_perm + kFusedCap;

    const int t = threadIdx.x;
    const int lane = t & 31;
    const int s0 = blockIdx.x * kFusedSlots;
    const int slot = s0 + t;
    const int last = min(s0 + kFusedSlots, A.S) - 1;
    int my_n = 0, my_a = 0;
    if (slot < A.S) {
        my_n = A.count[slot];
        my_a = A.start[slot];
    }
    const int a0 = A.start[s0];
    const int np = A.start[last] + A.count[last] - a0;

    if (np <= kFusedCap) {
        // ---- staged path ----
        for (int j = t; j < np; j += kFusedSlots) s_perm[j] = A.perm ? A.perm[a0 + j] : a0 + j;
        __syncthreads();
        if (A.perm && my_n > 1) sort_small<R>(s_perm + (my_a - a0), my_n);
        __syncthreads();
        for (int j = t; j < np; j += kFusedSlots) {
            int src = s_perm[j];
            s_vx[j] = A.in.vel.x[src];
            s_vy[j] = A.in.vel.y[src];
            s_vz[j] = A.in.vel.z[src];
            s_sp[j] = A.in.species[src];
        }
        __syncthreads();
        if (my_n > 1) {
            int o = my_a - a0;
            srd_cell<R>(s_vx + o, s_vy + o, s_vz + o, s_sp + o, my_n, slot, A);
        }
        __syncthreads();
        for (int jb = 0; jb < np; jb += kFusedSlots) {
            int j = jb + t;
            bool ok = j < np;
            int key = -1;
            if (ok) key = stream_write<R>(A, a0 + j, s_perm[j], s_vx[j], s_vy[j], s_vz[j], s_sp[j]);
            unsigned peers = __match_any_sync(0xffffffffu, key);
            if (ok && lane == __ffs(peers) - 1) atomicAdd(A.count_next + key, __popc(peers));
        }
    } else {
        // ---- oversized block (dense cells): same steps through global memory ----
        if (A.perm && my_n > 1) sort_small<R>(A.perm + my_a, my_n);
        __syncthreads();
        if (my_n > 0) {
            // gather the cell into its output place, then collide there
            for (int k = 0; k < my_n; k++) {
                int src = A.perm ? A.perm[my_a + k] : my_a + k;
                A.out.vel.x[my_a + k] = A.in.vel.x[src];
                A.out.vel.y[my_a + k] = A.in.vel.y[src];
                A.out.vel.z[my_a + k] = A.in.vel.z[src];
                A.out.species[my_a + k] = A.in.species[src];
            }
            if (my_n > 1)
                srd_cell<R>(A.out.vel.x + my_a, A.out.vel.y + my_a, A.out.vel.z + my_a,
                            A.out.species + my_a, my_n, slot, A);
        }
        __syncthreads();
        for (int jb = 0; jb < np; jb += kFusedSlots) {
            int j = a0 + jb + t;
            bool ok = jb + t < np;
            int key = -1;
            if (ok) {
                int src = A.perm ? A.perm[j] : j;
                key = stream_write<R>(A, j, src, A.out.vel.x[j], A.out.vel.y[j], A.out.vel.z[j],
                                      A.out.species[j]);
            }
            unsigned peers = __match_any_sync(0xffffffffu, key);
            if (ok && lane == __ffs(peers) - 1) atomicAdd(A.count_next + key, __popc(peers));
        }
    }
}

template <typename R>
constexpr size_t fused_smem()
{
    return (size_t)kFusedCap * (3 * sizeof(R) + 2 * sizeof(int));
}

__global__ void k_iota0(int *a, int N)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        a[i] = (int)i;
}

template <typename R>
static int bulk_run_fused(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r, double tau, int has_alpha,
                          double alpha, int n_intervals)
{
    cudaStream_t st = stream();
    static bool attr_set = false;
    if (!attr_set) {
        RMPCD_CUDA_TRY(cudaFuncSetAttribute(k_bulk_interval<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)fused_smem<float>()));
        RMPCD_CUDA_TRY(cudaFuncSetAttribute(k_bulk_interval<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)fused_smem<double>()));
        attr_set = true;
    }
    double sin_a = 1, cos_a = 0;
    if (has_alpha) {
        sin_a = sin(alpha);
        cos_a = cos(alpha);
    }
    const int nblocks = (c->S + kFusedSlots - 1) / kFusedSlots;
    int *perm = nullptr;  // identity for the first interval (data sorted on entry)
    for (int it = 0; it < n_intervals; it++) {
        uint64_t step_c = r->step;
        uint64_t step_s = r->step + 1;
        r->step += 2;
        double u0, u1, u2, u3;
        rng::uniform2(r->seed, step_s, 0, rng::SHIFT, 0, u0, u1);
        rng::uniform2(r->seed, step_s, 1, rng::SHIFT, 0, u2, u3);
        FusedArgs<R> A;
        A.in = cur<R>(p);
        A.out = alt<R>(p);
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
            k_bulk_interval<R><<<nblocks, kFusedSlots, fused_smem<R>(), st>>>(A);
            RMPCD_CHECK_LAUNCH();
        }
        p->cur = 1 - p->cur;
        for (int k = 0; k < 3; k++) c->origin[k] = A.g_next.origin[k];
        // the G_i arrays are consumed: the G_{i+1} counts become current
        {
            PhaseTimer t("scan");
            int *tmp = c->count;
            c->count = c->count_next;
            c->count_next = tmp;
            int rc = exclusive_scan(c->count, c->start, c->cursor, c->S, c->scan_tmp, false, st);
            if (rc) return rc;
            RMPCD_CUDA_TRY(cudaMemsetAsync(c->count_next, 0, (size_t)c->S * sizeof(int), st));
        }
        {
            PhaseTimer t("perm");
            int rc = build_perm_unsorted(c, p);
            if (rc) return rc;
        }
        perm = p->perm;
    }
    if (n_intervals > 0) {
        // complete the last sort: order each cell, then gather every field
        PhaseTimer t("sort");
        int rc = sort_perm_segments(c, p);
        if (rc) return rc;
        rc = gather_all(p);
        if (rc) return rc;
    }
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
