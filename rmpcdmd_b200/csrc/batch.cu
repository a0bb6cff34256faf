// Batched single-dimer engine: R independent single_dimer_pbc systems
// (programs/single_dimer_pbc.f90:303-443), each with its own box, seed and
// solvent, advanced together.  Every phase of the program's MD step and MPCD
// interval is one launch over all replicas: solvent work is cut into tiles of
// kTile particles (or slots) that each belong to one replica, colloid work is
// one thread or block per replica.  The replicas' solvents are concatenated
// in one particle system, their slot ranges in one slot space; a replica's
// Hilbert order stays inside its own range, so the sort kernels of a single
// system apply to every replica at once.
//
// The extra re-sort that single_dimer_pbc performs when a particle moved too
// far (programs/single_dimer_pbc.f90:320-330) is decided on the device: the
// colloid kernel writes one flag per replica and every re-sort kernel skips
// the tiles of replicas whose flag is clear.  The re-sort gathers into the
// alternate buffers and copies back, so the arrays never change place and a
// whole interval (N_MD MD steps + shift + sort + collision + refuel) can be
// captured once in a CUDA graph and replayed: the RNG step and the grid
// origins are read from device memory, never baked into the graph.
//
// Arithmetic per particle is that of the single-system kernels
// (stepops.cuh, nlist_ops.cuh), so replica r reproduces, bit for bit, the
// same program run alone through the C ABI with its own seed.
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "keys.cuh"
#include "nlist_ops.cuh"
#include "rmpcd_common.cuh"
#include "rng.cuh"
#include "sortcore.cuh"
#include "sortnet.cuh"
#include "state.cuh"
#include "stepops.cuh"
#include "timers.cuh"

namespace rmpcd {

constexpr int kTile = 1024;  // particles or slots per tile
constexpr int kBT = 256;     // threads per tile block

struct BTile {
    int r;
    int pad;
    long long begin, end;
};

struct BRep {
    long long off;  // first solvent particle of the replica
    int n;          // its solvent particles
    int soff;       // first slot
    int S;          // its slots
    int serial;     // the list stencil wraps this box: ordered single-thread force application
    uint64_t seed;
    double far;     // refuel distance (single-precision expression of the program)
    Grid g;         // cells; origin rewritten on the device by the grid shift
};

}  // namespace rmpcd

struct rmpcd_dimer_batch {
    int R = 0;
    int precision = RMPCD_FP64;
    rmpcd_dimer_params prm{};
    long long Ntot = 0;
    int Stot = 0;
    rmpcd_particles *sol = nullptr;  // all solvents, concatenated (buffer 0 current, 1 = gather target / pos_old)
    rmpcd_particles *col = nullptr;  // all colloids, 2 per replica
    std::vector<rmpcd::BRep> rep_h;
    rmpcd::BRep *rep = nullptr;
    rmpcd::BTile *ptile = nullptr, *stile = nullptr;
    int n_ptile = 0, n_stile = 0;
    int *stile_first = nullptr, *stile_count = nullptr;  // per replica
    long long *tile_sum = nullptr, *tile_off = nullptr;  // per slot tile
    int *count = nullptr, *start = nullptr, *cursor = nullptr;
    unsigned char *is_md = nullptr, *is_reac = nullptr;
    std::vector<int *> luts;
    int *stencil = nullptr;
    int n_stencil = 0;
    int Nmax = 0;
    int *list = nullptr, *nn = nullptr;
    double *pair_f = nullptr, *pair_e = nullptr;
    unsigned char *contrib = nullptr;
    int *ncontrib = nullptr, *max_contrib = nullptr, *clist = nullptr, *cn = nullptr;
    unsigned long long *so_max = nullptr;
    int *resort = nullptr, *n_extra = nullptr, *big = nullptr, *n_big = nullptr;
    double *rattle[3] = {nullptr, nullptr, nullptr};
    double *vv_mass = nullptr;
    uint64_t *d_step = nullptr;
    uint64_t step = 0;  // host copy of every replica's RNG step
    rmpcd::Masses ms{};
    rmpcd::LJDev lj_sc{}, lj_cc{};
    int parity = 0;  // 0: force = buffer force[0], force_old = force_old[0]; swapped by each MD step
    bool use_graph = true;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
};

namespace rmpcd {

// ------------------------------------------------------------------ views

template <typename R>
static PView<R> phys(const rmpcd_particles *p, int b)
{
    return view<R>(p, b);
}

// current arrays with force / force_old as the MD-step parity says
template <typename R>
static PView<R> live(const rmpcd_particles *p, int parity)
{
    PView<R> v = view<R>(p, 0);
    if (parity) {
        Vec3<R> t = v.force;
        v.force = v.force_old;
        v.force_old = t;
    }
    return v;
}

template <typename R>
__device__ inline PView<R> shifted(PView<R> v, long long off, int n)
{
    v.N = n;
    v.pos = {v.pos.x + off, v.pos.y + off, v.pos.z + off};
    v.vel = {v.vel.x + off, v.vel.y + off, v.vel.z + off};
    v.force = {v.force.x + off, v.force.y + off, v.force.z + off};
    v.force_old = {v.force_old.x + off, v.force_old.y + off, v.force_old.z + off};
    v.ix += off;
    v.iy += off;
    v.iz += off;
    v.id += off;
    v.species += off;
    v.flags += off;
    return v;
}

__device__ inline bool tile_active(const BTile &t, const int *flag)
{
    return !flag || flag[t.r];
}

// ------------------------------------------------------------ MD step

// md_pos + the PAST_MD/MD flag roll of compute_force + the solvent's
// maximum displacement (src/md.f90:61-77, src/neighbor_list.f90:180-188,
// src/particle_system.f90:357-378)
template <typename R>
__global__ void __launch_bounds__(kBT) kb_md_pos(const BTile *tiles, PView<R> v, Vec3<R> old, R dt, R dt_sq,
                                                 unsigned long long *so_max)
{
    const BTile t = tiles[blockIdx.x];
    double m = 0;
    for (long long i = t.begin + threadIdx.x; i < t.end; i += blockDim.x) {
        md_pos_one(v, i, dt, dt_sq);
        flag_roll_one(v.flags, i);
        double r = disp_sq_one(v.pos, old, v.species, i);
        m = m > r ? m : r;
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(so_max + t.r, m);
}

// colloid position half, RATTLE, colloid displacement and the re-sort
// decision of programs/single_dimer_pbc.f90:311-330 (one thread per replica)
__global__ void kb_colloid_pos(int R, const BRep *rep, PView<double> c, Vec3<double> cold, double *rx, double *ry,
                               double *rz, const double *mass, Masses ms, double d, double dt, double skin,
                               unsigned long long *so_max, int *resort, int *n_extra, unsigned *err)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        PView<double> cr = shifted(c, 2 * (long long)r, 2);
        for (int k = 0; k < 2; k++) {
            rx[2 * r + k] = cr.pos.x[k];
            ry[2 * r + k] = cr.pos.y[k];
            rz[2 * r + k] = cr.pos.z[k];
        }
        colloid_vv_pos_one(cr, 0, mass[2 * r], dt);
        colloid_vv_pos_one(cr, 1, mass[2 * r + 1], dt);
        E3 L{{rep[r].g.edges[0], rep[r].g.edges[1], rep[r].g.edges[2]}};
        rattle_pos_dimer(cr, rx + 2 * r, ry + 2 * r, rz + 2 * r, ms, d, dt, L, err);
        Vec3<double> o = {cold.x + 2 * r, cold.y + 2 * r, cold.z + 2 * r};
        double m0 = disp_sq_one(cr.pos, o, cr.species, 0), m1 = disp_sq_one(cr.pos, o, cr.species, 1);
        double co_max = sqrt(m0 > m1 ? m0 : m1);
        double so = sqrt(__longlong_as_double((long long)so_max[r]));
        int need = (co_max >= skin * 0.1) || (so >= skin * 0.89);
        resort[r] = need;
        if (need) n_extra[r] += 1;
        so_max[r] = 0;
    }
}

// list pair forces (src/neighbor_list.f90:198-219) fused with
// flag_particles_nl of the catalytic bead (programs/single_dimer_pbc.f90:493-509):
// both only read positions and species and OR bits into flags
template <typename R>
__global__ void kb_pair_forces(const BRep *rep, PView<double> c, PView<R> s, const int *list, const int *n, int Nmax,
                               LJDev lj, double *pf, double *pe, unsigned char *contrib, int *ncontrib,
                               int *max_contrib, double flag_cut_sq)
{
    const int i = blockIdx.y;
    const int r = i >> 1;
    const int ni = n[i];
    const double x[3] = {c.pos.x[i], c.pos.y[i], c.pos.z[i]};
    const int s1 = c.species[i];
    const double L0 = rep[r].g.edges[0], L1 = rep[r].g.edges[1], L2 = rep[r].g.edges[2];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ni; e += gridDim.x * blockDim.x) {
        size_t q = (size_t)i * Nmax + e;
        pair_force_entry(q, x, s1, s.pos.x, s.pos.y, s.pos.z, s.species, s.flags, list, L0, L1, L2, lj, pf, pe,
                         contrib, ncontrib, max_contrib + r);
        if ((i & 1) == 0)
            flag_nl_one(list[q], x, s.pos.x, s.pos.y, s.pos.z, s.species, s.flags, L0, L1, L2, flag_cut_sq);
    }
}

template <typename R>
__global__ void kb_apply_single(const int *list, const int *n, int Nmax, const unsigned char *contrib,
                                const double *pf, const int *ncontrib, R *fx, R *fy, R *fz)
{
    const int i = blockIdx.y;
    const int ni = n[i];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ni; e += gridDim.x * blockDim.x)
        apply_single_entry((size_t)i * Nmax + e, list, contrib, pf, ncontrib, fx, fy, fz);
}

template <typename R>
__global__ void kb_apply_multi(const BRep *rep, const int *list, const int *n, int Nmax, const unsigned char *contrib,
                               const double *pf, const int *ncontrib, const int *max_contrib, R *fx, R *fy, R *fz)
{
    const int r = blockIdx.x;
    if (max_contrib[r] < 2) return;
    const size_t q0 = (size_t)2 * r * Nmax;
    apply_multi_block(list + q0, n + 2 * r, 2, Nmax, contrib + q0, pf + 3 * q0, ncontrib, rep[r].serial, fx, fy, fz);
}

__global__ void kb_colloid_sum(const int *n, int Nmax, const unsigned char *contrib, const double *pf, double *cfx,
                               double *cfy, double *cfz, int *clist, int *cn)
{
    colloid_sum_block(blockIdx.x, n, Nmax, contrib, pf, cfx, cfy, cfz, clist, cn);
}

__global__ void kb_reset_contrib(const int *list, const int *n, int Nmax, const unsigned char *contrib,
                                 int *ncontrib, int *max_contrib)
{
    const int i = blockIdx.y;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n[i]; e += gridDim.x * blockDim.x) {
        size_t q = (size_t)i * Nmax + e;
        if (contrib[q]) ncontrib[list[q]] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (i & 1) == 0) max_contrib[i >> 1] = 0;
}

// compute_force_n2, colloid velocity half and RATTLE velocity correction
// (src/neighbor_list.f90:227-264, programs/single_dimer_pbc.f90:356-359,
// src/md.f90:298-319), one thread per replica
__global__ void kb_colloid_vel(int R, const BRep *rep, PView<double> c, const double *mass, Masses ms, LJDev lj,
                               double d, double dt, unsigned *err)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        PView<double> cr = shifted(c, 2 * (long long)r, 2);
        const double *e = rep[r].g.edges;
        for (int m = 0; m < 2; m++)
            force_n2_one(m, cr.pos.x, cr.pos.y, cr.pos.z, cr.species, 2, e[0], e[1], e[2], lj, cr.force.x,
                         cr.force.y, cr.force.z);
        colloid_vv_vel_one(cr, 0, mass[2 * r], dt);
        colloid_vv_vel_one(cr, 1, mass[2 * r + 1], dt);
        E3 L{{e[0], e[1], e[2]}};
        rattle_vel_dimer(cr, ms, d, L, err);
    }
}

// md_vel then change_species of every solvent particle
// (src/md.f90:219-237, programs/single_dimer_pbc.f90:511-542)
template <typename R>
__global__ void __launch_bounds__(kBT)
    kb_md_vel_species(const BTile *tiles, const BRep *rep, PView<R> v, PView<double> c, R dt, double cut_c,
                      double cut_n, double prob, const uint64_t *d_step, int step_off)
{
    const BTile t = tiles[blockIdx.x];
    const BRep &rp = rep[t.r];
    const double a[3] = {c.pos.x[2 * t.r], c.pos.y[2 * t.r], c.pos.z[2 * t.r]};
    const double b[3] = {c.pos.x[2 * t.r + 1], c.pos.y[2 * t.r + 1], c.pos.z[2 * t.r + 1]};
    const double L0 = rp.g.edges[0], L1 = rp.g.edges[1], L2 = rp.g.edges[2];
    const uint64_t step = *d_step + (uint64_t)step_off;
    const uint64_t seed = rp.seed;
    const long long off = rp.off;
    for (long long i = t.begin + threadIdx.x; i < t.end; i += blockDim.x) {
        md_vel_one(v, i, dt);
        change_species_one(v, i, i - off, a, b, L0, L1, L2, cut_c, cut_n, prob, seed, step);
    }
}

// ------------------------------------------------------ re-sort / sort

__global__ void kb_zero_slots(const BTile *tiles, const int *flag, int *count, unsigned char *is_md,
                              unsigned char *is_reac)
{
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    for (long long s = t.begin + threadIdx.x; s < t.end; s += blockDim.x) {
        count[s] = 0;
        is_md[s] = 0;
        is_reac[s] = 1;
    }
}

// apply_pbc (src/md.f90:202-217), then key = replica's first slot + the
// particle's slot, histogram with one atomic per distinct key per warp
template <typename R>
__global__ void __launch_bounds__(kBT)
    kb_pbc_key_count(const BTile *tiles, const int *flag, const BRep *rep, PView<R> v, int *key, int *count)
{
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    const BRep &rp = rep[t.r];
    const Grid g = rp.g;
    const int lane = threadIdx.x & 31;
    for (long long base = t.begin; base < t.end; base += blockDim.x) {
        long long i = base + threadIdx.x;
        bool ok = i < t.end;
        int k = -1;
        if (ok) {
            apply_pbc_one(v, i, g.edges[0], g.edges[1], g.edges[2]);
            k = rp.soff + slot_of(g, (double)v.pos.x[i], (double)v.pos.y[i], (double)v.pos.z[i]);
            key[i] = k;
        }
        unsigned peers = __match_any_sync(0xffffffffu, k);
        if (ok && lane == __ffs(peers) - 1) atomicAdd(count + k, __popc(peers));
    }
}

__device__ inline long long block_sum_ll(long long v)
{
    __shared__ long long ws[kBT / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    long long s = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kBT / 32; w++) s += ws[w];
    return s;
}

__global__ void __launch_bounds__(kBT) kb_scan_reduce(const BTile *tiles, const int *flag, const int *count,
                                                      long long *tile_sum)
{
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    long long a = 0;
    for (long long s = t.begin + threadIdx.x; s < t.end; s += blockDim.x) a += count[s];
    long long tot = block_sum_ll(a);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

// tile offsets of every active replica: its first particle + the sums of
// its earlier tiles
__global__ void kb_scan_reps(int R, const int *flag, const BRep *rep, const int *first, const int *ntiles,
                             const long long *tile_sum, long long *tile_off)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        if (flag && !flag[r]) continue;
        long long acc = rep[r].off;
        for (int k = 0; k < ntiles[r]; k++) {
            tile_off[first[r] + k] = acc;
            acc += tile_sum[first[r] + k];
        }
    }
}

// start = cursor = exclusive scan inside the tile + the tile's offset
__global__ void __launch_bounds__(kBT) kb_scan_apply(const BTile *tiles, const int *flag, const int *count,
                                                     const long long *tile_off, int *start, int *cursor)
{
    __shared__ long long ws[kBT / 32 + 1];
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    constexpr int PER = kTile / kBT;
    const long long b = t.begin + (long long)threadIdx.x * PER;
    int v[PER];
    long long sum = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        v[k] = b + k < t.end ? count[b + k] : 0;
        sum += v[k];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long inc = sum;
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) ws[w] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long acc = 0;
        for (int k = 0; k < kBT / 32; k++) {
            long long y = ws[k];
            ws[k] = acc;
            acc += y;
        }
    }
    __syncthreads();
    long long run = tile_off[blockIdx.x] + ws[w] + inc - sum;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        if (b + k < t.end) {
            start[b + k] = (int)run;
            cursor[b + k] = (int)run;
        }
        run += v[k];
    }
}

// place every particle inside its cell (in-cell order fixed by kb_segsort)
__global__ void __launch_bounds__(kBT) kb_perm(const BTile *tiles, const int *flag, const int *key, int *cursor,
                                               int *perm)
{
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    for (long long base = t.begin; base < t.end; base += blockDim.x) {
        long long i = base + threadIdx.x;
        int k = i < t.end ? key[i] : -1;
        unsigned peers = __match_any_sync(0xffffffffu, k);
        int b = 0;
        if (k >= 0 && lane == __ffs(peers) - 1) b = atomicAdd(cursor + k, __popc(peers));
        b = __shfl_sync(0xffffffffu, b, __ffs(peers) - 1);
        if (k >= 0) perm[b + __popc(peers & lt)] = (int)i;
    }
}

__global__ void kb_segsort(const BTile *tiles, const int *flag, const int *count, const int *start, int *perm,
                           int *big, int *n_big)
{
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    for (long long s = t.begin + threadIdx.x; s < t.end; s += blockDim.x) {
        int n = count[s];
        if (n <= 1) continue;
        if (n > kSmallSegmentMax) {
            int q = atomicAdd(n_big, 1);
            big[q] = (int)s;
            continue;
        }
        sort_segment(perm + start[s], n);
    }
}

template <typename R>
__global__ void __launch_bounds__(kBT)
    kb_gather(const BTile *tiles, const int *flag, PView<R> s, PView<R> d, const int *perm)
{
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    for (long long j = t.begin + threadIdx.x; j < t.end; j += blockDim.x) {
        const int i = perm[j];
        R px = s.pos.x[i], py = s.pos.y[i], pz = s.pos.z[i];
        R vx = s.vel.x[i], vy = s.vel.y[i], vz = s.vel.z[i];
        R fx = s.force.x[i], fy = s.force.y[i], fz = s.force.z[i];
        R gx = s.force_old.x[i], gy = s.force_old.y[i], gz = s.force_old.z[i];
        int ix = s.ix[i], iy = s.iy[i], iz = s.iz[i];
        int id = s.id[i], sp = s.species[i], fl = s.flags[i];
        d.pos.x[j] = px;
        d.pos.y[j] = py;
        d.pos.z[j] = pz;
        d.vel.x[j] = vx;
        d.vel.y[j] = vy;
        d.vel.z[j] = vz;
        d.force.x[j] = fx;
        d.force.y[j] = fy;
        d.force.z[j] = fz;
        d.force_old.x[j] = gx;
        d.force_old.y[j] = gy;
        d.force_old.z[j] = gz;
        d.ix[j] = ix;
        d.iy[j] = iy;
        d.iz[j] = iz;
        d.id[j] = id;
        d.species[j] = sp;
        d.flags[j] = fl;
    }
}

// the sorted arrays back into place; the gathered positions stay as pos_old
template <typename R>
__global__ void __launch_bounds__(kBT) kb_copyback(const BTile *tiles, const int *flag, PView<R> d, PView<R> s)
{
    const BTile t = tiles[blockIdx.x];
    if (!tile_active(t, flag)) return;
    for (long long j = t.begin + threadIdx.x; j < t.end; j += blockDim.x) {
        d.pos.x[j] = s.pos.x[j];
        d.pos.y[j] = s.pos.y[j];
        d.pos.z[j] = s.pos.z[j];
        d.vel.x[j] = s.vel.x[j];
        d.vel.y[j] = s.vel.y[j];
        d.vel.z[j] = s.vel.z[j];
        d.force.x[j] = s.force.x[j];
        d.force.y[j] = s.force.y[j];
        d.force.z[j] = s.force.z[j];
        d.force_old.x[j] = s.force_old.x[j];
        d.force_old.y[j] = s.force_old.y[j];
        d.force_old.z[j] = s.force_old.z[j];
        d.ix[j] = s.ix[j];
        d.iy[j] = s.iy[j];
        d.iz[j] = s.iz[j];
        d.id[j] = s.id[j];
        d.species[j] = s.species[j];
        d.flags[j] = s.flags[j];
    }
}

// apply_pbc of the colloids and pos_old = pos (one thread per replica)
__global__ void kb_colloid_resort(int R, const int *flag, const BRep *rep, PView<double> c, Vec3<double> cold)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        if (flag && !flag[r]) continue;
        const double *e = rep[r].g.edges;
        for (int k = 2 * r; k < 2 * r + 2; k++) {
            apply_pbc_one(c, k, e[0], e[1], e[2]);
            cold.x[k] = c.pos.x[k];
            cold.y[k] = c.pos.y[k];
            cold.z[k] = c.pos.z[k];
        }
    }
}

// update_list (src/neighbor_list.f90:76-157), one block per colloid
template <typename R>
__global__ void __launch_bounds__(kNlBlockThreads)
    kb_update_list(const int *flag, const BRep *rep, PView<double> c, PView<R> s, const int *count, const int *start,
                   const int *stencil, int n_stencil, double radiussq, LJDev lj, int Nmax, int *list, int *n,
                   unsigned char *is_md, unsigned char *is_reac, unsigned *err)
{
    const int i = blockIdx.x, r = i >> 1;
    if (flag && !flag[r]) return;
    const BRep &rp = rep[r];
    update_list_block<R>(i, rp.g, c.pos.x, c.pos.y, c.pos.z, c.species, s.pos.x, s.pos.y, s.pos.z, s.species,
                         count + rp.soff, start + rp.soff, stencil, n_stencil, radiussq, lj, 1, Nmax, list, n,
                         is_md + rp.soff, is_reac + rp.soff, err);
}

// ------------------------------------------------------------ interval

// random_shift (src/cell_system.f90:153-163) of every replica's grid
__global__ void kb_random_shift(int R, BRep *rep, const uint64_t *d_step, int step_off)
{
    const uint64_t step = *d_step + (uint64_t)step_off;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        double u0, u1, u2, u3;
        rng::uniform2(rep[r].seed, step, 0, rng::SHIFT, 0, u0, u1);
        rng::uniform2(rep[r].seed, step, 1, rng::SHIFT, 0, u2, u3);
        rep[r].g.origin[0] = u0 - 1;
        rep[r].g.origin[1] = u1 - 1;
        rep[r].g.origin[2] = u2 - 1;
    }
}

// simple_mpcd_step (src/mpcd.f90:71-183), one thread per slot
template <typename R>
__global__ void __launch_bounds__(kBT) kb_srd(const BTile *tiles, const BRep *rep, const int *count, const int *start,
                                              R *vx, R *vy, R *vz, const int *species, SrdParams q,
                                              const uint64_t *d_step, int step_off)
{
    const BTile t = tiles[blockIdx.x];
    const BRep &rp = rep[t.r];
    q.seed = rp.seed;
    q.step = *d_step + (uint64_t)step_off;
    for (long long s = t.begin + threadIdx.x; s < t.end; s += blockDim.x)
        srd_slot<R>(count[s], start[s], s - rp.soff, rp.off, vx, vy, vz, species, q);
}

// refuel (programs/single_dimer_pbc.f90:544-565)
template <typename R>
__global__ void __launch_bounds__(kBT) kb_refuel(const BTile *tiles, const BRep *rep, PView<R> v, PView<double> c)
{
    const BTile t = tiles[blockIdx.x];
    const BRep &rp = rep[t.r];
    const double a[3] = {c.pos.x[2 * t.r], c.pos.y[2 * t.r], c.pos.z[2 * t.r]};
    const double b[3] = {c.pos.x[2 * t.r + 1], c.pos.y[2 * t.r + 1], c.pos.z[2 * t.r + 1]};
    for (long long i = t.begin + threadIdx.x; i < t.end; i += blockDim.x)
        refuel_one(v, i, a, b, rp.g.edges[0], rp.g.edges[1], rp.g.edges[2], rp.far);
}

__global__ void kb_advance(uint64_t *d_step, uint64_t by)
{
    *d_step += by;
}

__global__ void k_add_offset(int *dst, const int *src, long long n, long long delta)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (int)(src[i] + delta);
}

// list entries are particle indices for entries e < n(i) only
__global__ void k_list_offset(int *dst, const int *src, const int *n, int points, int Nmax, long long delta)
{
    long long tot = (long long)points * Nmax;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        int i = (int)(q / Nmax), e = (int)(q % Nmax);
        dst[q] = e < n[i] ? (int)(src[q] + delta) : -1;
    }
}

// ----------------------------------------------------------- host side

using Batch = rmpcd_dimer_batch;

static int grid_cap(long long n, int bs)
{
    long long g = (n + bs - 1) / bs;
    if (g < 1) g = 1;
    if (g > 65535) g = 65535;
    return (int)g;
}

template <typename R>
static void resort_launches(Batch *b, const int *flag)
{
    cudaStream_t st = stream();
    PView<R> cur = phys<R>(b->sol, 0), alt = phys<R>(b->sol, 1);
    PView<double> cv = phys<double>(b->col, 0), ca = phys<double>(b->col, 1);
    kb_zero_slots<<<b->n_stile, kBT, 0, st>>>(b->stile, flag, b->count, b->is_md, b->is_reac);
    kb_pbc_key_count<R><<<b->n_ptile, kBT, 0, st>>>(b->ptile, flag, b->rep, cur, b->sol->key, b->count);
    kb_scan_reduce<<<b->n_stile, kBT, 0, st>>>(b->stile, flag, b->count, b->tile_sum);
    kb_scan_reps<<<grid_cap(b->R, 128), 128, 0, st>>>(b->R, flag, b->rep, b->stile_first, b->stile_count, b->tile_sum,
                                                      b->tile_off);
    kb_scan_apply<<<b->n_stile, kBT, 0, st>>>(b->stile, flag, b->count, b->tile_off, b->start, b->cursor);
    kb_perm<<<b->n_ptile, kBT, 0, st>>>(b->ptile, flag, b->sol->key, b->cursor, b->sol->perm);
    cudaMemsetAsync(b->n_big, 0, sizeof(int), st);
    kb_segsort<<<b->n_stile, kBT, 0, st>>>(b->stile, flag, b->count, b->start, b->sol->perm, b->big, b->n_big);
    launch_segsort_big(b->start, b->count, b->big, b->n_big, b->sol->perm, b->sol->key, st);
    kb_gather<R><<<b->n_ptile, kBT, 0, st>>>(b->ptile, flag, cur, alt, b->sol->perm);
    kb_copyback<R><<<b->n_ptile, kBT, 0, st>>>(b->ptile, flag, cur, alt);
    kb_colloid_resort<<<grid_cap(b->R, 128), 128, 0, st>>>(b->R, flag, b->rep, cv, ca.pos);
    kb_update_list<R><<<2 * b->R, kNlBlockThreads, 0, st>>>(
        flag, b->rep, cv, cur, b->count, b->start, b->stencil, b->n_stencil, b->prm.list_radius * b->prm.list_radius,
        b->lj_sc, b->Nmax, b->list, b->nn, b->is_md, b->is_reac, dev_error_word());
}

template <typename R>
static void md_step_launches(Batch *b, int k)
{
    cudaStream_t st = stream();
    const double dt = b->prm.tau / b->prm.N_MD;
    const double dt_sq = dt * dt / 2;
    PView<R> s = live<R>(b->sol, b->parity);
    PView<double> c = live<double>(b->col, b->parity);
    PView<R> alt = phys<R>(b->sol, 1);
    PView<double> ca = phys<double>(b->col, 1);
    kb_md_pos<R><<<b->n_ptile, kBT, 0, st>>>(b->ptile, s, alt.pos, (R)dt, (R)dt_sq, b->so_max);
    kb_colloid_pos<<<grid_cap(b->R, 128), 128, 0, st>>>(b->R, b->rep, c, ca.pos, b->rattle[0], b->rattle[1],
                                                        b->rattle[2], b->vv_mass, b->ms, b->prm.bond, dt, b->prm.skin,
                                                        b->so_max, b->resort, b->n_extra, dev_error_word());
    resort_launches<R>(b, b->resort);
    // switch_force + zero_force of both systems
    b->parity ^= 1;
    s = live<R>(b->sol, b->parity);
    c = live<double>(b->col, b->parity);
    for (int q = 0; q < 3; q++) {
        cudaMemsetAsync(s.force[q], 0, (size_t)b->Ntot * sizeof(R), st);
        cudaMemsetAsync(c.force[q], 0, (size_t)2 * b->R * sizeof(double), st);
    }
    int gx = (b->Nmax + 255) / 256;
    if (gx > 64) gx = 64;
    dim3 lg(gx, 2 * b->R);
    kb_pair_forces<R><<<lg, 256, 0, st>>>(b->rep, c, s, b->list, b->nn, b->Nmax, b->lj_sc, b->pair_f, b->pair_e,
                                          b->contrib, b->ncontrib, b->max_contrib, b->prm.cut_sq_C);
    kb_apply_single<R><<<lg, 256, 0, st>>>(b->list, b->nn, b->Nmax, b->contrib, b->pair_f, b->ncontrib, s.force.x,
                                           s.force.y, s.force.z);
    kb_apply_multi<R><<<b->R, 256, 0, st>>>(b->rep, b->list, b->nn, b->Nmax, b->contrib, b->pair_f, b->ncontrib,
                                            b->max_contrib, s.force.x, s.force.y, s.force.z);
    kb_colloid_sum<<<2 * b->R, kNlBlockThreads, 0, st>>>(b->nn, b->Nmax, b->contrib, b->pair_f, c.force.x, c.force.y,
                                                         c.force.z, b->clist, b->cn);
    kb_reset_contrib<<<lg, 256, 0, st>>>(b->list, b->nn, b->Nmax, b->contrib, b->ncontrib, b->max_contrib);
    kb_colloid_vel<<<grid_cap(b->R, 128), 128, 0, st>>>(b->R, b->rep, c, b->vv_mass, b->ms, b->lj_cc, b->prm.bond, dt,
                                                        dev_error_word());
    kb_md_vel_species<R><<<b->n_ptile, kBT, 0, st>>>(b->ptile, b->rep, s, c, (R)dt, b->prm.cut_sq_C, b->prm.cut_sq_N,
                                                     b->prm.prob, b->d_step, k);
}

template <typename R>
static void interval_launches(Batch *b)
{
    cudaStream_t st = stream();
    const int N_MD = b->prm.N_MD;
    for (int k = 0; k < N_MD; k++) md_step_launches<R>(b, k);
    kb_random_shift<<<grid_cap(b->R, 128), 128, 0, st>>>(b->R, b->rep, b->d_step, N_MD);
    resort_launches<R>(b, nullptr);
    SrdParams q{};
    q.sin_a = 1;
    q.cos_a = 0;
    q.thermostat = b->prm.thermostat ? 1 : 0;
    q.hydro = b->prm.hydro ? 1 : 0;
    q.t_factor = b->prm.thermostat ? sqrt(b->prm.T) : 0.0;
    PView<R> s = live<R>(b->sol, b->parity);
    kb_srd<R><<<b->n_stile, kBT, 0, st>>>(b->stile, b->rep, b->count, b->start, s.vel.x, s.vel.y, s.vel.z, s.species,
                                          q, b->d_step, N_MD + 1);
    kb_refuel<R><<<b->n_ptile, kBT, 0, st>>>(b->ptile, b->rep, s, live<double>(b->col, b->parity));
    kb_advance<<<1, 1, 0, st>>>(b->d_step, (uint64_t)N_MD + 2);
}

template <typename R>
static int run_t(Batch *b, int n_intervals)
{
    cudaStream_t st = stream();
    for (int it = 0; it < n_intervals; it++) {
        PhaseTimer t("batch_interval");
        if (!b->use_graph) {
            interval_launches<R>(b);
            RMPCD_CHECK_LAUNCH();
        } else {
            const int p0 = b->parity;
            if (!b->exec[p0]) {
                cudaGraph_t g = nullptr;
                RMPCD_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                interval_launches<R>(b);
                cudaError_t e = cudaStreamEndCapture(st, &g);
                if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "interval capture: %s", cudaGetErrorString(e));
                e = cudaGraphInstantiate(&b->exec[p0], g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) {
                    b->exec[p0] = nullptr;
                    return fail(RMPCD_ERR_CUDA, "interval graph: %s", cudaGetErrorString(e));
                }
            } else {
                b->parity ^= (b->prm.N_MD & 1);
            }
            RMPCD_CUDA_TRY(cudaGraphLaunch(b->exec[p0], st));
        }
        b->step += (uint64_t)b->prm.N_MD + 2;
    }
    return check_dev_error(nullptr);
}

static void free_batch(Batch *b)
{
    if (!b) return;
    cudaStreamSynchronize(stream());
    for (auto &e : b->exec)
        if (e) cudaGraphExecDestroy(e);
    rmpcd_particles_destroy(b->sol);
    rmpcd_particles_destroy(b->col);
    void *ptrs[] = {b->rep, b->ptile, b->stile, b->stile_first, b->stile_count, b->tile_sum, b->tile_off, b->count,
                    b->start, b->cursor, b->is_md, b->is_reac, b->stencil, b->list, b->nn, b->pair_f, b->pair_e,
                    b->contrib, b->ncontrib, b->max_contrib, b->clist, b->cn, b->so_max, b->resort, b->n_extra,
                    b->big, b->n_big, b->rattle[0], b->rattle[1], b->rattle[2], b->vv_mass, b->d_step};
    for (void *q : ptrs) cudaFree(q);
    for (int *l : b->luts) cudaFree(l);
    delete b;
}

template <typename T>
static int dalloc(T **p, size_t n)
{
    RMPCD_CUDA_TRY(cudaMalloc((void **)p, (n > 0 ? n : 1) * sizeof(T)));
    return RMPCD_OK;
}

static int d2d(void *dst, const void *src, size_t bytes)
{
    if (bytes) RMPCD_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream()));
    return RMPCD_OK;
}

// copy one particle system's current arrays (and pos_old) to/from the batch
// system at offset off; force/force_old follow the batch's parity
static int move_particles(Batch *b, rmpcd_particles *big, rmpcd_particles *p, long long off, bool to_batch)
{
    const size_t rs = (size_t)big->rsize, n = (size_t)p->N;
    const int bc = 0, pc = p->cur;
    for (int k = 0; k < 3; k++) {
        char *bp = (char *)big->pos[bc][k] + off * rs, *bo = (char *)big->pos[1][k] + off * rs;
        char *bv = (char *)big->vel[bc][k] + off * rs;
        char *bf = (char *)(b->parity ? big->force_old : big->force)[bc][k] + off * rs;
        char *bg = (char *)(b->parity ? big->force : big->force_old)[bc][k] + off * rs;
        int *bi = big->image[bc][k] + off;
        struct {
            void *a, *b;
            size_t bytes;
        } m[] = {{bp, p->pos[pc][k], n * rs},     {bo, p->pos[1 - pc][k], n * rs}, {bv, p->vel[pc][k], n * rs},
                 {bf, p->force[pc][k], n * rs},   {bg, p->force_old[pc][k], n * rs},
                 {bi, p->image[pc][k], n * sizeof(int)}};
        for (auto &e : m) {
            int rc = to_batch ? d2d(e.a, e.b, e.bytes) : d2d(e.b, e.a, e.bytes);
            if (rc) return rc;
        }
    }
    int *bi[3] = {big->id[bc] + off, big->species[bc] + off, big->flags[bc] + off};
    int *pi[3] = {p->id[pc], p->species[pc], p->flags[pc]};
    for (int k = 0; k < 3; k++) {
        int rc = to_batch ? d2d(bi[k], pi[k], n * sizeof(int)) : d2d(pi[k], bi[k], n * sizeof(int));
        if (rc) return rc;
    }
    if (!to_batch) {
        p->force_zero = false;
        p->force_old_zero = false;
    }
    return RMPCD_OK;
}

static int check_inputs(int R, rmpcd_particles *const *sol, rmpcd_particles *const *col, rmpcd_cells *const *cells,
                        rmpcd_nlist *const *nl, const rmpcd_rng *rngs, const rmpcd_dimer_params *prm)
{
    RMPCD_ARG(R >= 1, "dimer batch: n_replicas must be >= 1");
    RMPCD_ARG(sol && col && cells && nl && rngs && prm, "null argument");
    RMPCD_ARG(prm->N_MD >= 1 && prm->tau > 0, "dimer batch: N_MD >= 1 and tau > 0 required");
    for (int r = 0; r < R; r++) {
        if (!(sol[r] && col[r] && cells[r] && nl[r]))
            return fail(RMPCD_ERR_INVALID, "dimer batch: null handle for replica %d", r);
        RMPCD_ARG(sol[r]->precision == sol[0]->precision, "dimer batch: replicas mix solvent precisions");
        if (sol[r]->N < 1) return fail(RMPCD_ERR_INVALID, "dimer batch: replica %d has no solvent", r);
        RMPCD_ARG(col[r]->N == 2 && col[r]->precision == RMPCD_FP64, "dimer batch: colloids must be 2 FP64 beads");
        RMPCD_ARG(col[r]->n_species == col[0]->n_species &&
                      memcmp(col[r]->mass, col[0]->mass, sizeof(col[0]->mass)) == 0,
                  "dimer batch: replicas differ in colloid masses");
        RMPCD_ARG(!cells[r]->has_walls, "dimer batch: periodic boxes only");
        RMPCD_ARG(nl[r]->Npoints == 2 && nl[r]->Nmax == nl[0]->Nmax && nl[r]->stencil,
                  "dimer batch: neighbor lists must have 2 points, one capacity and a stencil");
        RMPCD_ARG(nl[r]->n_stencil == nl[0]->n_stencil, "dimer batch: replicas differ in list stencil");
        RMPCD_ARG(rngs[r].step == rngs[0].step, "dimer batch: replicas must start at the same RNG step");
    }
    return RMPCD_OK;
}

static int create(Batch **out, int R, rmpcd_particles *const *sol, rmpcd_particles *const *col,
                  rmpcd_cells *const *cells, rmpcd_nlist *const *nl, const rmpcd_rng *rngs, const rmpcd_lj *lj_sc,
                  const rmpcd_lj *lj_cc, const rmpcd_dimer_params *prm)
{
    int rc = check_inputs(R, sol, col, cells, nl, rngs, prm);
    if (rc) return rc;
    RMPCD_ARG(lj_sc && lj_cc, "null argument");
    Batch *b = new Batch();
    b->R = R;
    b->precision = sol[0]->precision;
    b->prm = *prm;
    b->step = rngs[0].step;
    b->Nmax = nl[0]->Nmax;
    b->n_stencil = nl[0]->n_stencil;
    b->lj_sc = lj_dev(lj_sc);
    b->lj_cc = lj_dev(lj_cc);
    b->ms.n = col[0]->n_species;
    for (int s = 0; s < RMPCD_MAX_SPECIES; s++) b->ms.m[s] = col[0]->mass[s];
    // replica layout and tiles
    std::vector<BTile> pt, stl;
    std::vector<int> sfirst(R), scount(R);
    std::map<std::vector<int>, int *> lut_of;
    b->rep_h.resize(R);
    long long off = 0;
    long long soff = 0;
    for (int r = 0; r < R; r++) {
        BRep &p = b->rep_h[r];
        rmpcd_cells *c = cells[r];
        p.off = off;
        p.n = sol[r]->N;
        p.soff = (int)soff;
        p.S = c->S;
        p.seed = rngs[r].seed;
        p.serial = 0;
        for (int k = 0; k < 3; k++)
            if (2 * nl[r]->max_i + 1 > c->L[k]) p.serial = 1;
        volatile float lf = (float)c->L[0] * 0.45f;
        volatile float ff = lf * lf;
        p.far = (double)ff;
        p.g = grid_of(c);
        std::vector<int> key = {c->L[0], c->L[1], c->L[2]};
        if (!lut_of.count(key)) {
            int *l = nullptr;
            if (dalloc(&l, (size_t)c->n_lut)) {
                free_batch(b);
                return RMPCD_ERR_CUDA;
            }
            b->luts.push_back(l);
            d2d(l, c->lut, (size_t)c->n_lut * sizeof(int));
            lut_of[key] = l;
        }
        p.g.lut = lut_of[key];
        for (long long t = 0; t < p.n; t += kTile) pt.push_back({r, 0, off + t, off + (t + kTile < p.n ? t + kTile : p.n)});
        sfirst[r] = (int)stl.size();
        for (long long t = 0; t < p.S; t += kTile) stl.push_back({r, 0, soff + t, soff + (t + kTile < p.S ? t + kTile : p.S)});
        scount[r] = (int)stl.size() - sfirst[r];
        off += p.n;
        soff += p.S;
    }
    if (off > 2000000000LL || soff > 2000000000LL) {
        free_batch(b);
        return fail(RMPCD_ERR_CAPACITY, "dimer batch: more than 2e9 particles or slots in total");
    }
    b->Ntot = off;
    b->Stot = (int)soff;
    b->n_ptile = (int)pt.size();
    b->n_stile = (int)stl.size();
    size_t ne = (size_t)2 * R * b->Nmax;
    bool ok = !dalloc(&b->rep, R) && !dalloc(&b->ptile, pt.size()) && !dalloc(&b->stile, stl.size()) &&
              !dalloc(&b->stile_first, R) && !dalloc(&b->stile_count, R) && !dalloc(&b->tile_sum, stl.size()) &&
              !dalloc(&b->tile_off, stl.size()) && !dalloc(&b->count, soff) && !dalloc(&b->start, soff) &&
              !dalloc(&b->cursor, soff) && !dalloc(&b->is_md, soff) && !dalloc(&b->is_reac, soff) &&
              !dalloc(&b->stencil, 3 * (size_t)b->n_stencil) && !dalloc(&b->list, ne) && !dalloc(&b->nn, 2 * (size_t)R) &&
              !dalloc(&b->pair_f, 3 * ne) && !dalloc(&b->pair_e, ne) && !dalloc(&b->contrib, ne) &&
              !dalloc(&b->ncontrib, off) && !dalloc(&b->max_contrib, R) && !dalloc(&b->clist, ne) &&
              !dalloc(&b->cn, 2 * (size_t)R) && !dalloc(&b->so_max, R) && !dalloc(&b->resort, R) &&
              !dalloc(&b->n_extra, R) && !dalloc(&b->big, soff) && !dalloc(&b->n_big, 1) &&
              !dalloc(&b->rattle[0], 2 * (size_t)R) && !dalloc(&b->rattle[1], 2 * (size_t)R) &&
              !dalloc(&b->rattle[2], 2 * (size_t)R) && !dalloc(&b->vv_mass, 2 * (size_t)R) && !dalloc(&b->d_step, 1);
    if (!ok) {
        free_batch(b);
        return RMPCD_ERR_CUDA;
    }
    if (rmpcd_particles_init(&b->sol, (int)off, sol[0]->n_species, sol[0]->mass, b->precision) ||
        rmpcd_particles_init(&b->col, 2 * R, col[0]->n_species, col[0]->mass, RMPCD_FP64)) {
        free_batch(b);
        return RMPCD_ERR_CUDA;
    }
    cudaStream_t st = stream();
    std::vector<double> vm(2 * (size_t)R);
    for (int r = 0; r < R; r++) {
        vm[2 * r] = prm->vv_mass[0];
        vm[2 * r + 1] = prm->vv_mass[1];
    }
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->rep, b->rep_h.data(), R * sizeof(BRep), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->ptile, pt.data(), pt.size() * sizeof(BTile), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->stile, stl.data(), stl.size() * sizeof(BTile), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->stile_first, sfirst.data(), R * sizeof(int), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->stile_count, scount.data(), R * sizeof(int), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->vv_mass, vm.data(), vm.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->d_step, &b->step, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->ncontrib, 0, (size_t)off * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->max_contrib, 0, (size_t)R * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->so_max, 0, (size_t)R * sizeof(unsigned long long), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->n_extra, 0, (size_t)R * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->resort, 0, (size_t)R * sizeof(int), st));
    d2d(b->stencil, nl[0]->stencil, 3 * (size_t)b->n_stencil * sizeof(int));
    for (int r = 0; r < R; r++) {
        const BRep &p = b->rep_h[r];
        if ((rc = move_particles(b, b->sol, sol[r], p.off, true)) || (rc = move_particles(b, b->col, col[r], 2 * r, true))) {
            free_batch(b);
            return rc;
        }
        rmpcd_cells *c = cells[r];
        d2d(b->count + p.soff, c->count, (size_t)p.S * sizeof(int));
        k_add_offset<<<grid_cap(p.S, 256), 256, 0, st>>>(b->start + p.soff, c->start, p.S, p.off);
        d2d(b->is_md + p.soff, c->is_md, (size_t)p.S);
        d2d(b->is_reac + p.soff, c->is_reac, (size_t)p.S);
        k_list_offset<<<grid_cap(2 * (long long)b->Nmax, 256), 256, 0, st>>>(b->list + (size_t)2 * r * b->Nmax, nl[r]->list,
                                                                          nl[r]->n, 2, b->Nmax, p.off);
        d2d(b->nn + 2 * r, nl[r]->n, 2 * sizeof(int));
    }
    rc = sync();
    if (rc) {
        free_batch(b);
        return rc;
    }
    *out = b;
    return RMPCD_OK;
}

static int scatter(Batch *b, int r, rmpcd_particles *sol, rmpcd_particles *col, rmpcd_cells *cells, rmpcd_nlist *nl,
                   rmpcd_rng *rng)
{
    RMPCD_ARG(b && r >= 0 && r < b->R, "dimer batch: replica index out of range");
    const BRep &p = b->rep_h[r];
    cudaStream_t st = stream();
    int rc;
    if (sol) {
        RMPCD_ARG(sol->N == p.n && sol->precision == b->precision, "dimer batch: solvent handle does not match");
        if ((rc = move_particles(b, b->sol, sol, p.off, false))) return rc;
    }
    if (col) {
        RMPCD_ARG(col->N == 2 && col->precision == RMPCD_FP64, "dimer batch: colloid handle does not match");
        if ((rc = move_particles(b, b->col, col, 2 * r, false))) return rc;
        if (!col->pos_rattle[0])
            for (int k = 0; k < 3; k++) RMPCD_CUDA_TRY(cudaMalloc(&col->pos_rattle[k], 2 * sizeof(double)));
        for (int k = 0; k < 3; k++) d2d(col->pos_rattle[k], b->rattle[k] + 2 * r, 2 * sizeof(double));
    }
    if (cells) {
        RMPCD_ARG(cells->S == p.S, "dimer batch: cell handle does not match");
        d2d(cells->count, b->count + p.soff, (size_t)p.S * sizeof(int));
        k_add_offset<<<grid_cap(p.S, 256), 256, 0, st>>>(cells->start, b->start + p.soff, p.S, -p.off);
        d2d(cells->is_md, b->is_md + p.soff, (size_t)p.S);
        d2d(cells->is_reac, b->is_reac + p.soff, (size_t)p.S);
        BRep now;
        RMPCD_CUDA_TRY(cudaMemcpyAsync(&now, b->rep + r, sizeof(BRep), cudaMemcpyDeviceToHost, st));
        if ((rc = sync())) return rc;
        for (int k = 0; k < 3; k++) cells->origin[k] = now.g.origin[k];
    }
    if (nl) {
        RMPCD_ARG(nl->Npoints == 2 && nl->Nmax == b->Nmax, "dimer batch: neighbor list does not match");
        k_list_offset<<<grid_cap(2 * (long long)b->Nmax, 256), 256, 0, st>>>(nl->list, b->list + (size_t)2 * r * b->Nmax,
                                                                          b->nn + 2 * r, 2, b->Nmax, -p.off);
        d2d(nl->n, b->nn + 2 * r, 2 * sizeof(int));
    }
    if (rng) rng->step = b->step;
    return sync();
}

}  // namespace rmpcd

using namespace rmpcd;

extern "C" {

int rmpcd_dimer_batch_create(rmpcd_dimer_batch **out, int n_replicas, rmpcd_particles *const *solvent,
                             rmpcd_particles *const *colloids, rmpcd_cells *const *cells,
                             rmpcd_nlist *const *nlists, const rmpcd_rng *rngs, const rmpcd_lj *solvent_colloid,
                             const rmpcd_lj *colloid_colloid, const rmpcd_dimer_params *params)
{
    RMPCD_ARG(out, "null argument");
    *out = nullptr;
    return create(out, n_replicas, solvent, colloids, cells, nlists, rngs, solvent_colloid, colloid_colloid, params);
}

int rmpcd_dimer_batch_destroy(rmpcd_dimer_batch *b)
{
    free_batch(b);
    return RMPCD_OK;
}

int rmpcd_dimer_batch_set_graph(rmpcd_dimer_batch *b, int use_graph)
{
    RMPCD_ARG(b, "null argument");
    b->use_graph = use_graph != 0;
    return RMPCD_OK;
}

int rmpcd_dimer_batch_run(rmpcd_dimer_batch *b, int n_intervals)
{
    RMPCD_ARG(b, "null argument");
    RMPCD_ARG(n_intervals >= 0, "n_intervals must be >= 0");
    if (b->precision == RMPCD_FP32) return run_t<float>(b, n_intervals);
    return run_t<double>(b, n_intervals);
}

int rmpcd_dimer_batch_scatter(rmpcd_dimer_batch *b, int replica, rmpcd_particles *solvent,
                              rmpcd_particles *colloids, rmpcd_cells *cells, rmpcd_nlist *nlist, rmpcd_rng *rng)
{
    return scatter(b, replica, solvent, colloids, cells, nlist, rng);
}

int rmpcd_dimer_batch_info(const rmpcd_dimer_batch *b, int *n_replicas, long long *n_solvent, int *n_extra_sorting)
{
    RMPCD_ARG(b, "null argument");
    if (n_replicas) *n_replicas = b->R;
    if (n_solvent) *n_solvent = b->Ntot;
    if (n_extra_sorting) {
        RMPCD_CUDA_TRY(cudaMemcpyAsync(n_extra_sorting, b->n_extra, (size_t)b->R * sizeof(int), cudaMemcpyDeviceToHost,
                                       stream()));
        return sync();
    }
    return RMPCD_OK;
}

}  // extern "C"
