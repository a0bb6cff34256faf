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
// One MD step is three kernels plus a conditional re-sort: the step-begin
// kernel (md_pos, flag roll, displacement; its last block runs every
// replica's colloid half and the program's re-sort test,
// programs/single_dimer_pbc.f90:306-330), the pair-force kernel, the kernel
// applying the pair forces, and the step-end kernel (md_vel, change_species,
// colloid velocity half).  The re-sort is decided on the device: one flag per
// replica, and in a captured graph an IF node whose body (the re-sort
// kernels, which skip the tiles of unflagged replicas) runs only when some
// replica needs it.  The re-sort gathers into the alternate buffers and
// copies back, so the arrays never change place and a whole interval (N_MD MD
// steps + shift + sort + collision + refuel) is captured once and replayed:
// the RNG step and the grid origins are read from device memory, never baked
// into the graph.
//
// Arithmetic per particle is that of the single-system kernels
// (stepops.cuh, nlist_ops.cuh), so replica r reproduces, bit for bit, the
// same program run alone through the C ABI with its own seed.
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
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

constexpr int kTile = 1024;  // slots per slot tile
constexpr int kBT = 256;     // threads per tile block

// Engine shapes (rmpcd_dimer_batch_autotune): the particles a thread of the
// step-begin / step-end kernel handles per pass, the blocks per SM they are
// compiled for, and (at run time) the particles per tile.  Every shape gives
// the same results bit for bit: tiles and passes only decide which thread
// handles which particle, and every per-particle result, the maximum
// displacement and the re-sort decision are independent of that.
template <int KB_, int KE_, int MINB_, int FIRST_>
struct BVar {
    static constexpr int KB = KB_;      // particles per thread and pass, step begin
    static constexpr int KE = KE_;      // the same, step end
    static constexpr int MINB = MINB_;  // resident blocks per SM (launch bound)
    // the colloid half of the step begin in an extra block 0 that runs while
    // the solvent streams (1), or in the block that finishes last (0)
    static constexpr bool FIRST = FIRST_ != 0;
};
template <typename R, int V>
struct BVarOf;
template <> struct BVarOf<float, 0> { using T = BVar<4, 4, 4, 0>; };
template <> struct BVarOf<float, 1> { using T = BVar<2, 4, 4, 0>; };
template <> struct BVarOf<float, 2> { using T = BVar<4, 2, 4, 0>; };
template <> struct BVarOf<float, 3> { using T = BVar<4, 16, 4, 0>; };
template <> struct BVarOf<float, 4> { using T = BVar<4, 4, 4, 1>; };
template <> struct BVarOf<double, 0> { using T = BVar<2, 4, 4, 1>; };
template <> struct BVarOf<double, 1> { using T = BVar<1, 4, 4, 1>; };
template <> struct BVarOf<double, 2> { using T = BVar<2, 2, 4, 1>; };
template <> struct BVarOf<double, 3> { using T = BVar<2, 8, 4, 1>; };
template <> struct BVarOf<double, 4> { using T = BVar<2, 4, 4, 0>; };
constexpr int kBVars = 5;
constexpr long long kPTiles[] = {256, 512, 1024, 2048, 4096};  // particles per tile
constexpr int kNPTiles = 5;
// list entries per thread of the list kernels (pair forces, their
// application, the contribution reset): their blocks per colloid are
// ceil(capacity / (256 x this)), at most 64
constexpr int kListPer[] = {1, 4};
constexpr int kNListPer = 2;
constexpr int kBShapes = kNListPer * kBVars * kNPTiles;
// shape s: particle tile kPTiles[s % kNPTiles], kernel variant
// (s / kNPTiles) % kBVars, list entries per thread kListPer[s / (kNPTiles * kBVars)]
__host__ __device__ inline int shape_tile(int s) { return s % kNPTiles; }
__host__ __device__ inline int shape_var(int s) { return (s / kNPTiles) % kBVars; }
__host__ __device__ inline int shape_list(int s) { return s / (kNPTiles * kBVars); }

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
    int cap_ptile = 0;  // particle tiles allocated (enough for the smallest tile size)
    int shape = 0;      // engine shape in use (kernel variant, particles per tile)
    int *stile_first = nullptr, *stile_count = nullptr;  // per replica
    int *ptile_first = nullptr, *ptile_count = nullptr;  // per replica
    int *act_p = nullptr, *act_s = nullptr, *n_act = nullptr;  // tiles of the replicas flagged for a re-sort
    int *all_p = nullptr, *all_s = nullptr, *n_all = nullptr;  // every tile
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
    double *co_max = nullptr;  // per replica: the colloids' displacement of this MD step
    double *csnap = nullptr;   // colloid positions at the step's force evaluation, 3 per colloid
    // whether some solvent species was negative at creation; species change
    // only to 1 or 2 inside the batch, so otherwise every particle passes
    // maximum_displacement's species >= 0 test and species need not be read
    bool read_species = true;
    int *resort = nullptr, *n_extra = nullptr, *big = nullptr, *n_big = nullptr;
    double *rattle[3] = {nullptr, nullptr, nullptr};
    double *vv_mass = nullptr;
    uint64_t *d_step = nullptr;
    uint64_t step = 0;  // host copy of every replica's RNG step
    rmpcd::Masses ms{};
    rmpcd::LJDev lj_sc{}, lj_cc{};
    int parity = 0;  // 0: force = buffer force[0], force_old = force_old[0]; swapped by each MD step
    unsigned *done = nullptr;   // blocks finished in the current step kernel (last-block hand-off)
    bool use_graph = true;
    bool capturing = false;
    cudaError_t cap_err = cudaSuccess;
    cudaStream_t body = nullptr;  // captures the bodies of the re-sort IF nodes
    cudaGraphConditionalHandle cond_next = 0;  // re-sort condition of the next MD step, while capturing
    cudaStream_t side = nullptr;   // captures the speculative force branch beside each re-sort IF node
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int *any = nullptr;  // 1 when the last MD-step beginning decided to re-sort some replica
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

// the tiles a re-sort kernel visits: tiles[ids[k]] for k < *n (every tile
// for the interval's sort, the flagged replicas' tiles for an MD step's)
struct TileSet {
    const BTile *tiles;
    const int *ids;
    const int *n;
};

// ------------------------------------------------------------ MD step
//
// Force entries that can be non-zero are known from the flags: MD set means
// the particle received a contribution in the last force evaluation (its
// `force` entry), PAST_MD in the one before (`force_old`).  Every other entry
// is exactly zero, so the MD-step kernels neither read nor clear it; the
// arithmetic uses a zero in its place and stays that of md_pos / md_vel.

__device__ inline bool same_bits(float a, float b) { return __float_as_int(a) == __float_as_int(b); }
__device__ inline bool same_bits(double a, double b) { return __double_as_longlong(a) == __double_as_longlong(b); }

template <typename R>
__device__ inline R flagged(const R *a, long long i, bool set)
{
    return set ? a[i] : (R)0;
}

// colloid position half, RATTLE and colloid displacement of replica r
// (programs/single_dimer_pbc.f90:311-322); clears the colloid force entries
// that become `force` after switch_force; returns the displacement.  Touches
// no solvent data.
__device__ inline double colloid_begin(int r, const BRep *rep, const PView<double> &c, const Vec3<double> &cold,
                                       const Vec3<double> &c_next, double *const rat[3], const double *mass,
                                       const Masses &ms, double d, double dt, unsigned *err)
{
    PView<double> cr = shifted(c, 2 * (long long)r, 2);
    for (int k = 0; k < 2; k++) {
        rat[0][2 * r + k] = cr.pos.x[k];
        rat[1][2 * r + k] = cr.pos.y[k];
        rat[2][2 * r + k] = cr.pos.z[k];
    }
    colloid_vv_pos_one(cr, 0, mass[2 * r], dt);
    colloid_vv_pos_one(cr, 1, mass[2 * r + 1], dt);
    E3 L{{rep[r].g.edges[0], rep[r].g.edges[1], rep[r].g.edges[2]}};
    rattle_pos_dimer(cr, rat[0] + 2 * r, rat[1] + 2 * r, rat[2] + 2 * r, ms, d, dt, L, err);
    Vec3<double> o = {cold.x + 2 * r, cold.y + 2 * r, cold.z + 2 * r};
    double m0 = disp_sq_one(cr.pos, o, cr.species, 0), m1 = disp_sq_one(cr.pos, o, cr.species, 1);
    for (int k = 2 * r; k < 2 * r + 2; k++) c_next.x[k] = c_next.y[k] = c_next.z[k] = 0;
    return sqrt(m0 > m1 ? m0 : m1);
}

// the re-sort decision of replica r (programs/single_dimer_pbc.f90:323-330),
// given its colloid displacement co, once the solvent's maximum displacement
// of the step is complete
__device__ inline int resort_decision(int r, double skin, double co, unsigned long long *so_max, int *resort,
                                      int *n_extra)
{
    double so = sqrt(__longlong_as_double((long long)__ldcg(so_max + r)));
    int need = (co >= skin * 0.1) || (so >= skin * 0.89);
    resort[r] = need;
    if (need) n_extra[r] += 1;
    so_max[r] = 0;
    return need;
}

struct ColloidStep {
    PView<double> c;       // colloids, force/force_old of this step
    Vec3<double> cold;     // colloid pos_old
    Vec3<double> c_next;   // colloid force entries cleared for the next evaluation
    double *rat[3];        // pos_rattle
    const double *mass;    // velocity-Verlet masses, 2 per replica
    Masses ms;
    double d, dt, skin;
    int R;
    double *co_max;        // per replica: the colloids' displacement of this step
};

// exclusive block scan of one int per thread; *total gets the block's sum
// (ws: kBT / 32 + 1 ints of shared memory)
__device__ inline int block_excl_scan(int v, int *ws, int *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) ws[w] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < kBT / 32; k++) {
            int y = ws[k];
            ws[k] = acc;
            acc += y;
        }
        ws[kBT / 32] = acc;
    }
    __syncthreads();
    int ex = ws[w] + inc - v;
    *total = ws[kBT / 32];
    __syncthreads();
    return ex;
}

// the tile lists of the replicas flagged for a re-sort
struct ResortLists {
    const int *pfirst, *pcount, *sfirst, *scount;  // per replica
    int *pids, *sids;                              // out: active particle / slot tiles
    int *n;                                        // out: n[0] particle tiles, n[1] slot tiles
};

// md_pos over the particle tile t (the solvent half of the MD step's
// beginning): returns this thread's largest squared displacement from pos_old
// among particles of species >= 0.  K particles per thread and pass, all
// loads issued before any use.
template <typename R, int K>
__device__ __forceinline__ double begin_tile(const BTile &t, const PView<R> &v, const Vec3<R> &old,
                                             const Vec3<R> &next, R dt, R dt_sq, int read_species)
{
    double m = 0;
    for (long long base = t.begin + threadIdx.x; base < t.end; base += (long long)K * blockDim.x) {
        int f[K], sp[K];
        R px[K], py[K], pz[K], vx[K], vy[K], vz[K], ox[K], oy[K], oz[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const long long i = base + (long long)k * blockDim.x;
            if (i < t.end) {
                f[k] = v.flags[i];
                sp[k] = read_species ? v.species[i] : 0;
                px[k] = v.pos.x[i];
                py[k] = v.pos.y[i];
                pz[k] = v.pos.z[i];
                vx[k] = v.vel.x[i];
                vy[k] = v.vel.y[i];
                vz[k] = v.vel.z[i];
                ox[k] = old.x[i];
                oy[k] = old.y[i];
                oz[k] = old.z[i];
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            const long long i = base + (long long)k * blockDim.x;
            if (i >= t.end) continue;
            const bool md = (f[k] >> MD_BIT) & 1, past = (f[k] >> PAST_MD_BIT) & 1;
            const R fx = flagged(v.force.x, i, md), fy = flagged(v.force.y, i, md), fz = flagged(v.force.z, i, md);
            const R qx = px[k] + dt * vx[k] + dt_sq * fx;
            const R qy = py[k] + dt * vy[k] + dt_sq * fy;
            const R qz = pz[k] + dt * vz[k] + dt_sq * fz;
            v.pos.x[i] = qx;
            v.pos.y[i] = qy;
            v.pos.z[i] = qz;
            if (past) next.x[i] = next.y[i] = next.z[i] = 0;
            if (md || past) flag_roll_one(v.flags, i);
            if (sp[k] >= 0) {
                double d0 = (double)qx - (double)ox[k], d1 = (double)qy - (double)oy[k],
                       d2 = (double)qz - (double)oz[k];
                double r = d0 * d0 + d1 * d1 + d2 * d2;
                m = m > r ? m : r;
            }
        }
    }
    return m;
}

// the block's maximum displacement (m, one value per thread) into its
// replica's so_max (r_tile < 0: a block without particles), then the
// last-block hand-off: true in the one block of the grid that finishes last
__device__ __forceinline__ bool block_done(double m, int r_tile, unsigned long long *so_max, unsigned *done,
                                           double *s_max, int *s_last)
{
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBT / 32; w++) m = m > s_max[w] ? m : s_max[w];
        // one atomic per block, skipped when it cannot raise the maximum
        if (r_tile >= 0 && m > __longlong_as_double((long long)__ldcg(so_max + r_tile)))
            atomic_max_nonneg(so_max + r_tile, m);
        __threadfence();
        *s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    return *s_last;
}

// the last block's part of an MD step's beginning: the colloid half of every
// replica unless an earlier block did it (kFirst), the re-sort decisions, the
// tile lists of the replicas to re-sort and the graph's re-sort condition
// (any_out, if given, receives whether some replica re-sorts)
template <bool kFirst>
__device__ __forceinline__ void begin_tail(const BRep *rep, unsigned long long *so_max, unsigned *done, int *resort,
                                           int *n_extra, const ColloidStep &cs, const ResortLists &rl,
                                           cudaGraphConditionalHandle cond, int use_cond, unsigned *err, int *ws,
                                           int *any_out = nullptr)
{
    __threadfence();
    int any = 0, base_p = 0, base_s = 0;
    for (int r0 = 0; r0 < cs.R; r0 += blockDim.x) {
        const int r = r0 + threadIdx.x;
        int need = 0;
        if (r < cs.R) {
            const double co = kFirst ? __ldcg(cs.co_max + r)
                                     : colloid_begin(r, rep, cs.c, cs.cold, cs.c_next, cs.rat, cs.mass, cs.ms, cs.d,
                                                     cs.dt, err);
            need = resort_decision(r, cs.skin, co, so_max, resort, n_extra);
        }
        any |= need;
        const int np = need ? rl.pcount[r] : 0, ns = need ? rl.scount[r] : 0;
        int tp, ts;
        const int ep = base_p + block_excl_scan(np, ws, &tp);
        const int es = base_s + block_excl_scan(ns, ws, &ts);
        for (int k = 0; k < np; k++) rl.pids[ep + k] = rl.pfirst[r] + k;
        for (int k = 0; k < ns; k++) rl.sids[es + k] = rl.sfirst[r] + k;
        base_p += tp;
        base_s += ts;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        rl.n[0] = base_p;
        rl.n[1] = base_s;
        if (use_cond && any) cudaGraphSetConditional(cond, 1);
        if (any_out) *any_out = any;
        *done = 0;
        __threadfence();
    }
}

// md_pos of every solvent particle, the PAST_MD/MD roll of compute_force,
// clearing of the entries that become `force` after switch_force and the
// solvent's maximum displacement (src/md.f90:61-77,
// src/neighbor_list.f90:180-188, src/particle_system.f90:357-378), one block
// per particle tile; the last block to finish takes the program's re-sort
// decision, lists the tiles of the replicas to re-sort and raises the graph's
// re-sort condition when there are any.  The colloid half of every replica
// runs either in that last block or in an extra block 0 while the solvent
// streams (V::FIRST, a choice of the engine shape: the extra block's registers
// make the FP32 streaming path spill, which costs the large FP32 batches more
// than the overlap gains, and the autotuner weighs the two).
template <typename R, typename V>
__global__ void __launch_bounds__(kBT, V::MINB)
    kb_step_begin(const BTile *tiles, const BRep *rep, PView<R> v, Vec3<R> old, Vec3<R> next, R dt, R dt_sq,
                  unsigned long long *so_max, unsigned *done, int *resort, int *n_extra, ColloidStep cs,
                  ResortLists rl, cudaGraphConditionalHandle cond, int use_cond, int read_species, unsigned *err,
                  int *any_out)
{
    __shared__ int s_last;
    __shared__ int ws[kBT / 32 + 1];
    __shared__ double s_max[kBT / 32];
    constexpr bool kFirst = V::FIRST;
    double m = 0;
    int r_tile = -1;
    if (kFirst && blockIdx.x == 0) {
        for (int r = threadIdx.x; r < cs.R; r += blockDim.x)
            cs.co_max[r] = colloid_begin(r, rep, cs.c, cs.cold, cs.c_next, cs.rat, cs.mass, cs.ms, cs.d, cs.dt, err);
    } else {
        const BTile t = tiles[blockIdx.x - (kFirst ? 1 : 0)];
        r_tile = t.r;
        m = begin_tile<R, V::KB>(t, v, old, next, dt, dt_sq, read_species);
    }
    if (!block_done(m, r_tile, so_max, done, s_max, &s_last)) return;
    begin_tail<kFirst>(rep, so_max, done, resort, n_extra, cs, rl, cond, use_cond, err, ws, any_out);
}

// list pair forces (src/neighbor_list.f90:198-219) fused with
// flag_particles_nl of the catalytic bead (programs/single_dimer_pbc.f90:493-509):
// both only read positions and species and OR bits into flags.  Block (0, i)
// also copies colloid i's position to csnap[3 i ..], the positions that the
// step's change_species uses.  skip (if given): the MD step's beginning
// decided to re-sort, so this launch is the graph's speculative one and the
// re-sort branch evaluates the forces instead.
template <typename R>
__global__ void kb_pair_forces(const BRep *rep, PView<double> c, PView<R> s, const int *list, const int *n, int Nmax,
                               LJDev lj, double *pf, double *pe, unsigned char *contrib, int *ncontrib,
                               int *max_contrib, double flag_cut_sq, double *csnap, const int *skip)
{
    if (skip && *(const volatile int *)skip) return;
    const int i = blockIdx.y;
    const int r = i >> 1;
    const int ni = n[i];
    const double x[3] = {c.pos.x[i], c.pos.y[i], c.pos.z[i]};
    if (blockIdx.x == 0 && threadIdx.x < 3) csnap[3 * i + threadIdx.x] = x[threadIdx.x];
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

// the three consumers of the pair forces, on disjoint data: solvent
// particles with one contribution, those with several (per replica, in
// order), and the colloid sums (list order in the FP64 form, a fixed tree in
// the FP32 form); skip: as kb_pair_forces
template <typename R>
__global__ void kb_apply_sum(const BRep *rep, int R_, int gx, const int *list, const int *n, int Nmax,
                             const unsigned char *contrib, const double *pf, const int *ncontrib,
                             const int *max_contrib, R *fx, R *fy, R *fz, double *cfx, double *cfy, double *cfz,
                             int *clist, int *cn, const int *skip)
{
    if (skip && *(const volatile int *)skip) return;
    const int b = blockIdx.x;
    const int n_single = gx * 2 * R_;
    if (b < n_single) {
        const int i = b / gx, bx = b % gx;
        for (int e = bx * blockDim.x + threadIdx.x; e < n[i]; e += gx * blockDim.x)
            apply_single_entry((size_t)i * Nmax + e, list, contrib, pf, ncontrib, fx, fy, fz);
    } else if (b < n_single + R_) {
        const int r = b - n_single;
        if (max_contrib[r] < 2) return;
        const size_t q0 = (size_t)2 * r * Nmax;
        apply_multi_block(list + q0, n + 2 * r, 2, Nmax, contrib + q0, pf + 3 * q0, ncontrib, rep[r].serial, fx, fy,
                          fz);
    } else if constexpr (sizeof(R) == 8) {
        colloid_sum_block(b - n_single - R_, n, Nmax, contrib, pf, cfx, cfy, cfz, clist, cn);
    } else {
        colloid_tree_block(b - n_single - R_, n, Nmax, contrib, pf, cfx, cfy, cfz);
    }
}

// the solvent half over the particle tile t of replica rp, whose colloid
// positions are a and bb; step is the random-number step of change_species
template <typename R, int K>
__device__ __forceinline__ void end_tile(const BTile &t, const BRep &rp, const PView<R> &v, const double a[3],
                                         const double bb[3], R dt, double cut_c, double cut_n, double prob,
                                         uint64_t step)
{
    const double L0 = rp.g.edges[0], L1 = rp.g.edges[1], L2 = rp.g.edges[2];
    const uint64_t seed = rp.seed;
    const long long off = rp.off;
    // The FP64 form reads every velocity: a zero-force update turns a -0
    // component into +0, as the reference's does.  The FP32 form reads
    // velocities only for particles with a force and leaves the others'
    // bits untouched, so it keeps a -0 component (an SRD rotation product
    // can round to one) where the reference would store +0: equal in
    // value, not in bits, which is why FP32 results are compared by value.
    constexpr bool kAllVel = sizeof(R) == 8;
    if constexpr (!kAllVel) {
        // FP32: only particles with a WALL, MD, PAST_MD or REAC bit do
        // anything, so the flags are read four at a time (one 16-byte
        // load; the arrays are allocated to a multiple of 4) and a group
        // of four without such a bit is skipped whole
        constexpr int kBits = (1 << WALL_BIT) | (1 << MD_BIT) | (1 << PAST_MD_BIT) | (1 << REAC_BIT);
        auto one = [&](long long i, int f) {
            if (!(f & kBits)) return;
            if (!((f >> WALL_BIT) & 1)) {
                const bool md = (f >> MD_BIT) & 1, past = (f >> PAST_MD_BIT) & 1;
                if (md || past) {
                    const R vx = v.vel.x[i], vy = v.vel.y[i], vz = v.vel.z[i];
                    R f0 = flagged(v.force.x, i, md), f1 = flagged(v.force.y, i, md),
                      f2 = flagged(v.force.z, i, md);
                    R g0 = flagged(v.force_old.x, i, past), g1 = flagged(v.force_old.y, i, past),
                      g2 = flagged(v.force_old.z, i, past);
                    v.vel.x[i] = vx + dt * (f0 + g0) / 2;
                    v.vel.y[i] = vy + dt * (f1 + g1) / 2;
                    v.vel.z[i] = vz + dt * (f2 + g2) / 2;
                }
            } else {
                v.flags[i] = f & ~(1 << WALL_BIT);
                f = f & ~(1 << WALL_BIT);
            }
            if ((f >> REAC_BIT) & 1)
                change_species_one(v, i, i - off, a, bb, L0, L1, L2, cut_c, cut_n, prob, seed, step);
        };
        const long long a4 = (t.begin + 3) & ~3LL, e4 = t.end & ~3LL;
        const long long h_end = a4 < t.end ? a4 : t.end;
        for (long long i = t.begin + threadIdx.x; i < h_end; i += blockDim.x) one(i, v.flags[i]);
        if (a4 < e4) {
            const int4 *f4 = (const int4 *)v.flags;
            constexpr int U = 4;
            for (long long q0 = a4 / 4 + threadIdx.x; q0 < e4 / 4; q0 += (long long)U * blockDim.x) {
                int4 g[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const long long q = q0 + (long long)u * blockDim.x;
                    g[u] = q < e4 / 4 ? f4[q] : make_int4(0, 0, 0, 0);
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (!((g[u].x | g[u].y | g[u].z | g[u].w) & kBits)) continue;
                    const long long i = 4 * (q0 + (long long)u * blockDim.x);
                    one(i, g[u].x);
                    one(i + 1, g[u].y);
                    one(i + 2, g[u].z);
                    one(i + 3, g[u].w);
                }
            }
        }
        const long long t_begin = e4 > h_end ? e4 : h_end;
        for (long long i = t_begin + threadIdx.x; i < t.end; i += blockDim.x) one(i, v.flags[i]);
        return;
    }
    for (long long base = t.begin + threadIdx.x; base < t.end; base += (long long)K * blockDim.x) {
      int fk[K];
      R vxk[K] = {}, vyk[K] = {}, vzk[K] = {};
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long i = base + (long long)k * blockDim.x;
        if (i < t.end) {
            fk[k] = v.flags[i];
            if (kAllVel) {
                vxk[k] = v.vel.x[i];
                vyk[k] = v.vel.y[i];
                vzk[k] = v.vel.z[i];
            }
        }
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        const long long i = base + (long long)k * blockDim.x;
        if (i >= t.end) continue;
        int f = fk[k];
        if (!kAllVel && !((f >> WALL_BIT) & 1) && (((f >> MD_BIT) & 1) || ((f >> PAST_MD_BIT) & 1))) {
            vxk[k] = v.vel.x[i];
            vyk[k] = v.vel.y[i];
            vzk[k] = v.vel.z[i];
        }
        const R vx = vxk[k], vy = vyk[k], vz = vzk[k];
        if (!((f >> WALL_BIT) & 1)) {
            const bool md = (f >> MD_BIT) & 1, past = (f >> PAST_MD_BIT) & 1;
            if (md || past) {
                R f0 = flagged(v.force.x, i, md), f1 = flagged(v.force.y, i, md), f2 = flagged(v.force.z, i, md);
                R g0 = flagged(v.force_old.x, i, past), g1 = flagged(v.force_old.y, i, past),
                  g2 = flagged(v.force_old.z, i, past);
                v.vel.x[i] = vx + dt * (f0 + g0) / 2;
                v.vel.y[i] = vy + dt * (f1 + g1) / 2;
                v.vel.z[i] = vz + dt * (f2 + g2) / 2;
            } else if (kAllVel) {
                // both forces are zero: the update changes a velocity
                // only if it is -0, so the store is kept for that case
                const R z = 0;
                const R nx = vx + dt * (z + z) / 2, ny = vy + dt * (z + z) / 2, nz = vz + dt * (z + z) / 2;
                if (!same_bits(nx, vx) || !same_bits(ny, vy) || !same_bits(nz, vz)) {
                    v.vel.x[i] = nx;
                    v.vel.y[i] = ny;
                    v.vel.z[i] = nz;
                }
            }
        } else {
            v.flags[i] = f & ~(1 << WALL_BIT);
            f = f & ~(1 << WALL_BIT);
        }
        if ((f >> REAC_BIT) & 1)
            change_species_one(v, i, i - off, a, bb, L0, L1, L2, cut_c, cut_n, prob, seed, step);
      }
    }
}

// clearing of the contribution counters over entries [bx * blockDim.x, ...)
// of list i, strided by gx blocks
__device__ __forceinline__ void end_reset(int i, int bx, int gx, const int *list, const int *n, int Nmax,
                                          const unsigned char *contrib, int *ncontrib, int *max_contrib)
{
    for (int e = bx * blockDim.x + threadIdx.x; e < n[i]; e += gx * blockDim.x) {
        size_t qq = (size_t)i * Nmax + e;
        if (contrib[qq]) ncontrib[list[qq]] = 0;
    }
    if (bx == 0 && threadIdx.x == 0 && (i & 1) == 0) max_contrib[i >> 1] = 0;
}

// compute_force_n2, the colloid velocity half and RATTLE's velocity
// correction of replica r
__device__ __forceinline__ void end_colloid(int r, const BRep *rep, const PView<double> &c, const ColloidStep &cs,
                                            const LJDev &lj_cc, unsigned *err)
{
    PView<double> cr = shifted(c, 2 * (long long)r, 2);
    const double *e = rep[r].g.edges;
    for (int m = 0; m < 2; m++)
        force_n2_one(m, cr.pos.x, cr.pos.y, cr.pos.z, cr.species, 2, e[0], e[1], e[2], lj_cc, cr.force.x,
                     cr.force.y, cr.force.z);
    colloid_vv_vel_one(cr, 0, cs.mass[2 * r], cs.dt);
    colloid_vv_vel_one(cr, 1, cs.mass[2 * r + 1], cs.dt);
    E3 L{{e[0], e[1], e[2]}};
    rattle_vel_dimer(cr, cs.ms, cs.d, L, err);
}

// md_vel then change_species of every solvent particle (src/md.f90:219-237,
// programs/single_dimer_pbc.f90:511-542), one block per particle tile;
// clearing of the per-particle contribution counters; compute_force_n2, the
// colloid velocity half and RATTLE's velocity correction per replica
// (src/neighbor_list.f90:227-264, programs/single_dimer_pbc.f90:356-359,
// src/md.f90:298-319).  The last MD step of an interval ends with this
// kernel; the others end inside kb_step_end_begin.
template <typename R, typename V>
__global__ void __launch_bounds__(kBT, V::MINB)
    kb_step_end(const BTile *tiles, int n_tiles, int gx, const BRep *rep, PView<R> v, PView<double> c, R dt,
                double cut_c, double cut_n, double prob, const uint64_t *d_step, int step_off, const int *list,
                const int *n, int Nmax, const unsigned char *contrib, int *ncontrib, int *max_contrib,
                ColloidStep cs, LJDev lj_cc, unsigned *err)
{
    const int b = blockIdx.x;
    if (b < n_tiles) {
        const BTile t = tiles[b];
        const double a[3] = {c.pos.x[2 * t.r], c.pos.y[2 * t.r], c.pos.z[2 * t.r]};
        const double bb[3] = {c.pos.x[2 * t.r + 1], c.pos.y[2 * t.r + 1], c.pos.z[2 * t.r + 1]};
        end_tile<R, V::KE>(t, rep[t.r], v, a, bb, dt, cut_c, cut_n, prob, *d_step + (uint64_t)step_off);
        return;
    }
    const int n_reset = gx * 2 * cs.R;
    if (b < n_tiles + n_reset) {
        const int q = b - n_tiles;
        end_reset(q / gx, q % gx, gx, list, n, Nmax, contrib, ncontrib, max_contrib);
        return;
    }
    for (int r = (b - n_tiles - n_reset) * blockDim.x + threadIdx.x; r < cs.R;
         r += (gridDim.x - n_tiles - n_reset) * blockDim.x)
        end_colloid(r, rep, c, cs, lj_cc, err);
}

// The arguments of the MD-step halves: the solvent view v and colloid view c
// with the force / force_old parity of the step whose forces were computed
// last, and what the halves read besides.
template <typename R>
struct StepArgs {
    const BTile *tiles;
    int n_tiles, gx;
    const BRep *rep;
    PView<R> v;
    Vec3<R> old;  // solvent pos_old
    PView<double> c;
    R dt, dt_sq;
    double cut_c, cut_n, prob;
    const uint64_t *d_step;
    const int *list, *n;
    int Nmax;
    const unsigned char *contrib;
    int *ncontrib, *max_contrib;
    const double *csnap;
    LJDev lj_cc;
    int read_species;
    unsigned *err;
};

// block b of the end of step k (RNG step offset step_off) merged with the
// beginning of step k + 1: [V::FIRST: one block for the colloids] n_tiles
// particle tiles, gx * 2R counter-clearing blocks, [without V::FIRST: n_col
// colloid velocity-half blocks].  Returns the thread's largest squared
// displacement and sets r_tile to the tile's replica (-1 for other blocks).
template <typename R, typename V>
__device__ __forceinline__ double eb_vblock(int b, int n_col, const StepArgs<R> &a, const ColloidStep &cs,
                                            int step_off, int &r_tile)
{
    constexpr bool kFirst = V::FIRST;
    const int n_reset = a.gx * 2 * cs.R;
    r_tile = -1;
    if (kFirst && b == 0) {
        for (int r = threadIdx.x; r < cs.R; r += blockDim.x) {
            end_colloid(r, a.rep, a.c, cs, a.lj_cc, a.err);
            cs.co_max[r] = colloid_begin(r, a.rep, cs.c, cs.cold, cs.c_next, cs.rat, cs.mass, cs.ms, cs.d, cs.dt,
                                         a.err);
        }
        return 0;
    }
    b -= kFirst ? 1 : 0;
    if (b < a.n_tiles) {
        const BTile t = a.tiles[b];
        const double *p = a.csnap + 6 * (size_t)t.r;
        const double ca[3] = {p[0], p[1], p[2]}, cb[3] = {p[3], p[4], p[5]};
        end_tile<R, V::KE>(t, a.rep[t.r], a.v, ca, cb, a.dt, a.cut_c, a.cut_n, a.prob,
                           *a.d_step + (uint64_t)step_off);
        // the beginning half reads what the end half wrote: velocities,
        // flags, species, force_old entries
        __syncthreads();
        r_tile = t.r;
        return begin_tile<R, V::KB>(t, a.v, a.old, a.v.force_old, a.dt, a.dt_sq, a.read_species);
    }
    if (b < a.n_tiles + n_reset) {
        const int q = b - a.n_tiles;
        end_reset(q / a.gx, q % a.gx, a.gx, a.list, a.n, a.Nmax, a.contrib, a.ncontrib, a.max_contrib);
    } else if (!kFirst) {
        for (int r = (b - a.n_tiles - n_reset) * blockDim.x + threadIdx.x; r < cs.R; r += n_col * blockDim.x)
            end_colloid(r, a.rep, a.c, cs, a.lj_cc, a.err);
    }
    return 0;
}

// The end of MD step k and the beginning of MD step k + 1 in one launch
// (no re-sort falls between them, and both halves see the same force /
// force_old parity): each particle tile's block runs the end half over its
// tile, then the beginning half; the clearing of the contribution counters
// and the colloid velocity half run in their own blocks as in kb_step_end.
// With V::FIRST, block 0 runs each replica's colloid velocity half and then
// its colloid position half (one thread per replica, in that order); without
// it the velocity halves run in the colloid blocks and the position halves in
// the last block, after every other block has finished.  change_species reads
// the colloid positions of step k from csnap (written by kb_pair_forces), as
// block 0 may already be moving the colloids.
template <typename R, typename V>
__global__ void __launch_bounds__(kBT, V::MINB)
    kb_step_end_begin(StepArgs<R> a, int step_off, unsigned long long *so_max, unsigned *done, int *resort,
                      int *n_extra, ColloidStep cs, ResortLists rl, cudaGraphConditionalHandle cond, int use_cond,
                      int *any_out)
{
    __shared__ int s_last;
    __shared__ int ws[kBT / 32 + 1];
    __shared__ double s_max[kBT / 32];
    const int n_col = V::FIRST ? 0 : (cs.R + kBT - 1) / kBT;
    int r_tile;
    const double m = eb_vblock<R, V>(blockIdx.x, n_col, a, cs, step_off, r_tile);
    if (!block_done(m, r_tile, so_max, done, s_max, &s_last)) return;
    begin_tail<V::FIRST>(a.rep, so_max, done, resort, n_extra, cs, rl, cond, use_cond, a.err, ws, any_out);
}

// ------------------------------------------------------ re-sort / sort

// count = 0, is_md = 0, is_reac = 1 over the active replicas' slots; block 0
// also clears the big-cell queue and, for the interval's sort, draws every
// replica's grid shift (random_shift, src/cell_system.f90:153-163)
__global__ void kb_zero_slots(TileSet ts, int *count, unsigned char *is_md,
                              unsigned char *is_reac, int *n_big, int R, BRep *rep, const uint64_t *d_step,
                              int shift_step_off)
{
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) *n_big = 0;
        if (shift_step_off >= 0) {
            const uint64_t step = *d_step + (uint64_t)shift_step_off;
            for (int r = threadIdx.x; r < R; r += blockDim.x) {
                double u0, u1, u2, u3;
                rng::uniform2(rep[r].seed, step, 0, rng::SHIFT, 0, u0, u1);
                rng::uniform2(rep[r].seed, step, 1, rng::SHIFT, 0, u2, u3);
                rep[r].g.origin[0] = u0 - 1;
                rep[r].g.origin[1] = u1 - 1;
                rep[r].g.origin[2] = u2 - 1;
            }
        }
    }
    for (int k = blockIdx.x; k < *ts.n; k += gridDim.x) {
        const BTile t = ts.tiles[ts.ids[k]];
        for (long long s = t.begin + threadIdx.x; s < t.end; s += blockDim.x) {
            count[s] = 0;
            is_md[s] = 0;
            is_reac[s] = 1;
        }
    }
}

// apply_pbc (src/md.f90:202-217), then key = replica's first slot + the
// particle's slot, histogram with one atomic per distinct key per warp
template <typename R>
__global__ void __launch_bounds__(kBT)
    kb_pbc_key_count(TileSet ts, const BRep *rep, PView<R> v, int *key, int *count)
{
    const int lane = threadIdx.x & 31;
    for (int kt = blockIdx.x; kt < *ts.n; kt += gridDim.x) {
        const BTile t = ts.tiles[ts.ids[kt]];
        const BRep &rp = rep[t.r];
        const Grid g = rp.g;
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

__global__ void __launch_bounds__(kBT) kb_scan_reduce(TileSet ts, const int *count, long long *tile_sum)
{
    for (int k = blockIdx.x; k < *ts.n; k += gridDim.x) {
        const int id = ts.ids[k];
        const BTile t = ts.tiles[id];
        long long a = 0;
        for (long long s = t.begin + threadIdx.x; s < t.end; s += blockDim.x) a += count[s];
        long long tot = block_sum_ll(a);
        if (threadIdx.x == 0) tile_sum[id] = tot;
        __syncthreads();
    }
}

// tile offsets of every active replica (its first particle + the sums of
// its earlier tiles); the replica's colloids get apply_pbc and pos_old = pos
__global__ void kb_scan_reps(int R, const int *flag, const BRep *rep, const int *first, const int *ntiles,
                             const long long *tile_sum, long long *tile_off, PView<double> c, Vec3<double> cold)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        if (flag && !flag[r]) continue;
        long long acc = rep[r].off;
        for (int k = 0; k < ntiles[r]; k++) {
            tile_off[first[r] + k] = acc;
            acc += tile_sum[first[r] + k];
        }
        const double *e = rep[r].g.edges;
        for (int k = 2 * r; k < 2 * r + 2; k++) {
            apply_pbc_one(c, k, e[0], e[1], e[2]);
            cold.x[k] = c.pos.x[k];
            cold.y[k] = c.pos.y[k];
            cold.z[k] = c.pos.z[k];
        }
    }
}

// start = cursor = exclusive scan inside the tile + the tile's offset
__global__ void __launch_bounds__(kBT) kb_scan_apply(TileSet ts, const int *count, const long long *tile_off,
                                                     int *start, int *cursor)
{
    __shared__ long long ws[kBT / 32 + 1];
    constexpr int PER = kTile / kBT;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int kt = blockIdx.x; kt < *ts.n; kt += gridDim.x) {
        const int id = ts.ids[kt];
        const BTile t = ts.tiles[id];
        const long long b = t.begin + (long long)threadIdx.x * PER;
        int v[PER];
        long long sum = 0;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            v[k] = b + k < t.end ? count[b + k] : 0;
            sum += v[k];
        }
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
        long long run = tile_off[id] + ws[w] + inc - sum;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            if (b + k < t.end) {
                start[b + k] = (int)run;
                cursor[b + k] = (int)run;
            }
            run += v[k];
        }
        __syncthreads();
    }
}

// place every particle inside its cell (in-cell order fixed by kb_segsort)
__global__ void __launch_bounds__(kBT) kb_perm(TileSet ts, const int *key, int *cursor, int *perm)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    for (int kt = blockIdx.x; kt < *ts.n; kt += gridDim.x) {
        const BTile t = ts.tiles[ts.ids[kt]];
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
}

__global__ void kb_segsort(TileSet ts, const int *count, const int *start, int *perm, int *big, int *n_big)
{
    for (int kt = blockIdx.x; kt < *ts.n; kt += gridDim.x) {
        const BTile t = ts.tiles[ts.ids[kt]];
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
}

template <typename R>
__global__ void __launch_bounds__(kBT) kb_gather(TileSet ts, PView<R> s, PView<R> d, const int *perm)
{
    for (int kt = blockIdx.x; kt < *ts.n; kt += gridDim.x) {
        const BTile t = ts.tiles[ts.ids[kt]];
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
}

// the sorted arrays back into place; the gathered positions stay as pos_old
template <typename R>
__global__ void __launch_bounds__(kBT) kb_copyback(TileSet ts, PView<R> d, PView<R> s)
{
    for (int kt = blockIdx.x; kt < *ts.n; kt += gridDim.x) {
        const BTile t = ts.tiles[ts.ids[kt]];
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
}

// update_list (src/neighbor_list.f90:76-157), one block per colloid; the
// candidate cells of each stencil chunk are staged in nl_stage_bytes<R>() of
// dynamic shared memory by bulk copies (a window may reach into a
// neighbouring replica's particles, which are read and not used)
template <typename R>
__global__ void __launch_bounds__(kNlBlockThreads)
    kb_update_list(const int *flag, const BRep *rep, PView<double> c, PView<R> s, const int *count, const int *start,
                   const int *stencil, int n_stencil, double radiussq, LJDev lj, int Nmax, int *list, int *n,
                   unsigned char *is_md, unsigned char *is_reac, unsigned *err)
{
    extern __shared__ __align__(16) unsigned char nl_stage[];
    __shared__ __align__(8) unsigned long long bar;
    const int i = blockIdx.x, r = i >> 1;
    if (flag && !flag[r]) return;
    const BRep &rp = rep[r];
    update_list_block<R>(i, rp.g, c.pos.x, c.pos.y, c.pos.z, c.species, s.pos.x, s.pos.y, s.pos.z, s.species,
                         count + rp.soff, start + rp.soff, stencil, n_stencil, radiussq, lj, 1, Nmax, list, n,
                         is_md + rp.soff, is_reac + rp.soff, err, NlStage{nl_stage, &bar});
}

// the list kernel's dynamic shared memory above the default limit, set once
// per precision (at batch creation, before any stream capture)
template <typename R>
static int allow_list_stage()
{
    static bool set = false;
    if (!set) {
        RMPCD_CUDA_TRY(cudaFuncSetAttribute(kb_update_list<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)nl_stage_bytes<R>()));
        set = true;
    }
    return RMPCD_OK;
}

// ------------------------------------------------------------ interval

// simple_mpcd_step (src/mpcd.f90:71-183), one thread per slot, and refuel
// (programs/single_dimer_pbc.f90:544-565), one thread per particle: the
// collision writes velocities, refuel reads positions and species only
template <typename R>
__global__ void __launch_bounds__(kBT)
    kb_srd_refuel(const BTile *stiles, int n_stiles, const BTile *ptiles, const BRep *rep, const int *count,
                  const int *start, PView<R> v, PView<double> c, SrdParams q, const uint64_t *d_step, int step_off)
{
    if ((int)blockIdx.x < n_stiles) {
        const BTile t = stiles[blockIdx.x];
        const BRep &rp = rep[t.r];
        q.seed = rp.seed;
        q.step = *d_step + (uint64_t)step_off;
        for (long long s = t.begin + threadIdx.x; s < t.end; s += blockDim.x)
            srd_slot<R>(count[s], start[s], s - rp.soff, rp.off, v.vel.x, v.vel.y, v.vel.z, v.species, q);
        return;
    }
    const BTile t = ptiles[blockIdx.x - n_stiles];
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

// grid of the re-sort kernels, which loop over their tile list
static int resort_grid(int n_tiles)
{
    int g = sm_count() * 8;
    return n_tiles < g ? (n_tiles > 0 ? n_tiles : 1) : g;
}

// the re-sort of the flagged replicas (flag = resort flags, lists = their
// tiles) or of every replica (flag = null, lists = all tiles)
template <typename R>
static void resort_launches(Batch *b, const int *flag, bool all, cudaStream_t st, int shift_step_off)
{
    PView<R> cur = phys<R>(b->sol, 0), alt = phys<R>(b->sol, 1);
    PView<double> cv = phys<double>(b->col, 0), ca = phys<double>(b->col, 1);
    TileSet pts{b->ptile, all ? b->all_p : b->act_p, all ? b->n_all : b->n_act};
    TileSet sts{b->stile, all ? b->all_s : b->act_s, (all ? b->n_all : b->n_act) + 1};
    const int gp = resort_grid(b->n_ptile), gs = resort_grid(b->n_stile);
    kb_zero_slots<<<gs, kBT, 0, st>>>(sts, b->count, b->is_md, b->is_reac, b->n_big, b->R, b->rep, b->d_step,
                                      shift_step_off);
    kb_pbc_key_count<R><<<gp, kBT, 0, st>>>(pts, b->rep, cur, b->sol->key, b->count);
    kb_scan_reduce<<<gs, kBT, 0, st>>>(sts, b->count, b->tile_sum);
    kb_scan_reps<<<grid_cap(b->R, 128), 128, 0, st>>>(b->R, flag, b->rep, b->stile_first, b->stile_count, b->tile_sum,
                                                      b->tile_off, cv, ca.pos);
    kb_scan_apply<<<gs, kBT, 0, st>>>(sts, b->count, b->tile_off, b->start, b->cursor);
    kb_perm<<<gp, kBT, 0, st>>>(pts, b->sol->key, b->cursor, b->sol->perm);
    kb_segsort<<<gs, kBT, 0, st>>>(sts, b->count, b->start, b->sol->perm, b->big, b->n_big);
    launch_segsort_big(b->start, b->count, b->big, b->n_big, b->sol->perm, b->sol->key, st);
    kb_gather<R><<<gp, kBT, 0, st>>>(pts, cur, alt, b->sol->perm);
    kb_copyback<R><<<gp, kBT, 0, st>>>(pts, cur, alt);
    kb_update_list<R><<<2 * b->R, kNlBlockThreads, nl_stage_bytes<R>(), st>>>(
        flag, b->rep, cv, cur, b->count, b->start, b->stencil, b->n_stencil, b->prm.list_radius * b->prm.list_radius,
        b->lj_sc, b->Nmax, b->list, b->nn, b->is_md, b->is_reac, dev_error_word());
}

static void note(Batch *b, cudaError_t e)
{
    if (e != cudaSuccess && b->cap_err == cudaSuccess) b->cap_err = e;
}

// blocks per colloid of the list kernels: ceil(capacity / (256 x the
// shape's list entries per thread)), at most 64
static int list_gx(const Batch *b)
{
    const int per = 256 * kListPer[shape_list(b->shape)];
    const int gx = (b->Nmax + per - 1) / per;
    return gx > 64 ? 64 : gx < 1 ? 1 : gx;
}

// the MD-step halves' arguments with force / force_old of the given parity
template <typename R>
static StepArgs<R> step_args(const Batch *b, int parity, int gx)
{
    const double dt = b->prm.tau / b->prm.N_MD;
    const double dt_sq = dt * dt / 2;
    return StepArgs<R>{b->ptile, b->n_ptile, gx, b->rep, live<R>(b->sol, parity), phys<R>(b->sol, 1).pos,
                       live<double>(b->col, parity), (R)dt, (R)dt_sq, b->prm.cut_sq_C, b->prm.cut_sq_N, b->prm.prob,
                       b->d_step, b->list, b->nn, b->Nmax, b->contrib, b->ncontrib, b->max_contrib, b->csnap,
                       b->lj_cc, b->read_species ? 1 : 0, dev_error_word()};
}

// the MD step's forces: the pair forces, then their three consumers (skip,
// if given: see kb_pair_forces)
template <typename R>
static void force_launches(Batch *b, cudaStream_t st, const int *skip)
{
    const PView<R> s = live<R>(b->sol, b->parity);
    const PView<double> c = live<double>(b->col, b->parity);
    const int gx = list_gx(b);
    kb_pair_forces<R><<<dim3(gx, 2 * b->R), 256, 0, st>>>(b->rep, c, s, b->list, b->nn, b->Nmax, b->lj_sc, b->pair_f,
                                                          b->pair_e, b->contrib, b->ncontrib, b->max_contrib,
                                                          b->prm.cut_sq_C, b->csnap, skip);
    kb_apply_sum<R><<<gx * 2 * b->R + 3 * b->R, 256, 0, st>>>(
        b->rep, b->R, gx, b->list, b->nn, b->Nmax, b->contrib, b->pair_f, b->ncontrib, b->max_contrib, s.force.x,
        s.force.y, s.force.z, c.force.x, c.force.y, c.force.z, b->clist, b->cn, skip);
}

// the program's re-sort test, as an IF node of the graph g being captured on
// st whose body (captured on `nested`) is the re-sort of the flagged
// replicas, followed by the step's forces when with_forces; cond was created
// before the kernel that sets it was captured
template <typename R>
static void capture_conditional_resort(Batch *b, cudaStream_t st, cudaGraph_t g, cudaGraphConditionalHandle cond,
                                       cudaStream_t nested, bool with_forces)
{
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    note(b, cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    note(b, cudaGraphAddNode(&node, g, deps, nd, &cp));
    if (b->cap_err != cudaSuccess) return;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    note(b, cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    note(b, cudaStreamBeginCaptureToGraph(nested, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    resort_launches<R>(b, b->resort, false, nested, -1);
    if (with_forces) force_launches<R>(b, nested, nullptr);
    cudaGraph_t out = nullptr;
    note(b, cudaStreamEndCapture(nested, &out));
}

// a fresh IF-node handle in the graph being captured on st (0 when not
// capturing)
static cudaGraphConditionalHandle new_cond(Batch *b, cudaStream_t st)
{
    cudaGraphConditionalHandle cond = 0;
    if (b->capturing) {
        cudaStreamCaptureStatus st_cap;
        cudaGraph_t g = nullptr;
        note(b, cudaStreamGetCaptureInfo(st, &st_cap, nullptr, &g, nullptr, nullptr));
        note(b, cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    }
    return cond;
}

// MD step k of the interval: its beginning (for k = 0; later steps begin in
// the previous step's kb_step_end_begin), the re-sort test, the forces and
// its end, merged with the beginning of step k + 1 unless k is the last
template <typename R, typename V>
static void md_step_launches(Batch *b, int k)
{
    cudaStream_t st = stream();
    const double dt = b->prm.tau / b->prm.N_MD;
    const double dt_sq = dt * dt / 2;
    PView<R> s = live<R>(b->sol, b->parity);
    PView<double> c = live<double>(b->col, b->parity);
    PView<R> alt = phys<R>(b->sol, 1);
    PView<double> ca = phys<double>(b->col, 1);
    ColloidStep cs{c, ca.pos, c.force_old, {b->rattle[0], b->rattle[1], b->rattle[2]}, b->vv_mass, b->ms,
                   b->prm.bond, dt, b->prm.skin, b->R, b->co_max};
    const ResortLists rl{b->ptile_first, b->ptile_count, b->stile_first, b->stile_count, b->act_p, b->act_s, b->n_act};
    const int use_cond = b->capturing ? 1 : 0, read_species = b->read_species ? 1 : 0;
    cudaGraphConditionalHandle cond = b->cond_next;
    if (k == 0) {
        cond = new_cond(b, st);
        kb_step_begin<R, V><<<b->n_ptile + (V::FIRST ? 1 : 0), kBT, 0, st>>>(
            b->ptile, b->rep, s, alt.pos, s.force_old, (R)dt, (R)dt_sq, b->so_max, b->done, b->resort, b->n_extra,
            cs, rl, cond, use_cond, read_species, dev_error_word(), b->any);
    }
    // switch_force: the cleared entries become `force` (the re-sort does not
    // read the force buffers)
    b->parity ^= 1;
    s = live<R>(b->sol, b->parity);
    c = live<double>(b->col, b->parity);
    cs.c = c;
    cs.c_next = c.force_old;
    const int gx = list_gx(b);
    if (b->capturing) {
        // the re-sort test as an IF node whose body re-sorts and then
        // evaluates the forces, beside a branch that evaluates them at once
        // unless the beginning decided to re-sort: the IF node's latency then
        // overlaps the forces of every step without a re-sort
        note(b, cudaEventRecord(b->ev_fork, st));
        note(b, cudaStreamWaitEvent(b->side, b->ev_fork, 0));
        cudaStreamCaptureStatus st_cap;
        cudaGraph_t g = nullptr;
        note(b, cudaStreamGetCaptureInfo(st, &st_cap, nullptr, &g, nullptr, nullptr));
        capture_conditional_resort<R>(b, st, g, cond, b->body, true);
        force_launches<R>(b, b->side, b->any);
        note(b, cudaEventRecord(b->ev_join, b->side));
        note(b, cudaStreamWaitEvent(st, b->ev_join, 0));
    } else {
        resort_launches<R>(b, b->resort, false, st, -1);
        force_launches<R>(b, st, nullptr);
    }
    const int n_col_blocks = (b->R + kBT - 1) / kBT;
    const int n_reset = gx * 2 * b->R;
    if (k + 1 < b->prm.N_MD) {
        b->cond_next = new_cond(b, st);
        kb_step_end_begin<R, V><<<(V::FIRST ? 1 : n_col_blocks) + b->n_ptile + n_reset, kBT, 0, st>>>(
            step_args<R>(b, b->parity, gx), k, b->so_max, b->done, b->resort, b->n_extra, cs, rl, b->cond_next,
            use_cond, b->any);
    } else {
        b->cond_next = 0;
        kb_step_end<R, V><<<b->n_ptile + n_reset + n_col_blocks, kBT, 0, st>>>(
            b->ptile, b->n_ptile, gx, b->rep, s, c, (R)dt, b->prm.cut_sq_C, b->prm.cut_sq_N, b->prm.prob, b->d_step,
            k, b->list, b->nn, b->Nmax, b->contrib, b->ncontrib, b->max_contrib, cs, b->lj_cc, dev_error_word());
    }
}

template <typename R, int Var>
static void md_steps(Batch *b)
{
    for (int k = 0; k < b->prm.N_MD; k++) md_step_launches<R, typename BVarOf<R, Var>::T>(b, k);
}

template <typename R>
static void interval_launches(Batch *b)
{
    cudaStream_t st = stream();
    const int N_MD = b->prm.N_MD;
    switch (shape_var(b->shape)) {
    case 1: md_steps<R, 1>(b); break;
    case 2: md_steps<R, 2>(b); break;
    case 3: md_steps<R, 3>(b); break;
    case 4: md_steps<R, 4>(b); break;
    default: md_steps<R, 0>(b); break;
    }
    resort_launches<R>(b, nullptr, true, st, N_MD);
    SrdParams q{};
    q.sin_a = 1;
    q.cos_a = 0;
    q.thermostat = b->prm.thermostat ? 1 : 0;
    q.hydro = b->prm.hydro ? 1 : 0;
    q.t_factor = b->prm.thermostat ? sqrt(b->prm.T) : 0.0;
    kb_srd_refuel<R><<<b->n_stile + b->n_ptile, kBT, 0, st>>>(b->stile, b->n_stile, b->ptile, b->rep, b->count, b->start,
                                                              live<R>(b->sol, b->parity), live<double>(b->col, b->parity),
                                                              q, b->d_step, N_MD + 1);
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
                b->cap_err = cudaSuccess;
                RMPCD_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                b->capturing = true;
                interval_launches<R>(b);
                b->capturing = false;
                cudaError_t e = cudaStreamEndCapture(st, &g);
                if (e == cudaSuccess && b->cap_err != cudaSuccess) e = b->cap_err;
                if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec[p0], g, 0);
                if (g) cudaGraphDestroy(g);
                if (e != cudaSuccess) {
                    b->exec[p0] = nullptr;
                    b->parity = p0;
                    cudaGetLastError();
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
    if (b->body) cudaStreamDestroy(b->body);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    rmpcd_particles_destroy(b->sol);
    rmpcd_particles_destroy(b->col);
    void *ptrs[] = {b->rep, b->ptile, b->stile, b->stile_first, b->stile_count, b->tile_sum, b->tile_off, b->count,
                    b->start, b->cursor, b->is_md, b->is_reac, b->stencil, b->list, b->nn, b->pair_f, b->pair_e,
                    b->contrib, b->ncontrib, b->max_contrib, b->clist, b->cn, b->so_max, b->co_max, b->csnap, b->resort,
                    b->n_extra,
                    b->big, b->n_big, b->rattle[0], b->rattle[1], b->rattle[2], b->vv_mass, b->d_step, b->done,
                    b->ptile_first, b->ptile_count, b->act_p, b->act_s, b->n_act, b->all_p, b->all_s, b->n_all,
                    b->any};
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

// *out = 1 if some a[i] < 0
__global__ void k_any_negative(const int *a, long long n, int *out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (a[i] < 0) {
            *out = 1;
            return;
        }
}

// the particle tiles of every replica at `ptile` particles per tile: tile
// list, each replica's first tile and count, and the every-tile id list
static int build_particle_tiles(Batch *b, long long ptile)
{
    std::vector<BTile> pt;
    std::vector<int> pfirst(b->R), pcount(b->R);
    for (int r = 0; r < b->R; r++) {
        const BRep &p = b->rep_h[r];
        pfirst[r] = (int)pt.size();
        for (long long t = 0; t < p.n; t += ptile)
            pt.push_back({r, 0, p.off + t, p.off + (t + ptile < p.n ? t + ptile : p.n)});
        pcount[r] = (int)pt.size() - pfirst[r];
    }
    if ((long long)pt.size() > b->cap_ptile)
        return fail(RMPCD_ERR_CAPACITY, "dimer batch: %zu particle tiles above the %d allocated", pt.size(),
                    b->cap_ptile);
    cudaStream_t st = stream();
    std::vector<int> ids(pt.size());
    for (size_t k = 0; k < ids.size(); k++) ids[k] = (int)k;
    const int n = (int)pt.size();
    if (n) {
        RMPCD_CUDA_TRY(cudaMemcpyAsync(b->ptile, pt.data(), pt.size() * sizeof(BTile), cudaMemcpyHostToDevice, st));
        RMPCD_CUDA_TRY(cudaMemcpyAsync(b->all_p, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->ptile_first, pfirst.data(), b->R * sizeof(int), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->ptile_count, pcount.data(), b->R * sizeof(int), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->n_all, &n, sizeof(int), cudaMemcpyHostToDevice, st));
    // the host vectors go out of scope: wait for the copies that read them
    RMPCD_CUDA_TRY(cudaStreamSynchronize(st));
    b->n_ptile = n;
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
    // default shape: variant 0 and 1024-particle tiles, smaller only for
    // batches too small to give ~2 tiles per SM: each tile's block is one
    // round trip to DRAM, so fewer, fuller tiles beat more blocks (one 32^3
    // dimer: 1024-particle tiles take the MD step from 45.8 to 38.0 us against
    // 256-particle ones); rmpcd_dimer_batch_autotune times the others
    long long n_total = 0;
    for (int r = 0; r < R; r++) n_total += sol[r]->N;
    int tile_k = 2;  // kPTiles[2] = 1024
    while (tile_k > 0 && n_total / kPTiles[tile_k] < 2LL * sm_count()) tile_k--;
    b->shape = tile_k;
    long long cap_p = 0;
    for (int r = 0; r < R; r++) cap_p += (sol[r]->N + kPTiles[0] - 1) / kPTiles[0];
    if (cap_p < 1) cap_p = 1;
    std::vector<BTile> stl;
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
    b->cap_ptile = (int)cap_p;
    b->n_stile = (int)stl.size();
    size_t ne = (size_t)2 * R * b->Nmax;
    bool ok = !dalloc(&b->rep, R) && !dalloc(&b->ptile, cap_p) && !dalloc(&b->stile, stl.size()) &&
              !dalloc(&b->stile_first, R) && !dalloc(&b->stile_count, R) && !dalloc(&b->tile_sum, stl.size()) &&
              !dalloc(&b->tile_off, stl.size()) && !dalloc(&b->count, soff) && !dalloc(&b->start, soff) &&
              !dalloc(&b->cursor, soff) && !dalloc(&b->is_md, soff) && !dalloc(&b->is_reac, soff) &&
              !dalloc(&b->stencil, 3 * (size_t)b->n_stencil) && !dalloc(&b->list, ne) && !dalloc(&b->nn, 2 * (size_t)R) &&
              !dalloc(&b->pair_f, 3 * ne) && !dalloc(&b->pair_e, ne) && !dalloc(&b->contrib, ne) &&
              !dalloc(&b->ncontrib, off) && !dalloc(&b->max_contrib, R) && !dalloc(&b->clist, ne) &&
              !dalloc(&b->cn, 2 * (size_t)R) && !dalloc(&b->so_max, R) && !dalloc(&b->co_max, R) &&
              !dalloc(&b->csnap, 6 * (size_t)R) && !dalloc(&b->resort, R) &&
              !dalloc(&b->n_extra, R) && !dalloc(&b->big, soff) && !dalloc(&b->n_big, 1) &&
              !dalloc(&b->rattle[0], 2 * (size_t)R) && !dalloc(&b->rattle[1], 2 * (size_t)R) &&
              !dalloc(&b->rattle[2], 2 * (size_t)R) && !dalloc(&b->vv_mass, 2 * (size_t)R) && !dalloc(&b->d_step, 1) &&
              !dalloc(&b->done, 1) && cudaStreamCreateWithFlags(&b->body, cudaStreamNonBlocking) == cudaSuccess &&
              !dalloc(&b->any, 1) &&
              cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) == cudaSuccess &&
              !dalloc(&b->ptile_first, R) && !dalloc(&b->ptile_count, R) && !dalloc(&b->act_p, cap_p) &&
              !dalloc(&b->act_s, stl.size()) && !dalloc(&b->n_act, 2) && !dalloc(&b->all_p, cap_p) &&
              !dalloc(&b->all_s, stl.size()) && !dalloc(&b->n_all, 2);
    if (!ok) {
        free_batch(b);
        return RMPCD_ERR_CUDA;
    }
    if (rmpcd_particles_init(&b->sol, (int)off, sol[0]->n_species, sol[0]->mass, b->precision) ||
        rmpcd_particles_init(&b->col, 2 * R, col[0]->n_species, col[0]->mass, RMPCD_FP64)) {
        free_batch(b);
        return RMPCD_ERR_CUDA;
    }
    if ((b->precision == RMPCD_FP32 ? allow_list_stage<float>() : allow_list_stage<double>()) != RMPCD_OK) {
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
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->stile, stl.data(), stl.size() * sizeof(BTile), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->stile_first, sfirst.data(), R * sizeof(int), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->stile_count, scount.data(), R * sizeof(int), cudaMemcpyHostToDevice, st));
    std::vector<int> ids_s(stl.size());
    for (size_t k = 0; k < ids_s.size(); k++) ids_s[k] = (int)k;
    const int n_all[2] = {0, (int)stl.size()}, n_none[2] = {0, 0};
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->all_s, ids_s.data(), ids_s.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->n_all, n_all, sizeof(n_all), cudaMemcpyHostToDevice, st));
    {
        int rc = build_particle_tiles(b, kPTiles[shape_tile(b->shape)]);
        if (rc) {
            free_batch(b);
            return rc;
        }
    }
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->n_act, n_none, sizeof(n_none), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->vv_mass, vm.data(), vm.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(b->d_step, &b->step, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->ncontrib, 0, (size_t)off * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->max_contrib, 0, (size_t)R * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->so_max, 0, (size_t)R * sizeof(unsigned long long), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->n_extra, 0, (size_t)R * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->resort, 0, (size_t)R * sizeof(int), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->done, 0, sizeof(unsigned), st));
    RMPCD_CUDA_TRY(cudaMemsetAsync(b->any, 0, sizeof(int), st));
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
    {
        int *neg = nullptr, h_neg = 1;
        if (cudaMalloc(&neg, sizeof(int)) == cudaSuccess && cudaMemsetAsync(neg, 0, sizeof(int), st) == cudaSuccess) {
            k_any_negative<<<grid_cap(b->sol->N, 256), 256, 0, st>>>(b->sol->species[0], b->sol->N, neg);
            if (cudaMemcpyAsync(&h_neg, neg, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) h_neg = 1;
        }
        rc = sync();
        cudaFree(neg);
        b->read_species = h_neg != 0;
    }
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

// shape in use <- s: kernel variant and particle tiles; the captured interval
// graphs hold the old launches and are dropped (captured again on the next run)
static int set_shape(Batch *b, int s)
{
    RMPCD_CUDA_TRY(cudaStreamSynchronize(stream()));
    int rc = build_particle_tiles(b, kPTiles[shape_tile(s)]);
    if (rc) return rc;
    for (auto &e : b->exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
    b->shape = s;
    return RMPCD_OK;
}

// chosen shapes per GPU, precision, N_MD and mix of boxes (batches on
// different host threads may tune at once: the map is guarded)
static std::map<std::string, int> g_batch_tuned;
static std::mutex g_batch_tuned_mu;

static bool tuned_lookup(const std::string &key, int *shape)
{
    std::lock_guard<std::mutex> lk(g_batch_tuned_mu);
    auto hit = g_batch_tuned.find(key);
    if (hit == g_batch_tuned.end()) return false;
    *shape = hit->second;
    return true;
}

static std::string tune_key(const Batch *b)
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::map<std::vector<int>, int> mix;
    for (const BRep &p : b->rep_h) mix[{p.g.L[0], p.g.L[1], p.g.L[2]}]++;
    std::string k = std::to_string(dev) + ":" + std::to_string(b->precision) + ":" + std::to_string(b->prm.N_MD);
    for (auto &m : mix)
        k += ":" + std::to_string(m.first[0]) + "x" + std::to_string(m.first[1]) + "x" + std::to_string(m.first[2]) +
             "*" + std::to_string(m.second);
    return k;
}

static int run_any(Batch *b, int n)
{
    if (b->precision == RMPCD_FP32) return run_t<float>(b, n);
    return run_t<double>(b, n);
}

static int autotune(Batch *b, int n_intervals, int *best, float *ms, int *ran)
{
    *ran = 0;
    const std::string key = tune_key(b);
    int remembered = 0;
    if (tuned_lookup(key, &remembered)) {
        *best = remembered;
        if (ms)
            for (int k = 0; k < kBShapes; k++) ms[k] = -1.0f;
        return set_shape(b, remembered);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    RMPCD_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(RMPCD_ERR_CUDA, "dimer batch autotune: event creation failed");
    }
    int rc = RMPCD_OK, b_best = b->shape;
    float best_ms = 0;
    if (ms)
        for (int k = 0; k < kBShapes; k++) ms[k] = -1.0f;
    // every tile size and kernel variant with one list entry per thread,
    // then the best of them with each other list setting
    std::vector<int> order;
    for (int k = 0; k < kNPTiles * kBVars; k++) order.push_back(k);
    for (size_t oi = 0; !rc; oi++) {
        if (oi == (size_t)kNPTiles * kBVars && order.size() == oi)
            for (int m = 1; m < kNListPer; m++) order.push_back(b_best + m * kNPTiles * kBVars);
        if (oi >= order.size()) break;
        const int k = order[oi];
        rc = set_shape(b, k);
        // one interval captures the shape's graph and warms it up; then the
        // timed ones
        if (!rc) rc = run_any(b, 1);
        if (!rc && cudaEventRecord(e0, stream()) != cudaSuccess) rc = fail(RMPCD_ERR_CUDA, "event record");
        if (!rc) rc = run_any(b, n_intervals);
        if (!rc && cudaEventRecord(e1, stream()) != cudaSuccess) rc = fail(RMPCD_ERR_CUDA, "event record");
        float t = 0;
        if (!rc && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
            rc = fail(RMPCD_ERR_CUDA, "dimer batch autotune: event timing failed");
        if (rc) break;
        *ran += 1 + n_intervals;
        t /= (float)n_intervals;
        if (ms) ms[k] = t;
        if (oi == 0 || t < best_ms) {
            best_ms = t;
            b_best = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(g_batch_tuned_mu);
        g_batch_tuned[key] = b_best;
    }
    *best = b_best;
    return set_shape(b, b_best);
}

}  // namespace rmpcd

using namespace rmpcd;

extern "C" {

int rmpcd_dimer_batch_shapes(int precision, int *n_shapes)
{
    RMPCD_ARG(n_shapes, "null argument");
    RMPCD_ARG(precision == RMPCD_FP32 || precision == RMPCD_FP64, "precision must be RMPCD_FP32 or RMPCD_FP64");
    *n_shapes = kBShapes;
    return RMPCD_OK;
}

int rmpcd_dimer_batch_shape_info(int precision, int shape, int *particles_per_tile, int *per_thread_begin,
                                 int *per_thread_end, int *blocks_per_sm, int *list_entries_per_thread,
                                 int *colloid_block_first)
{
    RMPCD_ARG(precision == RMPCD_FP32 || precision == RMPCD_FP64, "precision must be RMPCD_FP32 or RMPCD_FP64");
    RMPCD_ARG(shape >= 0 && shape < kBShapes, "no such engine shape");
    int kb, ke, mb;
    bool cf;
    const int v = shape_var(shape);
    if (precision == RMPCD_FP32) {
        using V0 = BVarOf<float, 0>::T;
        using V1 = BVarOf<float, 1>::T;
        using V2 = BVarOf<float, 2>::T;
        using V3 = BVarOf<float, 3>::T;
        using V4 = BVarOf<float, 4>::T;
        kb = v == 0 ? V0::KB : v == 1 ? V1::KB : v == 2 ? V2::KB : v == 3 ? V3::KB : V4::KB;
        ke = v == 0 ? V0::KE : v == 1 ? V1::KE : v == 2 ? V2::KE : v == 3 ? V3::KE : V4::KE;
        mb = v == 0 ? V0::MINB : v == 1 ? V1::MINB : v == 2 ? V2::MINB : v == 3 ? V3::MINB : V4::MINB;
        cf = v == 0 ? V0::FIRST : v == 1 ? V1::FIRST : v == 2 ? V2::FIRST : v == 3 ? V3::FIRST : V4::FIRST;
    } else {
        using V0 = BVarOf<double, 0>::T;
        using V1 = BVarOf<double, 1>::T;
        using V2 = BVarOf<double, 2>::T;
        using V3 = BVarOf<double, 3>::T;
        using V4 = BVarOf<double, 4>::T;
        kb = v == 0 ? V0::KB : v == 1 ? V1::KB : v == 2 ? V2::KB : v == 3 ? V3::KB : V4::KB;
        ke = v == 0 ? V0::KE : v == 1 ? V1::KE : v == 2 ? V2::KE : v == 3 ? V3::KE : V4::KE;
        mb = v == 0 ? V0::MINB : v == 1 ? V1::MINB : v == 2 ? V2::MINB : v == 3 ? V3::MINB : V4::MINB;
        cf = v == 0 ? V0::FIRST : v == 1 ? V1::FIRST : v == 2 ? V2::FIRST : v == 3 ? V3::FIRST : V4::FIRST;
    }
    if (particles_per_tile) *particles_per_tile = (int)kPTiles[shape_tile(shape)];
    if (list_entries_per_thread) *list_entries_per_thread = kListPer[shape_list(shape)];
    if (colloid_block_first) *colloid_block_first = cf ? 1 : 0;
    if (per_thread_begin) *per_thread_begin = kb;
    if (per_thread_end) *per_thread_end = ke;
    if (blocks_per_sm) *blocks_per_sm = mb;
    return RMPCD_OK;
}

int rmpcd_dimer_batch_set_shape(rmpcd_dimer_batch *b, int shape)
{
    RMPCD_ARG(b, "null argument");
    RMPCD_ARG(shape >= 0 && shape < kBShapes, "no such engine shape");
    return set_shape(b, shape);
}

int rmpcd_dimer_batch_get_shape(const rmpcd_dimer_batch *b, int *shape)
{
    RMPCD_ARG(b && shape, "null argument");
    *shape = b->shape;
    return RMPCD_OK;
}

int rmpcd_dimer_batch_autotune(rmpcd_dimer_batch *b, int n_intervals, int *best, float *ms_per_interval,
                               int *intervals_run)
{
    RMPCD_ARG(b && best && intervals_run, "null argument");
    RMPCD_ARG(n_intervals >= 1, "n_intervals must be >= 1");
    return autotune(b, n_intervals, best, ms_per_interval, intervals_run);
}

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
