// The main loops of programs/n_colloids_pbc.f90 (:221-276 thermalisation,
// :304-324 production) as one native call: passive LJ colloids in an SRD
// fluid with lazy, cell-wise solvent streaming.  The loop performs the
// program's steps in the program's order, so the results are those of the
// module entry points called one by one (rmpcdmd_b200.programs.NColloidsPBC
// .interval does exactly that); it differs in how the work is issued:
//   * the MD cells (is_md) are listed once per neighbor-list update, and the
//     per-MD-step cell_md_pos / cell_md_vel / cell_maximum_displacement run
//     over that list instead of over every slot;
//   * zero_force of the solvent and the PAST_MD/MD roll of compute_force are
//     one pass that clears only the force entries that can be non-zero
//     (particles with MD or PAST_MD set: every other entry is exactly zero),
//     over all N for the first two MD steps after a sort and over the MD
//     cells after that;
//   * the re-sort test of an MD step (its two displacement maxima against
//     the skin) runs on the device in the host's double arithmetic and
//     writes its decision to page-locked mapped host memory;
//   * an MD step without energies is one replayed CUDA graph, captured once
//     per set of buffers it touches (the sort and the force switch exchange
//     buffers): the part up to the re-sort test, then the part after it
//     (flag roll, forces) with every kernel gated by the device's decision.
//     The host reads the decision as soon as the kernel writes it, while the
//     forces run; on a step that re-sorts the gated kernels return at once
//     and the host issues the sort, then the forces.
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "keys.cuh"
#include "nlist_ops.cuh"
#include "rmpcd_common.cuh"
#include "sortcore.cuh"
#include "state.cuh"
#include "stepops.cuh"
#include "timers.cuh"

namespace rmpcd {

// the is_md slots, in any order (one atomic per warp)
__global__ void k_md_slot_list(const unsigned char *is_md, int S, int *list, int *n_list)
{
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < S; base += (long long)gridDim.x * blockDim.x) {
        const long long s = base + threadIdx.x;
        const bool md = s < S && is_md[s];
        const unsigned bal = __ballot_sync(0xffffffffu, md);
        int b = 0;
        if (lane == 0 && bal) b = atomicAdd(n_list, __popc(bal));
        b = __shfl_sync(0xffffffffu, b, 0);
        if (md) list[b + __popc(bal & ((1u << lane) - 1u))] = (int)s;
    }
}

constexpr int kLanesPerCell = 8;

// In this program a solvent particle with neither MD nor PAST_MD set has zero
// force and force_old: compute_force writes a force only together with the
// MD bit, the roll moves MD to PAST_MD as the force moves to force_old, and
// entries are cleared when both bits go.  So the force arrays are read only
// for flagged particles and a zero takes their place otherwise; the
// arithmetic is that of md_pos / md_vel with the zero entry, bit for bit.
constexpr int kForceFlags = (1 << MD_BIT) | (1 << PAST_MD_BIT);

// md_pos of one particle (src/md.f90:61-77 form): its new position, from
// the velocity before md_vel (flags f), for the caller to store
template <typename R>
__device__ inline void moved_pos(const PView<R> &v, long long i, int f, R dt, R dt_sq, R &x, R &y, R &z)
{
    R fx = 0, fy = 0, fz = 0;
    if (f & kForceFlags) {
        fx = v.force.x[i];
        fy = v.force.y[i];
        fz = v.force.z[i];
    }
    x = v.pos.x[i] + dt * v.vel.x[i] + dt_sq * fx;
    y = v.pos.y[i] + dt * v.vel.y[i] + dt_sq * fy;
    z = v.pos.z[i] + dt * v.vel.z[i] + dt_sq * fz;
}

// md_vel of one particle (src/md.f90:219-237 form).  The FP32 form skips the
// update of a particle without forces: its velocity keeps its value (a -0
// component stays -0 where the reference's update stores +0, as in the
// replica engine's FP32 step), and its 12 bytes are not written again.
template <typename R>
__device__ inline void stream_vel_gated(const PView<R> &v, long long i, int f, R dt)
{
    if (!((f >> WALL_BIT) & 1)) {
        if constexpr (sizeof(R) == 4) {
            if (!(f & kForceFlags)) return;
        }
        R fx = 0, fy = 0, fz = 0, ox = 0, oy = 0, oz = 0;
        if (f & kForceFlags) {
            fx = v.force.x[i];
            fy = v.force.y[i];
            fz = v.force.z[i];
            ox = v.force_old.x[i];
            oy = v.force_old.y[i];
            oz = v.force_old.z[i];
        }
        v.vel.x[i] = v.vel.x[i] + dt * (fx + ox) / 2;
        v.vel.y[i] = v.vel.y[i] + dt * (fy + oy) / 2;
        v.vel.z[i] = v.vel.z[i] + dt * (fz + oz) / 2;
    } else {
        v.flags[i] = f & ~(1 << WALL_BIT);
    }
}

// The catch-up of cell_md_pos then cell_md_vel with md_flag = .false.
// (src/md.f90:79-102, :239-263) for every particle outside the MD cells
// (cellmap: each particle's slot, from the last sort), fused with the key
// pass of the sort that follows (apply_pbc, the slot in the cells' grid and
// its count, as k_pbc_key_count): one linear pass, the streamed position kept
// in registers and written once with its wrap.  Per particle the arithmetic
// is the catch-up's (the position step reading the velocity before its
// update) followed by the key pass's.
template <typename R>
__global__ void k_catch_up_key_count(const int *__restrict__ cellmap, const unsigned char *__restrict__ is_md, int N,
                                     PView<R> v, R dt, R dt_sq, Grid g, double e0, double e1, double e2,
                                     int *__restrict__ key, int *__restrict__ count)
{
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < N; base += stride) {
        const long long i = base + threadIdx.x;
        const bool ok = i < N;
        int slot = -1;
        if (ok) {
            R x, y, z;
            const bool catch_up = !is_md[cellmap[i]];
            if (catch_up) {
                const int f = v.flags[i];
                moved_pos(v, i, f, dt, dt_sq, x, y, z);
                stream_vel_gated(v, i, f, dt);
            } else {
                x = v.pos.x[i];
                y = v.pos.y[i];
                z = v.pos.z[i];
            }
            const int jx = floor_div_edge((double)x, e0), jy = floor_div_edge((double)y, e1),
                      jz = floor_div_edge((double)z, e2);
            if (jx) {
                v.ix[i] += jx;
                x = x - (R)(jx * e0);
            }
            if (jy) {
                v.iy[i] += jy;
                y = y - (R)(jy * e1);
            }
            if (jz) {
                v.iz[i] += jz;
                z = z - (R)(jz * e2);
            }
            if (catch_up || jx) v.pos.x[i] = x;
            if (catch_up || jy) v.pos.y[i] = y;
            if (catch_up || jz) v.pos.z[i] = z;
            slot = slot_of(g, (double)x, (double)y, (double)z);
            key[i] = slot;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, slot);
        if (ok && lane == __ffs(peers) - 1) atomicAdd(count + slot, __popc(peers));
    }
}

// cellmap[i] = the slot of particle i of the sorted arrays
__global__ void k_fill_cellmap(const int *count, const int *start, int S, int *cellmap)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < (long long)S * kLanesPerCell;
         q += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(q / kLanesPerCell), g = (int)(q % kLanesPerCell);
        for (int i = start[s] + g; i < start[s] + count[s]; i += kLanesPerCell) cellmap[i] = s;
    }
}

// cell_md_pos with md_flag = .true. (src/md.f90:79-102) over the listed MD
// cells, eight lanes per cell, fused with cell_maximum_displacement over the
// same cells (src/particle_system.f90:380-410): each new position is measured
// against pos_old as it is written (the value that is stored); the squared
// maximum goes to *out.  kVel: the previous MD step's cell_md_vel
// (src/md.f90:239-263) runs first, particle by particle (nothing changes the
// flags or forces between the two)
template <typename R, bool kVel>
__global__ void k_md_cells_pos_disp(const int *list, const int *n_list, const int *count, const int *start,
                                    PView<R> v, Vec3<R> old, R dt, R dt_sq, unsigned long long *out)
{
    const long long n = (long long)*n_list * kLanesPerCell;
    double m = 0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int s = list[q / kLanesPerCell], g = (int)(q % kLanesPerCell);
        const int a = start[s], c = count[s];
        for (int i = a + g; i < a + c; i += kLanesPerCell) {
            const int f = v.flags[i];
            if (kVel) stream_vel_gated(v, i, f, dt);
            R x, y, z;
            moved_pos(v, i, f, dt, dt_sq, x, y, z);
            v.pos.x[i] = x;
            v.pos.y[i] = y;
            v.pos.z[i] = z;
            if (v.species[i] >= 0) {
                const double d0 = (double)x - (double)old.x[i];
                const double d1 = (double)y - (double)old.y[i];
                const double d2 = (double)z - (double)old.z[i];
                const double r = d0 * d0 + d1 * d1 + d2 * d2;
                m = m > r ? m : r;
            }
        }
    }
    warp_max_into(out, m);
}

// cell_md_vel with md_flag = .true. (src/md.f90:239-263) over the listed MD
// cells, eight lanes per cell

template <typename R>
__global__ void k_md_cells_vel(const int *list, const int *n_list, const int *count, const int *start, PView<R> v,
                               R dt)
{
    const long long n = (long long)*n_list * kLanesPerCell;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int s = list[q / kLanesPerCell], g = (int)(q % kLanesPerCell);
        const int a = start[s], c = count[s];
        for (int i = a + g; i < a + c; i += kLanesPerCell) stream_vel_gated(v, i, v.flags[i], dt);
    }
}

// pos_old = pos over the listed cells: inside the loop only the MD cells'
// pos_old is read (cell_maximum_displacement) before the next sort rewrites
// the buffer
template <typename R>
__global__ void k_md_cells_copy_pos(const int *list, const int *n_list, const int *count, const int *start,
                                    Vec3<R> pos, Vec3<R> old)
{
    const long long n = (long long)*n_list * kLanesPerCell;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int s = list[q / kLanesPerCell], g = (int)(q % kLanesPerCell);
        const int a = start[s], c = count[s];
        for (int i = a + g; i < a + c; i += kLanesPerCell) {
            old.x[i] = pos.x[i];
            old.y[i] = pos.y[i];
            old.z[i] = pos.z[i];
        }
    }
}

// zero_force of the colloids (the entries that the step's compute_force and
// compute_force_n2 accumulate into), done by the first threads of the solvent
// roll that starts the step's force part
__device__ inline void zero_colloid_force(const Vec3<double> &cf, int nc)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nc; q += gridDim.x * blockDim.x) {
        cf.x[q] = 0;
        cf.y[q] = 0;
        cf.z[q] = 0;
    }
}

// the roll + clear below restricted to the listed MD cells.  Between two
// sorts the list is fixed and compute_force flags only list entries, which
// lie in MD cells; so once two rolls have run over every particle after a
// sort (the first turns flags carried through the sort into PAST_MD, the
// second clears them), no particle outside the MD cells has MD or PAST_MD
// set or a non-zero force entry, and rolling the MD cells alone gives the
// same flags and forces as rolling all N.
template <typename R>
__global__ void k_md_cells_roll_clear(const int *list, const int *n_list, const int *count, const int *start,
                                      int *flags, Vec3<R> force, Vec3<double> cf, int nc, const int *gate)
{
    if (gate && *gate) return;
    zero_colloid_force(cf, nc);
    const long long n = (long long)*n_list * kLanesPerCell;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int s = list[q / kLanesPerCell], g = (int)(q % kLanesPerCell);
        const int a = start[s], c = count[s];
        for (int i = a + g; i < a + c; i += kLanesPerCell) {
            const int f = flags[i];
            if (f & ((1 << MD_BIT) | (1 << PAST_MD_BIT))) {
                force.x[i] = 0;
                force.y[i] = 0;
                force.z[i] = 0;
                flag_roll_one(flags, i);
            }
        }
    }
}

// zero_force of the solvent fused with the PAST_MD/MD roll: only entries of
// particles with MD or PAST_MD set can be non-zero
template <typename R>
__global__ void k_roll_clear(int *flags, Vec3<R> force, long long N, Vec3<double> cf, int nc, const int *gate)
{
    if (gate && *gate) return;
    zero_colloid_force(cf, nc);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int f = flags[i];
        if (f & ((1 << MD_BIT) | (1 << PAST_MD_BIT))) {
            force.x[i] = 0;
            force.y[i] = 0;
            force.z[i] = 0;
            flag_roll_one(flags, i);
        }
    }
}

// The program's re-sort test (programs/n_colloids_pbc.f90:230-231) on the
// device, in the host's double arithmetic: ctl[0] counts the MD steps since
// the last sort (delta_t = dt * ctl[0]), ctl[1] receives the decision and
// ctl[2] counts the tests; the host's mapped word h_ctl[0] gets count * 2 +
// decision in one store, so the host that sees the count sees its decision.  The
// maxima are the squared displacements taken by the MD step's position pass
// (solvent, floored at max_v * delta_t) and of the colloids.
__device__ inline void nc_resort_test(unsigned long long *so_bits, double co_sq, int *ctl, int *h_ctl, double dt,
                                      double max_v, double skin)
{
    const int n = ctl[0] + 1;
    ctl[0] = n;
    const double delta_t = __dmul_rn(dt, (double)n);
    const double a = sqrt(__longlong_as_double((long long)*so_bits));
    const double b = __dmul_rn(max_v, delta_t);
    const double so_max = a > b ? a : b;
    const double co_max = sqrt(co_sq);
    const int resort = (co_max >= __dmul_rn(skin, 0.1)) || (so_max >= __dmul_rn(skin, 0.9)) ? 1 : 0;
    ctl[1] = resort;
    const int seq = ctl[2] + 1;
    ctl[2] = seq;
    ((volatile int *)h_ctl)[0] = seq * 2 + resort;
    *so_bits = 0;  // cleared for the next MD step's position pass
}

// The colloid part of an MD step up to the re-sort test, one block: the
// previous MD step's velocity half when due, the position half (the colloid
// velocity Verlet of programs/n_colloids_pbc.f90:222-224, :248-249), the
// colloids' largest displacement since the last sort (maximum_displacement,
// src/particle_system.f90:357-378; a maximum, so the same in any order), then
// the re-sort test.  Each colloid's updates are those of rmpcd_colloid_vv_vel
// and rmpcd_colloid_vv_pos, which touch no other colloid.
constexpr int kNcColloidThreads = 256;

template <bool kVel>
__global__ void __launch_bounds__(kNcColloidThreads)
    k_nc_colloid_begin(PView<double> c, Vec3<double> c_old, double mass, double dt,
                       unsigned long long *so_bits, int *ctl, int *h_ctl, double max_v, double skin)
{
    __shared__ double s_m[kNcColloidThreads / 32];
    double m = 0;
    for (int i = threadIdx.x; i < c.N; i += blockDim.x) {
        if (kVel) colloid_vv_vel_one(c, i, mass, dt);
        colloid_vv_pos_one(c, i, mass, dt);
        const double r = disp_sq_one(c.pos, c_old, c.species, i);
        m = m > r ? m : r;
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kNcColloidThreads / 32; w++) m = m > s_m[w] ? m : s_m[w];
        nc_resort_test(so_bits, m, ctl, h_ctl, dt, max_v, skin);
    }
}

__global__ void k_nc_set_since(int *ctl, int since)
{
    ctl[0] = since;
    ctl[1] = 0;
    ctl[2] = 0;
}

struct NcLoop {
    rmpcd_particles *s, *c;
    rmpcd_cells *cells;
    rmpcd_nlist *nl;
    const rmpcd_lj *lj_sc, *lj_cc;
    rmpcd_rng *rng;
    const rmpcd_ncolloids_params *prm;
    rmpcd_ncolloids_state *st;
    std::vector<double> vv_mass;
    double dt;
    int *md_list = nullptr;  // is_md slots
    int *cellmap = nullptr;  // slot of every solvent particle (set by each sort)
    int *n_md = nullptr;     // their number (device)
    int *ctl = nullptr;      // device: MD steps since the last sort, re-sort decision, test count
    int *h_ctl = nullptr;    // page-locked, device-mapped word: test count * 2 + decision (written by the kernel)
    int *h_ctl_dev = nullptr;  // its device address
    // second stream of the force evaluation (colloid sums and colloid-colloid
    // forces beside the solvent force application)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int full_rolls = 2;  // rolls over all N still due since the last sort
    // replayed parts of an MD step, keyed by the buffers they use: part_a up
    // to the re-sort test, part_b the forces, and step = part_a then part_b
    // gated by the test's decision (the key's last entry: vel_due + 2 full)
    using Key = std::tuple<const void *, const void *, const void *, int>;
    std::map<Key, cudaGraphExec_t> part_a, part_b, step;
    bool graphs = false;
    unsigned seq = 0;  // re-sort tests issued in this call
    cudaEvent_t ev_step = nullptr;  // end of the last step graph
    // what the captured graphs depend on besides their keys (see nc_signature)
    std::vector<unsigned long long> sig;

    ~NcLoop()
    {
        for (auto &kv : part_a) cudaGraphExecDestroy(kv.second);
        for (auto &kv : part_b) cudaGraphExecDestroy(kv.second);
        for (auto &kv : step) cudaGraphExecDestroy(kv.second);
        cudaFree(md_list);
        cudaFree(n_md);
        cudaFree(cellmap);
        cudaFree(ctl);
        if (h_ctl) cudaFreeHost(h_ctl);
        if (ev_step) cudaEventDestroy(ev_step);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
    }
};

// Everything a captured MD-step graph bakes in besides the buffers of its key:
// the device, the handles and every device array of theirs that a graph can touch, the
// sizes, the box, max_v, the LJ tables (passed by value to the kernels) and
// the step parameters (tau, N_MD, skin and the colloid mass).  The loop's scratch and graphs are kept for the next
// call while this is unchanged.
static std::vector<unsigned long long> nc_signature(const rmpcd_particles *s, const rmpcd_particles *c,
                                                     const rmpcd_cells *cells, const rmpcd_nlist *nl,
                                                     const rmpcd_lj *lj_sc, const rmpcd_lj *lj_cc,
                                                     const rmpcd_ncolloids_params *prm)
{
    std::vector<unsigned long long> v;
    int dev = -1;
    cudaGetDevice(&dev);
    v.push_back((unsigned long long)dev);
    auto add = [&](const void *p) { v.push_back((unsigned long long)(uintptr_t)p); };
    auto num = [&](double x) {
        unsigned long long b;
        memcpy(&b, &x, 8);
        v.push_back(b);
    };
    auto bytes = [&](const void *p, size_t n) {
        for (size_t o = 0; o < n; o += 8) {
            unsigned long long b = 0;
            memcpy(&b, (const char *)p + o, n - o < 8 ? n - o : 8);
            v.push_back(b);
        }
    };
    for (const rmpcd_particles *p : {s, c}) {
        add(p);
        v.push_back((unsigned long long)p->N);
        v.push_back((unsigned long long)p->precision);
        for (int b = 0; b < 2; b++) {
            for (int k = 0; k < 3; k++) {
                add(p->pos[b][k]);
                add(p->vel[b][k]);
                add(p->force[b][k]);
                add(p->force_old[b][k]);
                add(p->image[b][k]);
            }
            add(p->id[b]);
            add(p->species[b]);
            add(p->flags[b]);
        }
        add(p->d_max);
    }
    add(cells);
    v.push_back((unsigned long long)cells->S);
    for (int k = 0; k < 3; k++) num(cells->edges[k]);
    num(cells->max_v);
    add(cells->count);
    add(cells->start);
    add(cells->is_md);
    add(cells->is_reac);
    add(nl);
    v.push_back((unsigned long long)nl->Npoints);
    v.push_back((unsigned long long)nl->Nmax);
    v.push_back((unsigned long long)nl->max_i);
    for (int k = 0; k < 3; k++) v.push_back((unsigned long long)nl->box_cells[k]);
    add(nl->list);
    add(nl->n);
    add(nl->pair_f);
    add(nl->pair_e);
    add(nl->contrib);
    add(nl->ncontrib);
    add(nl->d_status);
    add(nl->mkeys);
    add(nl->e_pre);
    const LJDev a = lj_dev(lj_sc), b = lj_dev(lj_cc);
    bytes(&a, sizeof a);
    bytes(&b, sizeof b);
    num(prm->tau);
    v.push_back((unsigned long long)prm->N_MD);
    num(prm->skin);
    num(prm->mass);
    return v;
}

// scratch, events and the second stream of a loop
static int nc_alloc(NcLoop &L, int S, int N)
{
    if (cudaMalloc(&L.md_list, (size_t)(S > 0 ? S : 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&L.n_md, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&L.cellmap, (size_t)(N > 0 ? N : 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&L.ctl, 3 * sizeof(int)) != cudaSuccess ||
        cudaHostAlloc(&L.h_ctl, 2 * sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&L.h_ctl_dev, L.h_ctl, 0) != cudaSuccess ||
        cudaEventCreateWithFlags(&L.ev_step, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&L.ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&L.ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&L.side, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return fail(RMPCD_ERR_CUDA, "rmpcd_ncolloids_run: allocation failed");
    }
    return RMPCD_OK;
}

// run issue() once under stream capture the first time `key` is seen, then
// replay the instantiated graph
template <typename F>
static int replay(std::map<NcLoop::Key, cudaGraphExec_t> &cache, const NcLoop::Key &key, F issue)
{
    cudaStream_t st = stream();
    auto it = cache.find(key);
    if (it == cache.end()) {
        RMPCD_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int rc = issue();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "n_colloids step capture: %s", cudaGetErrorString(e));
        cudaGraphExec_t x = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess)
            return fail(RMPCD_ERR_CUDA, "n_colloids step instantiate: %s", cudaGetErrorString(ei));
        it = cache.emplace(key, x).first;
    }
    RMPCD_CUDA_TRY(cudaGraphLaunch(it->second, st));
    return RMPCD_OK;
}

// fixed grid of the MD-cell kernels (their item count is on the device)
static inline int md_cells_grid() { return sm_count() * 16; }

// list the MD cells after a neighbor-list update
static int list_md_cells(NcLoop &L)
{
    cudaStream_t st = stream();
    RMPCD_CUDA_TRY(cudaMemsetAsync(L.n_md, 0, sizeof(int), st));
    k_md_slot_list<<<grid_for(L.cells->S, 256), 256, 0, st>>>(L.cells->is_md, L.cells->S, L.md_list, L.n_md);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

// cell_md_pos over the MD cells, after the previous MD step's cell_md_vel
// when that is due, and their maximum displacement (into the solvent's d_max,
// zero on entry: cleared when the loop starts and by each re-sort test)
template <typename R>
static int md_cells_pos_disp_t(NcLoop &L, bool vel_due)
{
    cudaStream_t st = stream();
    const R dt = (R)L.dt, dt_sq = (R)(L.dt * L.dt / 2);
    const PView<R> v = cur<R>(L.s);
    const Vec3<R> old = alt<R>(L.s).pos;
    if (vel_due)
        k_md_cells_pos_disp<R, true><<<md_cells_grid(), 256, 0, st>>>(L.md_list, L.n_md, L.cells->count,
                                                                     L.cells->start, v, old, dt, dt_sq, L.s->d_max);
    else
        k_md_cells_pos_disp<R, false><<<md_cells_grid(), 256, 0, st>>>(L.md_list, L.n_md, L.cells->count,
                                                                      L.cells->start, v, old, dt, dt_sq, L.s->d_max);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

template <typename R>
static int md_cells_vel_t(NcLoop &L)
{
    k_md_cells_vel<R><<<md_cells_grid(), 256, 0, stream()>>>(L.md_list, L.n_md, L.cells->count,
                                                                       L.cells->start, cur<R>(L.s), (R)L.dt);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

template <typename R>
static int roll_clear_t(NcLoop &L, const int *gate)
{
    PView<R> v = cur<R>(L.s);
    const Vec3<double> cf = cur<double>(L.c).force;
    const int nc = L.c->N;
    if (L.full_rolls > 0) {
        const long long n = L.s->N > nc ? L.s->N : nc;
        k_roll_clear<R><<<grid_for(n > 0 ? n : 1, 256), 256, 0, stream()>>>(v.flags, v.force, L.s->N, cf, nc, gate);
        L.full_rolls--;
    } else {
        k_md_cells_roll_clear<R><<<md_cells_grid(), 256, 0, stream()>>>(L.md_list, L.n_md, L.cells->count,
                                                                        L.cells->start, v.flags, v.force, cf, nc,
                                                                        gate);
    }
    RMPCD_CHECK_LAUNCH();
    L.c->force_zero = true;
    return RMPCD_OK;
}

// the particles outside the MD cells caught up over dtl, and every particle
// keyed and counted for the sort (k_catch_up_key_count)
template <typename R>
static int catch_up_key_t(NcLoop &L, double dtl)
{
    const double dt_sq = dtl * dtl / 2;
    rmpcd_cells *c = L.cells;
    cudaStream_t st = stream();
    RMPCD_CUDA_TRY(cudaMemsetAsync(c->count, 0, (size_t)c->S * sizeof(int), st));
    if (L.s->N > 0)
        k_catch_up_key_count<R><<<grid_for(L.s->N, 256), 256, 0, st>>>(
            L.cellmap, c->is_md, L.s->N, cur<R>(L.s), (R)dtl, (R)dt_sq, grid_of(c), c->edges[0], c->edges[1],
            c->edges[2], L.s->key, c->count);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

template <typename R>
static int md_cells_copy_pos_t(NcLoop &L)
{
    PView<R> a = cur<R>(L.s), b = alt<R>(L.s);
    k_md_cells_copy_pos<R><<<md_cells_grid(), 256, 0, stream()>>>(L.md_list, L.n_md, L.cells->count,
                                                                  L.cells->start, a.pos, b.pos);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

#define NC_DISPATCH(L, fn) ((L).s->precision == RMPCD_FP32 ? fn<float>(L) : fn<double>(L))

// the colloid part of the MD step and the re-sort test (the solvent's
// maximum displacement over the MD cells was taken with its positions), whose
// kernel also writes the decision to the host
static int colloid_begin(NcLoop &L, bool vel_due)
{
    cudaStream_t st = stream();
    const PView<double> c = cur<double>(L.c);
    const Vec3<double> c_old = alt<double>(L.c).pos;
    if (vel_due)
        k_nc_colloid_begin<true><<<1, kNcColloidThreads, 0, st>>>(c, c_old, L.prm->mass, L.dt, L.s->d_max, L.ctl,
                                                                  L.h_ctl_dev, L.cells->max_v, L.prm->skin);
    else
        k_nc_colloid_begin<false><<<1, kNcColloidThreads, 0, st>>>(c, c_old, L.prm->mass, L.dt, L.s->d_max, L.ctl,
                                                                   L.h_ctl_dev, L.cells->max_v, L.prm->skin);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

// the re-sort decision of the MD step, after a synchronisation of the stream
static int read_resort(NcLoop &L, bool *resort)
{
    const int rc = sync();
    if (rc) return rc;
    *resort = (((volatile int *)L.h_ctl)[0] & 1) != 0;
    return RMPCD_OK;
}

// the re-sort decision of test number seq, read from the mapped copy as soon
// as the kernel has written it, while the rest of the step graph runs; the
// step graph's end event bounds the wait (once it has completed, the decision
// is there or the step failed)
static int wait_resort(NcLoop &L, unsigned seq, bool *resort)
{
    volatile int *h = (volatile int *)L.h_ctl;
    for (unsigned long it = 1;; it++) {
        const unsigned w = (unsigned)h[0];
        if ((w >> 1) == seq) {
            *resort = (w & 1u) != 0;
            return RMPCD_OK;
        }
        if ((it & 1023ul) == 0) {
            const cudaError_t e = cudaEventQuery(L.ev_step);
            if (e == cudaSuccess) {
                if (((unsigned)h[0] >> 1) == seq) continue;
                return fail(RMPCD_ERR_CUDA, "n_colloids step: re-sort decision %u missing after its step", seq);
            }
            if (e != cudaErrorNotReady) return fail(RMPCD_ERR_CUDA, "n_colloids step: %s", cudaGetErrorString(e));
        }
    }
}

// stream the non-MD cells over the time since the last sort, wrap, sort,
// rebuild the list (programs/n_colloids_pbc.f90:230-241).  The solvent's
// pos_old is copied for the MD cells only, except on the call's last sort
// (after which the caller may read any of it).
static int catch_up_and_sort(NcLoop &L, bool full_pos_old)
{
    const double dtl = (L.st->t - L.st->last_sort) * L.dt;
    int rc = L.s->precision == RMPCD_FP32 ? catch_up_key_t<float>(L, dtl) : catch_up_key_t<double>(L, dtl);
    if (!rc) rc = rmpcd_apply_pbc(L.c, L.cells->edges);
    if (!rc) rc = sort_keyed_flagged(L.cells, L.s, L.cellmap);  // the solvent's wrap and keys are done
    L.st->last_sort = L.st->t;
    if (!rc && cudaMemsetAsync(L.ctl, 0, sizeof(int), stream()) != cudaSuccess)
        rc = fail(RMPCD_ERR_CUDA, "n_colloids sort: step counter reset failed");
    L.full_rolls = 2;
    if (!rc) rc = rmpcd_nlist_update(L.nl, L.c, L.s, L.prm->list_radius, L.cells, nullptr);
    if (!rc) rc = list_md_cells(L);
    if (!rc) rc = full_pos_old ? rmpcd_particles_copy_pos_old(L.s) : NC_DISPATCH(L, md_cells_copy_pos_t);
    if (!rc) rc = rmpcd_particles_copy_pos_old(L.c);
    return rc;
}

// md_loop up to the displacement maxima (programs/n_colloids_pbc.f90:221-229)
// (vel_due: the previous MD step's velocity halves, of the solvent's MD cells
// and of the colloids, run first)
static int issue_part_a(NcLoop &L, bool vel_due)
{
    int rc = L.s->precision == RMPCD_FP32 ? md_cells_pos_disp_t<float>(L, vel_due)
                                          : md_cells_pos_disp_t<double>(L, vel_due);
    if (!rc) rc = colloid_begin(L, vel_due);
    return rc;
}

// md_loop after the re-sort test (programs/n_colloids_pbc.f90:243-254) up to
// the velocity halves, the force switch done; energies only when asked for
// (they synchronise).  The velocity halves run with the next MD step's
// position pass, or in vel_tail after the interval's last MD step.  gate
// (without energies): a device word that, when non-zero, makes every kernel
// of the part return at once.
static int issue_part_b(NcLoop &L, double *e1, double *e2, const int *gate = nullptr)
{
    // zero_force of the colloids included in the roll
    int rc = L.s->precision == RMPCD_FP32 ? roll_clear_t<float>(L, gate) : roll_clear_t<double>(L, gate);
    if (!e1 && !e2) {
        const ForceN2Branch n2{L.lj_cc, L.side, L.ev_fork, L.ev_join, gate};
        if (!rc) rc = compute_force_impl(L.c, L.s, L.nl, L.cells->edges, L.lj_sc, nullptr, false, &n2);
        return rc;
    }
    if (!rc) rc = compute_force_impl(L.c, L.s, L.nl, L.cells->edges, L.lj_sc, e1, false);
    if (!rc) rc = rmpcd_compute_force_n2(L.c, L.cells->edges, L.lj_cc, e2);
    return rc;
}

// the velocity halves of the interval's last MD step
static int vel_tail(NcLoop &L)
{
    int rc = NC_DISPATCH(L, md_cells_vel_t);
    if (!rc) rc = rmpcd_colloid_vv_vel(L.c, L.dt, L.vv_mass.data());
    return rc;
}

// md_loop after the re-sort (programs/n_colloids_pbc.f90:243-254): the force
// switch, then part_b (replayed, or issued with the energies when asked for)
static int md_step_forces(NcLoop &L, bool want_energy)
{
    int rc = rmpcd_particles_switch_force(L.s);
    if (!rc) rc = rmpcd_particles_switch_force(L.c);
    if (rc) return rc;
    if (L.graphs && !want_energy) {
        // the roll over all N or over the MD cells is part of the key; the
        // host-side bookkeeping of the captured calls is redone after a replay
        const int full = L.full_rolls > 0;
        const NcLoop::Key kb{L.s->pos[L.s->cur][0], L.s->force[L.s->cur][0], L.c->force[L.c->cur][0], full};
        const int before = L.full_rolls;
        rc = replay(L.part_b, kb, [&] { return issue_part_b(L, nullptr, nullptr); });
        L.full_rolls = before > 0 ? before - 1 : 0;
        L.s->force_zero = false;
        L.c->force_zero = false;
        return rc;
    }
    double e1 = 0, e2 = 0;
    rc = issue_part_b(L, want_energy ? &e1 : nullptr, want_energy ? &e2 : nullptr);
    if (!rc && want_energy) {
        L.st->e1 = e1;
        L.st->e2 = e2;
    }
    return rc;
}

// one pass of md_loop (programs/n_colloids_pbc.f90:221-254); vel_due: the
// previous MD step's velocity halves are still to run (every step of an
// interval but its first)
static int md_step(NcLoop &L, bool want_energy, bool vel_due)
{
    L.st->t += 1;
    const unsigned seq = ++L.seq;
    int rc;
    if (L.graphs && !want_energy) {
        // the whole MD step as one graph: part_a, then part_b gated by the
        // step's re-sort decision, which the host reads from mapped memory
        // while the forces run; on a step that re-sorts the gated part does
        // nothing and the host issues the sort, then the forces
        const int before = L.full_rolls;
        const bool fz[4] = {L.s->force_zero, L.s->force_old_zero, L.c->force_zero, L.c->force_old_zero};
        const NcLoop::Key ks{L.s->pos[L.s->cur][0], L.s->force[L.s->cur][0], L.c->force[L.c->cur][0],
                             (vel_due ? 1 : 0) + (before > 0 ? 2 : 0)};
        bool captured = false;
        rc = replay(L.step, ks, [&] {
            captured = true;
            int r = issue_part_a(L, vel_due);
            if (!r) r = rmpcd_particles_switch_force(L.s);
            if (!r) r = rmpcd_particles_switch_force(L.c);
            if (!r) r = issue_part_b(L, nullptr, nullptr, L.ctl + 1);
            return r;
        });
        if (rc) return rc;
        // a replay does the capture's host-side force switch here
        if (!captured) {
            rc = rmpcd_particles_switch_force(L.s);
            if (!rc) rc = rmpcd_particles_switch_force(L.c);
            if (rc) return rc;
        }
        RMPCD_CUDA_TRY(cudaEventRecord(L.ev_step, stream()));
        bool resort = false;
        rc = wait_resort(L, seq, &resort);
        if (rc) return rc;
        if (!resort) {
            L.full_rolls = before > 0 ? before - 1 : 0;
            L.s->force_zero = false;
            L.c->force_zero = false;
            return RMPCD_OK;
        }
        // the gated part did nothing: back to the state before the force
        // switch, then the sort and the forces
        L.full_rolls = before;
        L.s->force_zero = fz[0];
        L.s->force_old_zero = fz[1];
        L.c->force_zero = fz[2];
        L.c->force_old_zero = fz[3];
        rc = rmpcd_particles_switch_force(L.s);
        if (!rc) rc = rmpcd_particles_switch_force(L.c);
        if (!rc) rc = catch_up_and_sort(L, false);
        if (rc) return rc;
        L.st->n_extra_sorting += 1;
        return md_step_forces(L, false);
    }
    if (L.graphs) {
        const NcLoop::Key ka{L.s->pos[L.s->cur][0], L.s->force[L.s->cur][0], L.c->force[L.c->cur][0],
                             vel_due ? 1 : 0};
        rc = replay(L.part_a, ka, [&] { return issue_part_a(L, vel_due); });
    } else {
        rc = issue_part_a(L, vel_due);
    }
    if (rc) return rc;
    bool resort = false;
    rc = read_resort(L, &resort);
    if (rc) return rc;
    if (resort) {
        rc = catch_up_and_sort(L, false);
        if (rc) return rc;
        L.st->n_extra_sorting += 1;
    }
    return md_step_forces(L, want_energy);
}

}  // namespace rmpcd

using namespace rmpcd;

static bool g_nc_graphs = true;
// the loop kept from the last call (scratch and captured graphs), and the
// lock that one thread at a time holds while it runs on it
static std::mutex g_nc_mutex;
static NcLoop *g_nc_loop = nullptr;

namespace rmpcd {

void ncolloids_forget(const void *handle)
{
    std::lock_guard<std::mutex> lk(g_nc_mutex);
    NcLoop *L = g_nc_loop;
    if (L && (handle == L->s || handle == L->c || handle == L->cells || handle == L->nl)) {
        cudaStreamSynchronize(stream());
        delete L;
        g_nc_loop = nullptr;
    }
}

}  // namespace rmpcd

extern "C" int rmpcd_ncolloids_set_graphs(int on)
{
    g_nc_graphs = on != 0;
    return RMPCD_OK;
}

extern "C" int rmpcd_ncolloids_run(rmpcd_particles *solvent, rmpcd_particles *colloids, rmpcd_cells *cells,
                                   rmpcd_nlist *nl, const rmpcd_lj *solvent_colloid, const rmpcd_lj *colloid_colloid,
                                   rmpcd_rng *rng, const rmpcd_ncolloids_params *params, int n_intervals,
                                   int thermostat, const double *T, int first_interval, int rescale_every,
                                   double T_rescale, rmpcd_ncolloids_state *state)
{
    RMPCD_ARG(solvent && colloids && cells && nl && solvent_colloid && colloid_colloid && rng && params && state,
              "null argument");
    RMPCD_ARG(n_intervals >= 0 && params->N_MD >= 1 && params->tau > 0, "n_intervals >= 0, N_MD >= 1, tau > 0");
    RMPCD_ARG(!thermostat || T, "a thermostatted run needs the temperatures T");
    RMPCD_ARG(colloids->precision == RMPCD_FP64, "colloids must be FP64");
    // the loop of the previous call is reused (scratch and graphs) when its
    // signature matches; a call that finds it in use by another thread runs
    // on a loop of its own
    std::unique_lock<std::mutex> lk(g_nc_mutex, std::try_to_lock);
    std::unique_ptr<NcLoop> own;
    NcLoop *Lp = nullptr;
    std::vector<unsigned long long> sig;
    const bool keep = lk.owns_lock() && g_nc_graphs;
    if (keep) {
        sig = nc_signature(solvent, colloids, cells, nl, solvent_colloid, colloid_colloid, params);
        if (g_nc_loop && g_nc_loop->sig == sig) {
            Lp = g_nc_loop;
        } else if (g_nc_loop) {
            cudaStreamSynchronize(stream());
            delete g_nc_loop;
            g_nc_loop = nullptr;
        }
    }
    if (!Lp) {
        own.reset(new NcLoop);
        Lp = own.get();
        const int rc = nc_alloc(*Lp, cells->S, solvent->N);
        if (rc) return rc;
    }
    NcLoop &L = *Lp;
    L.s = solvent;
    L.c = colloids;
    L.cells = cells;
    L.nl = nl;
    L.lj_sc = solvent_colloid;
    L.lj_cc = colloid_colloid;
    L.rng = rng;
    L.prm = params;
    L.st = state;
    L.vv_mass.assign((size_t)colloids->N, params->mass);
    L.dt = params->tau / params->N_MD;
    L.full_rolls = 2;
    L.graphs = false;
    PhaseTimer timer("ncolloids_run");
    // the solvent is sorted on entry: its slots from the cell ranges
    k_fill_cellmap<<<grid_full((long long)cells->S * kLanesPerCell, 256), 256, 0, stream()>>>(
        cells->count, cells->start, cells->S, L.cellmap);
    L.seq = 0;
    ((volatile int *)L.h_ctl)[0] = 0;
    k_nc_set_since<<<1, 1, 0, stream()>>>(L.ctl, state->t - state->last_sort);
    RMPCD_CUDA_TRY(cudaMemsetAsync(solvent->d_max, 0, 8, stream()));
    int rc0 = list_md_cells(L);
    for (int k = 0; !rc0 && k < n_intervals; k++) {
        const int i = first_interval + k;
        int rc = 0;
        for (int j = 0; !rc && j < params->N_MD; j++) {
            rc = md_step(L, j == params->N_MD - 1, j > 0);
            // the first MD step runs uncaptured (it allocates the force
            // scratch on a first use); graphs stay off while phase timers run
            L.graphs = g_nc_graphs && !timers_on();
        }
        if (!rc) rc = vel_tail(L);
        if (!rc) rc = rmpcd_cells_random_shift(cells, rng);
        if (!rc) rc = catch_up_and_sort(L, k == n_intervals - 1);
        if (!rc)
            rc = rmpcd_simple_mpcd_step(solvent, cells, rng, 0, 0.0, thermostat, T ? T[k] : 0.0, params->do_hydro);
        if (!rc && rescale_every > 0 && i % rescale_every == 0) rc = rmpcd_rescale_cells(solvent, cells, nullptr, T_rescale);
        rc0 = rc;
    }
    cudaStreamSynchronize(stream());
    if (keep) {
        if (rc0) {
            // an error drops the kept loop
            if (Lp == g_nc_loop) {
                delete g_nc_loop;
                g_nc_loop = nullptr;
            }
        } else if (own) {
            // the force scratch may have been allocated by this call: the
            // signature is taken again before the loop is kept
            L.sig = nc_signature(solvent, colloids, cells, nl, solvent_colloid, colloid_colloid, params);
            g_nc_loop = own.release();
        }
    }
    if (rc0) return rc0;
    return check_dev_error(nullptr);
}
