// Handle types behind the C ABI and typed device views of them.
//
// Solvent layout in HBM (per particle system, double-buffered for the sort):
//   pos[b][k], vel[b][k], force[b][k], force_old[b][k]  -- one array per
//       component k (SoA), element type float (FP32 form) or double (FP64);
//   image[b][k] (int32 per component), id[b], species[b], flags[b] (int32).
// Component arrays give every warp 128-byte (float) or 256-byte (double)
// coalesced transactions per field.  The buffer index `cur` selects the live
// copy; the other copy is the sort target and doubles as pos_old, exactly as
// the reference's pointer pair (pos, pos_old) after particle_system_t%sort.
#pragma once
#include "rmpcd_common.cuh"

struct rmpcd_cells {
    int L[3];          // cell counts (wall layer included in L[2])
    double edges[3];   // L_in * a
    double a;
    double origin[3];
    int M[3];
    int S;             // 2^(M0+M1+M2) Hilbert slots
    int n_lut;         // L[0]*L[1]*L[2]
    int has_walls;
    int bc[3];
    double max_v;
    // device arrays
    int *count = nullptr;      // S
    int *start = nullptr;      // S, 0-based
    int *cursor = nullptr;     // S, scatter cursors
    int *count_next = nullptr; // S, counts of the next grid in fused schedules
    int *start_next = nullptr; // S ints of fused-schedule scratch (per tile: first particle, count)
    unsigned char *is_md = nullptr;
    unsigned char *is_reac = nullptr;
    int *lut = nullptr;        // n_lut: slot of cell (p0 + L0*(p1 + L1*p2))
    int *scan_tmp = nullptr;   // tile totals of the slot scan
    int scan_blocks = 0;
    double *axes = nullptr;    // injected SRD axes (3*S) or null
    double *d_red = nullptr;   // reduction scratch (temperature etc.)
    int red_cap = 0;
};

// The per-particle arrays made at init (pos ... flags, key, perm) are
// allocated to a multiple of 4 elements: bulk copies read 16-byte windows
// rounded outward.
struct rmpcd_particles {
    int N = 0;
    int n_species = 1;
    int precision = RMPCD_FP64;
    size_t rsize = 8;
    double mass[RMPCD_MAX_SPECIES] = {0, 0, 0, 0};
    int cur = 0;
    void *pos[2][3] = {};
    void *vel[2][3] = {};
    void *force[2][3] = {};
    void *force_old[2][3] = {};
    void *pos_rattle[3] = {};
    int *image[2][3] = {};
    int *id[2] = {};
    int *species[2] = {};
    int *flags[2] = {};
    // scratch
    int *key = nullptr;              // N, slot of each particle
    int *perm = nullptr;             // N, source index of each sorted slot
    int *id_to_idx = nullptr;        // N, built on demand
    double *gauss = nullptr;         // injected normals (3*N) or null
    unsigned long long *d_max = nullptr;  // max-reduction word
    double *d_sums = nullptr;        // reduction scratch
    int sums_cap = 0;
    int *d_ints = nullptr;           // small integer scratch (64 ints)
    void *stage = nullptr;           // (3,N) layout staging for host transfers, 24 B/particle
    size_t stage_bytes = 0;
    // packed particle records of the fused bulk schedule (double-buffered):
    // 6 reals (pos, vel) + 6 ints (image, id, species, flags) per particle
    unsigned char *rec[2] = {nullptr, nullptr};
    size_t rec_bytes = 0;
    // force / force_old entries known to be exactly zero: the sort skips
    // permuting them (a permutation of zeros is zeros)
    bool force_zero = true;
    bool force_old_zero = true;
    double *n2_terms = nullptr;  // pair energies of compute_force_n2, C (C - 1) / 2
    long long n2_cap = 0;
};

struct rmpcd_nlist {
    int Npoints = 0;
    int Nmax = 0;
    int *list = nullptr;   // Npoints*Nmax, 0-based solvent index, point-major
    int *n = nullptr;      // Npoints
    int *stencil = nullptr;  // device, 3*n_stencil
    int n_stencil = 0;
    int max_i = 0;
    int box_cells[3] = {0, 0, 0};  // cell counts of the box the stencil was built for
    // compute_force scratch
    double *pair_f = nullptr;   // 3 * Npoints*Nmax pair forces
    double *pair_e = nullptr;   // Npoints*Nmax pair energies
    unsigned char *contrib = nullptr;  // Npoints*Nmax
    int *ncontrib = nullptr;    // per solvent particle contribution counter
    int ncontrib_cap = 0;
    int *d_status = nullptr;
    unsigned long long *mkeys = nullptr;  // multi-contribution keys (kMultiSortMax)
    int *e_pre = nullptr;       // Npoints + 1, offsets of the energy terms per point
};

namespace rmpcd {

template <typename R>
struct Vec3 {
    R *x, *y, *z;
    __host__ __device__ R *operator[](int k) const { return k == 0 ? x : (k == 1 ? y : z); }
};

template <typename R>
struct PView {
    int N;
    Vec3<R> pos, vel, force, force_old;
    int *ix, *iy, *iz;
    int *id, *species, *flags;
};

template <typename R>
inline PView<R> view(const rmpcd_particles *p, int b)
{
    PView<R> v;
    v.N = p->N;
    v.pos = {(R *)p->pos[b][0], (R *)p->pos[b][1], (R *)p->pos[b][2]};
    v.vel = {(R *)p->vel[b][0], (R *)p->vel[b][1], (R *)p->vel[b][2]};
    v.force = {(R *)p->force[b][0], (R *)p->force[b][1], (R *)p->force[b][2]};
    v.force_old = {(R *)p->force_old[b][0], (R *)p->force_old[b][1], (R *)p->force_old[b][2]};
    v.ix = p->image[b][0];
    v.iy = p->image[b][1];
    v.iz = p->image[b][2];
    v.id = p->id[b];
    v.species = p->species[b];
    v.flags = p->flags[b];
    return v;
}
template <typename R>
inline PView<R> cur(const rmpcd_particles *p) { return view<R>(p, p->cur); }
template <typename R>
inline PView<R> alt(const rmpcd_particles *p) { return view<R>(p, 1 - p->cur); }

// Grid parameters a kernel needs for cartesian_indices and the key lookup.
struct Grid {
    int L[3];
    int M[3];
    double origin[3];
    double a;
    double edges[3];
    int has_walls;
    const int *lut;
};

inline Grid grid_of(const rmpcd_cells *c)
{
    Grid g;
    for (int k = 0; k < 3; k++) {
        g.L[k] = c->L[k];
        g.M[k] = c->M[k];
        g.origin[k] = c->origin[k];
        g.edges[k] = c->edges[k];
    }
    g.a = c->a;
    g.has_walls = c->has_walls;
    g.lut = c->lut;
    return g;
}

}  // namespace rmpcd
