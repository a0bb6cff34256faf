// Counting and stable cell sort of a particle system (the core of
// count_particles, src/cell_system.f90:86-129, and particle_system_t%sort,
// src/particle_system.f90:304-355).
//
// Schedule (all on the library stream):
//   key/count  one pass over positions: key[i] = slot, warp-aggregated
//              atomic histogram into count[]
//   scan       exclusive scan count -> start, cursor
//   perm       one pass over keys: warp-aggregated cursor atomics give every
//              particle a place inside its cell: perm[place] = i
//   segsort    each cell's perm segment is sorted ascending, which restores
//              the reference's single-thread order (stable in i)
//   gather     dst[j] = src[perm[j]] for every field: coalesced writes,
//              reads local in the Hilbert order
#pragma once
#include "state.cuh"

namespace rmpcd {

// key[] and count/start/cursor of p under the current origin of c
int count_and_scan(rmpcd_cells *c, rmpcd_particles *p, bool keep_key);
// perm[] from key[] and cursor[] (cell order fixed, in-cell order arbitrary)
int build_perm_unsorted(rmpcd_cells *c, rmpcd_particles *p, int *cellmap = nullptr);
// ascending sort of every cell's perm segment (uses cursor[] and key[] as scratch)
int sort_perm_segments(rmpcd_cells *c, rmpcd_particles *p);
// both of the above
int build_perm(rmpcd_cells *c, rmpcd_particles *p, int *cellmap = nullptr);
// gather every field through perm into the other buffer and flip buffers
int gather_all(rmpcd_particles *p);
// full sort
int sort_particles(rmpcd_cells *c, rmpcd_particles *p);
// positions of `from` into `to` in cell order (cell_system_t%sort_particles)
int sort_positions(rmpcd_cells *c, const rmpcd_particles *from, rmpcd_particles *to);
// apply_pbc with the given edges, then the full sort, for a system in which a
// particle with neither MD nor PAST_MD set has zero force and force_old (the
// state compute_force and its flag roll maintain): those entries are written
// as zeros instead of being gathered
int sort_particles_flagged(rmpcd_cells *c, rmpcd_particles *p, const double edges[3]);
// the same sort after its key pass (p->key holds every particle's slot in the
// cells' grid, c->count their counts): scan, placement and gated gather;
// cellmap (if given) receives the slot of every particle of the sorted arrays
int sort_keyed_flagged(rmpcd_cells *c, rmpcd_particles *p, int *cellmap);
// ascending merge sort of the *n_big queued cells big[] of more than 64
// particles (tmp: scratch of the extent of perm)
void launch_segsort_big(const int *start, const int *count, const int *big, const int *n_big, int *perm,
                        int *tmp, cudaStream_t st);
// maximum-displacement reductions into p->d_max (r^2 as ordered bits), no
// synchronisation: maximum_displacement over all particles, and over the
// particles of is_md cells (src/particle_system.f90:357-410)
int launch_max_disp(rmpcd_particles *p);
int launch_cell_max_disp(rmpcd_cells *c, rmpcd_particles *p);
// compute_force_n2 of the colloids run right after compute_force, with the
// colloid sums, on a second stream beside the solvent force application
// (the two branches write disjoint arrays; each array sees the arithmetic
// of the two calls in sequence)
struct ForceN2Branch {
    const rmpcd_lj *lj_cc;      // colloid-colloid parameters of compute_force_n2
    cudaStream_t side;
    cudaEvent_t ev_fork, ev_join;
    const int *gate;            // device word; non-zero: every kernel of the evaluation returns at once (or null)
};
// compute_force (src/neighbor_list.f90:159-225); roll_flags = false leaves
// the PAST_MD/MD roll to the caller (which must then have done it).  n2 (no
// energy only): also compute_force_n2 of ps1, as above.
int compute_force_impl(rmpcd_particles *ps1, rmpcd_particles *ps2, rmpcd_nlist *nl, const double L[3],
                       const rmpcd_lj *lj, double *energy, bool roll_flags, const ForceN2Branch *n2 = nullptr);
// drops the n_colloids loop kept between calls if it refers to `handle` (a
// particle system, cell system or neighbor list being destroyed)
void ncolloids_forget(const void *handle);
// largest cell handled by sort_segment; larger ones go to launch_segsort_big
constexpr int kSmallSegmentMax = 64;

}  // namespace rmpcd
