/*
 * rmpcd.h -- C ABI of the B200-native RMPCDMD solvent hot path.
 *
 * The reference (pdebuyl-lab/RMPCDMD, Fortran 2008) has no plugin layer: its
 * programs call module procedures directly through `use rmpcdmd_module`.
 * This header exposes the same procedures as plain C entry points over opaque
 * handles whose particle and cell data live in GPU memory.  Each entry point
 * names the reference procedure it replaces (file:line in the reference tree).
 *
 * Conventions
 *   - Every function returns 0 (RMPCD_OK) or an rmpcd_status code;
 *     rmpcd_last_error_string() describes the last failure of the calling
 *     thread.  Reference `stop` / `error stop` conditions become
 *     RMPCD_ERR_STOP / RMPCD_ERR_NLIST_FULL with the reference's message.
 *   - Host arrays use the reference layout: positions, velocities, forces
 *     and images are column-major (3,N), i.e. x(k,i) = a[3*i + k]; cell
 *     starts, neighbor-list entries and id_to_idx are 1-based; cells are
 *     addressed by 0-based compact Hilbert index (slot), S slots in total.
 *   - All work runs on one CUDA stream owned by the library; calls that
 *     return host data synchronize it.  A handle must not be used from two
 *     host threads at once.
 *   - Solvent systems are FP64 (RMPCD_FP64, results identical to the
 *     reference arithmetic) or FP32 (RMPCD_FP32, positions/velocities in
 *     single precision with compensated per-cell sums).  Colloid systems are
 *     always FP64.
 *   - Randomness: an rmpcd_rng {seed, step} replaces the reference's
 *     threefry_rng_t state(:) arrays.  Each random consumer uses the current
 *     step and advances it by one.  Draws are Philox4x32-10 keyed by
 *     (seed, step, index, stream), so results do not depend on scheduling.
 */
#ifndef RMPCD_H
#define RMPCD_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum rmpcd_status {
    RMPCD_OK = 0,
    RMPCD_ERR_INVALID = 1,     /* bad argument or handle */
    RMPCD_ERR_CUDA = 2,        /* CUDA runtime failure */
    RMPCD_ERR_NLIST_FULL = 3,  /* 'maximum of neighbor list reached' */
    RMPCD_ERR_STOP = 4,        /* a reference stop / error stop condition */
    RMPCD_ERR_CAPACITY = 5,    /* a size above a documented maximum */
    RMPCD_ERR_NO_DEVICE = 6,   /* no CUDA device visible */
    RMPCD_ERR_DEVICE = 7       /* a kernel reported an error (see message) */
};

enum { RMPCD_FP64 = 64, RMPCD_FP32 = 32 };
enum { RMPCD_PERIODIC_BC = 1, RMPCD_BOUNCE_BACK_BC = 2, RMPCD_SPECULAR_BC = 3 };

typedef struct rmpcd_cells rmpcd_cells;         /* cell_system_t   */
typedef struct rmpcd_particles rmpcd_particles; /* particle_system_t */
typedef struct rmpcd_nlist rmpcd_nlist;         /* neighbor_list_t */

/* lj_params_t, src/interaction.f90:23-34.  Tables are column-major (n1,n2)
 * with the solvent species first: t[(s1-1) + n1*(s2-1)]. */
#define RMPCD_MAX_SPECIES 4
typedef struct rmpcd_lj {
    int n1, n2;
    double epsilon[RMPCD_MAX_SPECIES * RMPCD_MAX_SPECIES];
    double sigma[RMPCD_MAX_SPECIES * RMPCD_MAX_SPECIES];
    double sigma_sq[RMPCD_MAX_SPECIES * RMPCD_MAX_SPECIES];
    double cut[RMPCD_MAX_SPECIES * RMPCD_MAX_SPECIES];
    double cut_sq[RMPCD_MAX_SPECIES * RMPCD_MAX_SPECIES];
    double cut_energy[RMPCD_MAX_SPECIES * RMPCD_MAX_SPECIES];
} rmpcd_lj;

/* Replaces type(threefry_rng_t) :: state(:) (src/mpcd.f90:75). */
typedef struct rmpcd_rng {
    uint64_t seed;
    uint64_t step;
} rmpcd_rng;

/* ------------------------------------------------------------------ */
/* library                                                             */
/* ------------------------------------------------------------------ */
const char *rmpcd_last_error_string(void);
int rmpcd_version(int *major, int *minor);
/* Select the CUDA device for this process; must precede every other call
 * that touches the GPU (one process per GPU). */
int rmpcd_set_device(int device);
/* Synchronize the library stream and report device-side errors. */
int rmpcd_get_status(void);
int rmpcd_synchronize(void);
/* Per-phase device timers (the reference's timer_t, src/common.f90:99-108,
 * with names such as "stream", "step", "sort", "count", "md_pos", "md_vel",
 * "neigh list update", "neigh list force"): when enabled, CUDA events on the
 * library stream bracket each phase and accumulate its time. */
int rmpcd_timers_enable(int on);
int rmpcd_timers_reset(void);
int rmpcd_timers_read(int idx, char *name, int name_len, double *seconds, long long *calls);
/* Elapsed device time, in ms, of an event pair recorded on the library
 * stream: rmpcd_mark() returns a mark id, rmpcd_elapsed_ms() reads two. */
int rmpcd_mark(int *mark_id);
int rmpcd_elapsed_ms(int mark_a, int mark_b, float *ms);
/* Page-locked host memory for callers that stream particle arrays in and
 * out every step (uploads and downloads from it run at full link speed). */
int rmpcd_host_alloc(size_t bytes, void **ptr);
int rmpcd_host_free(void *ptr);

/* Host evaluation of the counter-based draws the kernels use, so a host
 * program can reproduce them (initial conditions, replay, checks):
 * two uniforms in [0,1) for (seed, step, index, stream, attempt); the unit
 * axis of rand_sphere (src/mpcd.f90:43-62) for a slot; one normal deviate.
 * Streams: 1 random_shift, 2 SRD axis, 3 normals, 4 change_species,
 * 5 random_placement, 7 bulk_reaction. */
int rmpcd_rng_uniform2(uint64_t seed, uint64_t step, uint32_t index, uint32_t stream,
                       uint32_t attempt, double out[2]);
int rmpcd_rng_sphere(uint64_t seed, uint64_t step, uint32_t index, double out[3]);
int rmpcd_rng_normal(uint64_t seed, uint64_t step, uint32_t index, uint32_t sub, double *out);

/* ------------------------------------------------------------------ */
/* Hilbert keys, src/hilbert.f90                                       */
/* ------------------------------------------------------------------ */
/* compact_p_to_h, src/hilbert.f90:241-271 (host evaluation) */
int rmpcd_compact_p_to_h(const int p[3], const int M[3], int *h);
/* compact_h_to_p, src/hilbert.f90:273-307 (host evaluation) */
int rmpcd_compact_h_to_p(int h, const int M[3], int p[3]);

/* ------------------------------------------------------------------ */
/* cell_system_t, src/cell_system.f90:20-41                            */
/* ------------------------------------------------------------------ */
/* cell_system_t%init, src/cell_system.f90:49-84 */
int rmpcd_cells_init(rmpcd_cells **cells, const int L[3], double a, int has_walls);
int rmpcd_cells_destroy(rmpcd_cells *cells);
/* L (with the wall layer), M, S and edges */
int rmpcd_cells_info(const rmpcd_cells *cells, int L[3], int M[3], int *S, double edges[3]);
/* cells%origin, cells%bc, cells%max_v assignments in the programs */
int rmpcd_cells_set_origin(rmpcd_cells *cells, const double origin[3]);
int rmpcd_cells_get_origin(const rmpcd_cells *cells, double origin[3]);
int rmpcd_cells_set_bc(rmpcd_cells *cells, const int bc[3]);
int rmpcd_cells_set_max_v(rmpcd_cells *cells, double max_v);
/* random_shift, src/cell_system.f90:153-163 */
int rmpcd_cells_random_shift(rmpcd_cells *cells, rmpcd_rng *rng);
/* count_particles, src/cell_system.f90:86-129, on the positions of p */
int rmpcd_cells_count_particles(rmpcd_cells *cells, rmpcd_particles *p);
/* sort_particles, src/cell_system.f90:131-151: the positions of position_old
 * written, in cell order, as the positions of position_new (a different system
 * of the same size and precision; nothing else of either changes), through the
 * starts of the last count_particles on those positions.  Inside a cell the
 * order is ascending in position_old (the reference's single-thread order).
 * Afterwards every cell_start has advanced by its cell's count, as the
 * reference's scatter leaves it; call count_particles again before using the
 * starts.  Counts or starts that do not belong to these positions are
 * RMPCD_ERR_INVALID, with nothing written. */
int rmpcd_cells_sort_particles(rmpcd_cells *cells, const rmpcd_particles *position_old,
                               rmpcd_particles *position_new);
/* cell_count(S), cell_start(S) (1-based), is_md(S), is_reac(S) */
int rmpcd_cells_download_count(const rmpcd_cells *cells, int *count);
int rmpcd_cells_download_start(const rmpcd_cells *cells, int *start);
int rmpcd_cells_download_is_md(const rmpcd_cells *cells, unsigned char *is_md);
int rmpcd_cells_download_is_reac(const rmpcd_cells *cells, unsigned char *is_reac);
int rmpcd_cells_upload_is_md(rmpcd_cells *cells, const unsigned char *is_md);
int rmpcd_cells_upload_is_reac(rmpcd_cells *cells, const unsigned char *is_reac);
/* Injected SRD rotation axes, one unit vector per slot (3*S doubles, slot
 * major); NULL returns to the Philox axes.  Used for parity runs that replay
 * a recorded stream of rand_sphere draws (src/mpcd.f90:162). */
int rmpcd_cells_set_axes(rmpcd_cells *cells, const double *axes);

/* ------------------------------------------------------------------ */
/* particle_system_t, src/particle_system.f90:22-77                    */
/* ------------------------------------------------------------------ */
/* particle_system_t%init, src/particle_system.f90:81-184.  mass may be NULL
 * (n_species masses otherwise).  ids start at 1..Nmax, image and flags at 0;
 * positions, velocities and forces start at 0. */
int rmpcd_particles_init(rmpcd_particles **p, int Nmax, int n_species,
                         const double *mass, int precision);
int rmpcd_particles_destroy(rmpcd_particles *p);
int rmpcd_particles_info(const rmpcd_particles *p, int *Nmax, int *n_species, int *precision);
/* Host <-> device copies of the reference arrays.  field is one of
 * "pos", "pos_old", "vel", "force", "force_old", "pos_rattle" (double, (3,N)),
 * "image" (int, (3,N)), "id", "species", "flags" (int, N),
 * "id_to_idx" (int, N, download only, 1-based). */
int rmpcd_particles_upload(rmpcd_particles *p, const char *field, const void *host);
int rmpcd_particles_download(const rmpcd_particles *p, const char *field, void *host);
/* particle_system_t%sort, src/particle_system.f90:304-355 (stable in the
 * previous order, as the reference's single-thread loop) */
int rmpcd_particles_sort(rmpcd_particles *p, rmpcd_cells *cells);
/* maximum_displacement, src/particle_system.f90:357-378 */
int rmpcd_particles_maximum_displacement(rmpcd_particles *p, double *r);
/* cell_maximum_displacement, src/particle_system.f90:380-410 */
int rmpcd_cell_maximum_displacement(rmpcd_cells *cells, rmpcd_particles *p,
                                    double delta_t, double *r);
/* random_placement, src/particle_system.f90:250-302 (other/lj may be NULL).
 * The draws are keyed by state->seed alone (the reference's state(1)); the
 * step is not advanced. */
int rmpcd_particles_random_placement(rmpcd_particles *p, const double L[3],
                                     rmpcd_particles *other, const rmpcd_lj *lj,
                                     const rmpcd_rng *state);
/* Maxwell velocities with the mean removed, programs/single_dimer_pbc.f90:240-245 */
int rmpcd_particles_maxwell(rmpcd_particles *p, double T, uint64_t seed);
/* Number of particles with a NaN or infinite position or velocity component
 * (no counterpart in the reference, which has no such check; a run fed with
 * such values keeps running, every slot index staying inside the grid). */
int rmpcd_particles_count_nonfinite(const rmpcd_particles *p, long long *n_bad);
/* switch(force, force_old), src/common.f90:268-276; force = 0;
 * pos_old = pos; pos_rattle = pos (programs/single_dimer_pbc.f90:311-348) */
int rmpcd_particles_switch_force(rmpcd_particles *p);
int rmpcd_particles_zero_force(rmpcd_particles *p);
int rmpcd_particles_copy_pos_old(rmpcd_particles *p);
int rmpcd_particles_copy_pos_rattle(rmpcd_particles *p);
int rmpcd_particles_copy_force_old(rmpcd_particles *p);
/* Injected MPC-AT normals (3*N doubles in sorted position order); NULL
 * returns to Philox normals (src/mpcd.f90:148-150). */
int rmpcd_particles_set_gauss(rmpcd_particles *p, const double *gauss);

/* ------------------------------------------------------------------ */
/* MPCD, src/mpcd.f90                                                   */
/* ------------------------------------------------------------------ */
/* simple_mpcd_step, src/mpcd.f90:71-183.  has_alpha selects present(alpha);
 * thermostat selects MPC-AT; hydro defaults to 1 in the reference. */
int rmpcd_simple_mpcd_step(rmpcd_particles *p, rmpcd_cells *cells, rmpcd_rng *rng,
                           int has_alpha, double alpha, int thermostat, double T,
                           int hydro);
/* wall_mpcd_step, src/mpcd.f90:193-337.  wall arrays may all be NULL. */
int rmpcd_wall_mpcd_step(rmpcd_particles *p, rmpcd_cells *cells, rmpcd_rng *rng,
                         const double wall_temperature[2], const double wall_v[6],
                         const int wall_n[2], int thermostat, double bulk_temperature,
                         int has_alpha, double alpha, int keep_cell_v);
/* compute_temperature, src/mpcd.f90:342-407 */
int rmpcd_compute_temperature(rmpcd_particles *p, rmpcd_cells *cells, double *te);
/* rescale_cells, src/mpcd.f90:748-801; rng may be NULL (the reference takes
 * state(:) and draws nothing from it) */
int rmpcd_rescale_cells(rmpcd_particles *p, rmpcd_cells *cells, rmpcd_rng *rng, double T);
/* mpcd_stream_periodic, src/mpcd.f90:440-457 */
int rmpcd_mpcd_stream_periodic(rmpcd_particles *p, rmpcd_cells *cells, double dt);
/* mpcd_stream_xforce_yzwall, src/mpcd.f90:464-506 (+ yzwall_collision :511-589) */
int rmpcd_mpcd_stream_xforce_yzwall(rmpcd_particles *p, rmpcd_cells *cells, double dt,
                                    double g);
/* mpcd_stream_nogravity_zwall, src/mpcd.f90:702-745 */
int rmpcd_mpcd_stream_nogravity_zwall(rmpcd_particles *p, rmpcd_cells *cells, double dt);
/* bulk_reaction, src/mpcd.f90:605-643 */
int rmpcd_bulk_reaction(rmpcd_particles *p, rmpcd_cells *cells, int from, int to,
                        double rate, double tau, rmpcd_rng *rng);
/* bulk_reaction_endothermic, src/mpcd.f90:645-700 (the reaction also needs the
 * cell's relative kinetic energy to exceed delta_u, and removes delta_u from it) */
int rmpcd_bulk_reaction_endothermic(rmpcd_particles *p, rmpcd_cells *cells, int from, int to,
                                    double rate, double tau, rmpcd_rng *rng, double delta_u);

/* ------------------------------------------------------------------ */
/* MD, src/md.f90                                                       */
/* ------------------------------------------------------------------ */
int rmpcd_md_pos(rmpcd_particles *p, double dt);                 /* :61-77 */
int rmpcd_md_vel(rmpcd_particles *p, double dt);                 /* :219-237 */
int rmpcd_cell_md_pos(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag); /* :79-102 */
int rmpcd_cell_md_vel(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag); /* :239-263 */
int rmpcd_cell_md_pos_ywall(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag); /* :104-151 */
int rmpcd_cell_md_pos_zwall(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag); /* :153-200 */
int rmpcd_apply_pbc(rmpcd_particles *p, const double edges[3]);  /* :202-217 */
int rmpcd_rattle_dimer_pos(rmpcd_particles *p, double d, double dt, const double edges[3]); /* :265-296 */
int rmpcd_rattle_dimer_vel(rmpcd_particles *p, double d, double dt, const double edges[3]); /* :298-319 */

/* ------------------------------------------------------------------ */
/* Rigid-body colloids (programs/single_body.f90), FP64 systems.        */
/* links: n_link pairs of 1-based particle numbers, the reference's     */
/* links(2, n_link); distances: n_link target lengths.                   */
/* ------------------------------------------------------------------ */
/* rattle_body_pos, src/md.f90:321-408.  Needs pos_rattle (which is left
 * unwrapped relative to particle 1, as the reference leaves it).
 * *iterations = the reference's rattle_i at exit: the sweep that converged,
 * or 1001 when 1000 sweeps did not (the reference warns when it is 1000). */
int rmpcd_rattle_body_pos(rmpcd_particles *p, const int *links, const double *distances, int n_link,
                          double dt, const double edges[3], double precision, int *iterations);
/* rattle_body_vel, src/md.f90:410-480 */
int rmpcd_rattle_body_vel(rmpcd_particles *p, const int *links, const double *distances, int n_link,
                          double dt, const double edges[3], double precision, int *iterations);
/* elastic_network, src/md.f90:516-544: adds the harmonic link forces to
 * force and returns the energy */
int rmpcd_elastic_network(rmpcd_particles *p, const int *links, const double *distances, int n_link,
                          double k, const double edges[3], double *energy);

/* rigid_body_t, src/md.f90:40-58: the body's scalar state (device
 * resident; read and written with rmpcd_rigid_body_get / _set).  q is
 * (s, x, y, z). */
typedef struct rmpcd_rigid_body_state {
    double mass;
    double pos[3], vel[3], force[3];
    double q[4];
    double L[3], torque[3];
    double I_body[3], omega_body[3];
} rmpcd_rigid_body_state;
typedef struct rmpcd_rigid_body rmpcd_rigid_body;
/* rigid_body_init, src/md.f90:547-588 (beads i_start..i_stop, 1-based) */
int rmpcd_rigid_body_init(rmpcd_rigid_body **rb, rmpcd_particles *p, int i_start, int i_stop,
                          const double edges[3]);
int rmpcd_rigid_body_destroy(rmpcd_rigid_body *rb);
/* rigid_body_compute_force_torque, src/md.f90:591-607 */
int rmpcd_rigid_body_compute_force_torque(rmpcd_rigid_body *rb, rmpcd_particles *p);
/* rigid_body_vv1, src/md.f90:613-673 (the quaternion iteration, unbounded
 * in the reference, stops after 100000 rounds with RMPCD_ERR_DEVICE) */
int rmpcd_rigid_body_vv1(rmpcd_rigid_body *rb, rmpcd_particles *p, double dt, double treshold,
                         const double edges[3]);
/* rigid_body_vv2, src/md.f90:679-700 */
int rmpcd_rigid_body_vv2(rmpcd_rigid_body *rb, rmpcd_particles *p, double dt);
/* state (and, if pos_body is not null, the 3 x n_beads body-frame positions) */
int rmpcd_rigid_body_get(const rmpcd_rigid_body *rb, rmpcd_rigid_body_state *state, double *pos_body);
int rmpcd_rigid_body_set(rmpcd_rigid_body *rb, const rmpcd_rigid_body_state *state);
/* colloid velocity-Verlet halves written inline in the programs
 * (programs/single_dimer_pbc.f90:312-315,356-359); mass[k] per particle */
int rmpcd_colloid_vv_pos(rmpcd_particles *p, double dt, const double *mass);
int rmpcd_colloid_vv_vel(rmpcd_particles *p, double dt, const double *mass);
/* rmpcd_colloid_vv_pos without any device allocation; no counterpart in the
 * reference.  rmpcd_colloid_vv_pos keeps the masses in a device buffer that it
 * allocates (and frees, which synchronises the whole device) whenever a larger
 * system comes along; a caller that cannot allocate at that point (device
 * memory already committed to the solvent, or other streams that must not be
 * stalled by a synchronising free) calls this one instead.  The masses go to a
 * fixed 64 KB scratch array inside the library, so N must be <= 8192
 * (RMPCD_ERR_CAPACITY otherwise).  The first call on each device looks up the
 * scratch address (one-time setup): make it before starting any stream
 * capture.  `mass` is read by an asynchronous host-to-device copy on the
 * library stream: from pageable memory the driver has taken the values when
 * the call returns; from page-locked memory it reads them later, so keep them
 * unchanged until the library stream has passed the call (rmpcd_synchronize).
 * Nothing in the scratch has to start at zero.  There is one scratch array
 * per device, so calls that overlap (several host threads) race on it. */
int rmpcd_colloid_vv_pos_noalloc(rmpcd_particles *p, double dt, const double *mass);

/* ------------------------------------------------------------------ */
/* Lennard-Jones, src/interaction.f90                                   */
/* ------------------------------------------------------------------ */
/* lj_params_init, src/interaction.f90:38-80 (host only) */
int rmpcd_lj_init(rmpcd_lj *lj, int n1, int n2, const double *epsilon,
                  const double *sigma, const double *cut);

/* ------------------------------------------------------------------ */
/* neighbor_list_t, src/neighbor_list.f90:23-34                        */
/* ------------------------------------------------------------------ */
int rmpcd_nlist_init(rmpcd_nlist **nl, int Npoints, int Nmax);          /* :38-53 */
int rmpcd_nlist_destroy(rmpcd_nlist *nl);
int rmpcd_nlist_make_stencil(rmpcd_nlist *nl, rmpcd_cells *cells, double cut); /* :271-308 */
int rmpcd_nlist_stencil_size(const rmpcd_nlist *nl, int *n);
/* update_list, src/neighbor_list.f90:76-157 (lj may be NULL) */
int rmpcd_nlist_update(rmpcd_nlist *nl, rmpcd_particles *system1, rmpcd_particles *system2,
                       double radius, rmpcd_cells *cells, const rmpcd_lj *lj);
/* list(Nmax, Npoints) column-major 1-based, n(Npoints) */
int rmpcd_nlist_download(const rmpcd_nlist *nl, int *list, int *n);
/* compute_force, src/neighbor_list.f90:159-225 (energy may be NULL).  Each
 * colloid's force sum is in list order for an FP64 solvent (ps2); for an
 * FP32 solvent it is an FP64 sum by a fixed tree over the list (the same bits
 * on every call, not the list-order bits). */
int rmpcd_compute_force(rmpcd_particles *ps1, rmpcd_particles *ps2, rmpcd_nlist *nl,
                        const double L[3], const rmpcd_lj *lj, double *energy);
/* compute_force_n2, src/neighbor_list.f90:227-264 (energy may be NULL) */
int rmpcd_compute_force_n2(rmpcd_particles *ps, const double L[3], const rmpcd_lj *lj,
                           double *energy);

/* ------------------------------------------------------------------ */
/* program-local solvent loops, programs/single_dimer_pbc.f90           */
/* ------------------------------------------------------------------ */
/* flag_particles_nl, :493-509 (point = 0-based list column, usually 0) */
int rmpcd_flag_particles_nl(rmpcd_nlist *nl, int point, rmpcd_particles *colloids,
                            rmpcd_particles *solvent, const double edges[3], double cut_sq);
/* change_species, :511-542 */
int rmpcd_change_species(rmpcd_particles *solvent, rmpcd_particles *colloids,
                         const double edges[3], double cut_sq_C, double cut_sq_N,
                         double prob, rmpcd_rng *rng);
/* refuel, :544-565 (far = (L1*0.45)**2 in single precision, as written) */
int rmpcd_refuel(rmpcd_particles *solvent, rmpcd_particles *colloids,
                 const double edges[3], int L1);
/* n_solvent, :432-437 */
int rmpcd_n_solvent(rmpcd_particles *solvent, int n_species, int *counts);
/* compute_cylindrical_shell_histogram, src/particle_system.f90:412-445 */
int rmpcd_cylindrical_shell_histogram(rmpcd_particles *solvent, const double x1[3],
                                      const double x2[3], const double L[3],
                                      int bin_species, double r_min, double r_max,
                                      double xmin, double dx, int nbins, double *hist);
/* sum(vel**2), sum(vel, dim=2) of the thermo observables, :390-396 */
int rmpcd_velocity_sums(rmpcd_particles *p, double out[4]);

/* ------------------------------------------------------------------ */
/* fused schedules                                                      */
/* ------------------------------------------------------------------ */
/* n_intervals iterations of the bulk-fluid loop of
 * test/setup_bulk_decay.f90:112-121 (simple_mpcd_step -> mpcd_stream_periodic
 * -> random_shift -> sort).  The system must be sorted for the current
 * origin on entry and is sorted for the final origin on return.  Interval i
 * uses rng step s+2i for the collision and s+2i+1 for the shift.  FP64:
 * results equal the reference's single-thread arithmetic and order.  FP32:
 * the cell means come from exact fixed-point sums (2^-40 resolution), which
 * do not depend on the order of a cell's particles; on return each cell's
 * particles are in ascending order of their position on entry. */
int rmpcd_bulk_run(rmpcd_particles *p, rmpcd_cells *cells, rmpcd_rng *rng,
                   double tau, int has_alpha, double alpha, int n_intervals);
/* Tile shapes of the fused interval kernel (slots per block, resident
 * blocks per SM).  All shapes give the same results bit for bit; one is in
 * use per precision (shape 0 until set).  No counterpart in the reference. */
int rmpcd_bulk_shapes(int precision, int *n_shapes, int *slots, int *min_blocks);
int rmpcd_bulk_set_shape(int precision, int shape);
int rmpcd_bulk_get_shape(int precision, int *shape);
/* Autotuner: builds a synthetic bulk fluid of box L at density 10 (seeded
 * placement, Maxwell kT = 1/3), times n_intervals intervals with every
 * shape, puts the fastest in use for `precision` and returns its index in
 * *best; ms_per_shape (may be NULL) receives each shape's time. */
int rmpcd_bulk_autotune(const int L[3], int precision, double tau, int n_intervals, int *best,
                        float *ms_per_shape);

/* The main loops of programs/n_colloids_pbc.f90 (:221-276, :304-324) in one
 * call: n_intervals intervals of N_MD MD steps with lazy cell-wise solvent
 * streaming (cell_md_pos/vel on is_md cells, catch-up of the other cells
 * before each sort), the program's re-sort test, velocity-Verlet colloids,
 * then random_shift, catch-up + sort, simple_mpcd_step(thermostat, T[k],
 * do_hydro) and, for interval numbers i = first_interval + k divisible by
 * rescale_every (> 0), rescale_cells(T_rescale).  The calls and their order
 * are those of the program, so the results equal the same calls made one by
 * one; the loop state (MD step counters, re-sort count, the energies e1, e2
 * of each interval's last MD step) is carried in *state.  The call keeps its
 * scratch (about 4 B per slot and 4 B per solvent particle) and its captured
 * MD-step graphs for the next call, and reuses them while the handles, their
 * device arrays, the box, the LJ tables and tau, N_MD, skin and mass are the
 * same;
 * other arguments make it rebuild them.  A call made while another thread is
 * inside this function works with scratch of its own.  No module counterpart
 * in the reference. */
typedef struct rmpcd_ncolloids_params {
    double tau;          /* dt = tau / N_MD */
    int N_MD;
    double skin;         /* re-sort when a colloid moved >= skin/10 or the solvent >= 0.9 skin */
    double list_radius;  /* update_list radius: cut + skin */
    double mass;         /* colloid mass of the velocity-Verlet halves */
    int do_hydro;
} rmpcd_ncolloids_params;
typedef struct rmpcd_ncolloids_state {
    int t;               /* MD steps of the current loop */
    int last_sort;       /* t at the last sort */
    int n_extra_sorting;
    double e1, e2;       /* compute_force / compute_force_n2 energies */
} rmpcd_ncolloids_state;
int rmpcd_ncolloids_run(rmpcd_particles *solvent, rmpcd_particles *colloids, rmpcd_cells *cells,
                        rmpcd_nlist *nlist, const rmpcd_lj *solvent_colloid, const rmpcd_lj *colloid_colloid,
                        rmpcd_rng *rng, const rmpcd_ncolloids_params *params, int n_intervals, int thermostat,
                        const double *T, int first_interval, int rescale_every, double T_rescale,
                        rmpcd_ncolloids_state *state);
/* Whether rmpcd_ncolloids_run replays its MD steps as CUDA graphs (default
 * on; the results are the same either way).  No counterpart in the
 * reference. */
int rmpcd_ncolloids_set_graphs(int on);

/* Batched single_dimer_pbc: the main loop of programs/single_dimer_pbc.f90
 * (:303-443: N_MD MD steps with the program's re-sort test, then
 * random_shift, re-sort, simple_mpcd_step and refuel) for R independent
 * systems advanced together, one launch per phase for all of them, the
 * whole interval captured once in a CUDA graph.  This replaces the program's
 * own loop (it has no module counterpart in the reference): each replica is
 * set up with the module entry points above exactly as the program does,
 * handed over with rmpcd_dimer_batch_create, and copied back into handles
 * with rmpcd_dimer_batch_scatter for output.  Replica r then holds, bit for
 * bit, the state of its own handles advanced by the same calls one by one. */
typedef struct rmpcd_dimer_batch rmpcd_dimer_batch;
typedef struct rmpcd_dimer_params {
    double tau;          /* MPCD interval; dt = tau / N_MD */
    int N_MD;            /* MD steps per interval */
    double bond;         /* dimer bond length d (rattle) */
    double skin;         /* list skin: re-sort when a colloid moved >= skin/10
                            or a solvent particle >= 0.89 skin */
    double list_radius;  /* update_list radius: max cut + skin */
    double prob;         /* A -> B probability of change_species */
    double cut_sq_C;     /* cut_sq(1,1): flag_particles_nl and change_species */
    double cut_sq_N;     /* cut_sq(1,2): change_species */
    double vv_mass[2];   /* masses of the two beads in the velocity-Verlet halves */
    int thermostat;      /* simple_mpcd_step options */
    int hydro;
    double T;
} rmpcd_dimer_params;
/* solvent[r], colloids[r] (2 FP64 beads), cells[r] (periodic), nlists[r]
 * (2 points, stencil made) and rngs[r] (same step for every r) describe
 * replica r after the program's set-up; their state is copied, the handles
 * stay the caller's.  solvent_colloid / colloid_colloid are the two
 * lj_params_t of the program. */
int rmpcd_dimer_batch_create(rmpcd_dimer_batch **batch, int n_replicas, rmpcd_particles *const *solvent,
                             rmpcd_particles *const *colloids, rmpcd_cells *const *cells,
                             rmpcd_nlist *const *nlists, const rmpcd_rng *rngs,
                             const rmpcd_lj *solvent_colloid, const rmpcd_lj *colloid_colloid,
                             const rmpcd_dimer_params *params);
int rmpcd_dimer_batch_destroy(rmpcd_dimer_batch *batch);
/* n_intervals MPCD intervals of every replica */
int rmpcd_dimer_batch_run(rmpcd_dimer_batch *batch, int n_intervals);
/* replay a captured interval graph (1, the default) or launch the kernels
 * one by one (0) */
int rmpcd_dimer_batch_set_graph(rmpcd_dimer_batch *batch, int use_graph);
/* copy replica r's state into handles shaped like the ones it came from
 * (any of them may be NULL) */
int rmpcd_dimer_batch_scatter(rmpcd_dimer_batch *batch, int replica, rmpcd_particles *solvent,
                              rmpcd_particles *colloids, rmpcd_cells *cells, rmpcd_nlist *nlist,
                              rmpcd_rng *rng);
/* replica count, total solvent, and per replica the number of extra re-sorts
 * (the program's n_extra_sorting; array of n_replicas, may be NULL) */
int rmpcd_dimer_batch_info(const rmpcd_dimer_batch *batch, int *n_replicas, long long *n_solvent,
                           int *n_extra_sorting);
/* Engine shapes (no counterpart in the reference): particles per tile of
 * the solvent kernels, particles per thread and pass of the MD step's
 * begin / end halves, the blocks per SM they are compiled for, the list
 * entries per thread of the list kernels (pair forces, their application,
 * the contribution reset), and whether the colloid half of the step begin
 * runs in an extra first block while the solvent streams (1) or in the block
 * that finishes last (0).  Every shape gives the same results
 * bit for bit.  A batch starts on 1024-particle tiles (smaller when that
 * gives fewer than ~2 tiles per SM) and one list entry per thread. */
int rmpcd_dimer_batch_shapes(int precision, int *n_shapes);
int rmpcd_dimer_batch_shape_info(int precision, int shape, int *particles_per_tile, int *per_thread_begin,
                                 int *per_thread_end, int *blocks_per_sm, int *list_entries_per_thread,
                                 int *colloid_block_first);
int rmpcd_dimer_batch_set_shape(rmpcd_dimer_batch *batch, int shape);
int rmpcd_dimer_batch_get_shape(const rmpcd_dimer_batch *batch, int *shape);
/* The engine's autotuner: every tile size and kernel variant with one list
 * entry per thread, then the fastest of them with each other list setting,
 * runs one interval (capture and warm-up) and n_intervals timed intervals of
 * the batch itself -- real intervals of the run, since every shape gives the
 * same results -- and the fastest is kept (*best; ms_per_interval, if not
 * NULL, receives the time of each of the n_shapes, -1 for those not run).  The choice is remembered per GPU, precision, N_MD
 * and mix of boxes: a later batch of the same kind takes it without running
 * anything (*intervals_run = 0, ms_per_interval entries -1).
 * *intervals_run = the intervals the call advanced every replica by. */
int rmpcd_dimer_batch_autotune(rmpcd_dimer_batch *batch, int n_intervals, int *best, float *ms_per_interval,
                               int *intervals_run);

#ifdef __cplusplus
}
#endif
#endif
