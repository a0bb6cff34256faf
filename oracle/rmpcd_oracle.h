/*
 * rmpcd_oracle.h -- CPU FP64 restatement of the RMPCDMD solvent hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in rmpcdmd_b200/: only tests/, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py load it.  Nothing in the product links it.
 *
 * Parity status: the reference (Fortran 2008 + OpenMP) cannot be compiled in
 * this environment (no Fortran compiler; its Threefry/H5MD/ParseText
 * submodules are empty), and it ships no numeric golden vectors.  The
 * restatement is pinned against the property checks the reference's own
 * tests hold (test/test_cell_system_0.f90, test/test_neighbor_list_0.f90,
 * test/test_md_0.f90, test/test_particle_system_0.f90, test/dimer_test.py)
 * and against Hilbert-curve invariants; element-wise values are otherwise
 * "parity unpinned" against the Fortran binary.
 *
 * Conventions follow the reference exactly:
 *   - particle arrays are column-major (3,N) FP64: x(k,i) = a[3*i + k];
 *   - cell_start holds 1-based particle indices; neighbor lists hold 1-based
 *     particle indices; ids are 1-based labels;
 *   - cells are addressed by 0-based compact Hilbert index (slot), arrays of
 *     size S = 2^(M1+M2+M3);
 *   - flags use the reference bit positions (REAC=1, MD=2, WALL=3, PAST_MD=4,
 *     CATALYZED=6).
 * Floating-point expressions keep the reference's association order and are
 * compiled with -ffp-contract=off (no FMA), so results are reproducible.
 *
 * Randomness: the reference draws from Threefry streams whose source is not
 * available.  Every random quantity here comes from a counter-based
 * Philox4x32-10 generator (Salmon et al., SC'11) keyed by (seed, step, index,
 * stream, attempt), so a GPU implementation of the same generator reproduces
 * the exact draws; in addition, SRD rotation axes and MPC-AT Gaussians can be
 * injected from caller arrays.
 */
#ifndef RMPCD_ORACLE_H
#define RMPCD_ORACLE_H

#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

/* bit positions, src/common.f90:49-55 */
enum { ORC_REAC_BIT = 1, ORC_MD_BIT = 2, ORC_WALL_BIT = 3, ORC_PAST_MD_BIT = 4,
       ORC_OUTBOUND_BIT = 5, ORC_CATALYZED_BIT = 6 };
/* boundary conditions, src/cell_system.f90:43-45 */
enum { ORC_PERIODIC_BC = 1, ORC_BOUNCE_BACK_BC = 2, ORC_SPECULAR_BC = 3 };
/* RNG stream identifiers */
enum { ORC_RNG_SHIFT = 1, ORC_RNG_AXIS = 2, ORC_RNG_GAUSS = 3, ORC_RNG_REACT = 4,
       ORC_RNG_PLACE = 5, ORC_RNG_MAXWELL = 6, ORC_RNG_BULK = 7, ORC_RNG_WALL = 8 };

int orc_num_threads(void);
void orc_set_num_threads(int n);

/* ---------------- hilbert (src/hilbert.f90) ---------------- */
int orc_p_to_h(const int p[3], int m);
void orc_h_to_p(int h, int m, int p[3]);
int orc_compact_p_to_h(const int p[3], const int M[3]);
void orc_compact_h_to_p(int h, const int M[3], int p[3]);

/* ---------------- rng ---------------- */
void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]);
/* two uniform doubles in [0,1) for (seed, step, index, stream, attempt) */
void orc_rng_u2(uint64_t seed, uint64_t step, uint32_t index, uint32_t stream,
                uint32_t attempt, double u[2]);
/* Marsaglia (1972) unit vector, the rand_sphere of src/mpcd.f90:43-62 */
void orc_rand_sphere(uint64_t seed, uint64_t step, uint32_t index, double n[3]);
/* standard normal deviate by Leva's ratio-of-uniforms method (ACM TOMS 18, 1992) */
double orc_normal(uint64_t seed, uint64_t step, uint32_t index, uint32_t sub);
/* random_shift, src/cell_system.f90:153-163: origin(k) = u_k - 1 */
void orc_random_shift_values(uint64_t seed, uint64_t step, double origin[3]);

/* ---------------- cell system (src/cell_system.f90) ---------------- */
typedef struct {
    int L[3];           /* cell counts; with walls L[2] = L_in + 1 */
    double edges[3];    /* L_in * a */
    double a;
    double origin[3];
    int M[3];
    int S;              /* number of Hilbert slots, 2^(M1+M2+M3) */
    int has_walls;
    int bc[3];
    double max_v;
} orc_grid;

void orc_grid_init(orc_grid *g, const int L[3], double a, int has_walls);
void orc_cartesian_indices(const orc_grid *g, const double x[3], int p[3]);
void orc_count_particles(const orc_grid *g, int N, const double *pos,
                         int *cell_count, int *cell_start);
/* particle_system_t%sort, src/particle_system.f90:304-355.  All arrays are
 * permuted in place; pos_old receives the pre-sort positions (the buffer the
 * reference leaves in pos_old after its pointer swap).  Any of the optional
 * arrays may be NULL.  id_to_idx (1-based) is filled when not NULL. */
void orc_sort(const orc_grid *g, int N, int *cell_count, int *cell_start,
              double *pos, double *pos_old, int *image, double *vel,
              double *force, double *force_old, int *id, int *species,
              int *flags, int *id_to_idx);
/* cell_system_t%sort_particles, src/cell_system.f90:131-151 (cell_start is
 * advanced by the counts, as in the reference) */
void orc_sort_particles(const orc_grid *g, int N, int *cell_start,
                        const double *pos_in, double *pos_out);

/* ---------------- MPCD (src/mpcd.f90) ---------------- */
/* simple_mpcd_step, src/mpcd.f90:71-183.
 *   axes:   optional per-slot unit axes (3*S doubles); NULL draws
 *           orc_rand_sphere(seed, step, slot)
 *   gauss:  optional per-particle normals (3*N doubles, sorted position
 *           order); NULL draws orc_normal(seed, step, j, k)
 *   has_alpha=0 uses sin=1, cos=0 as the reference does when alpha is absent */
int orc_simple_mpcd_step(const orc_grid *g, int N, const int *cell_count,
                         const int *cell_start, double *vel, const int *species,
                         int has_alpha, double alpha, int thermostat, double T,
                         int hydro, uint64_t seed, uint64_t step,
                         const double *axes, const double *gauss);
/* wall_mpcd_step, src/mpcd.f90:193-337 (Lamura virtual particles) */
int orc_wall_mpcd_step(const orc_grid *g, int N, const int *cell_count,
                       const int *cell_start, double *vel,
                       int has_wall, const double wall_temperature[2],
                       const double wall_v[6], const int wall_n[2],
                       int thermostat, double bulk_temperature,
                       int has_alpha, double alpha, int keep_cell_v,
                       uint64_t seed, uint64_t step);
/* compute_temperature, src/mpcd.f90:342-407 */
double orc_compute_temperature(const orc_grid *g, int N, const int *cell_count,
                               const int *cell_start, const double *vel,
                               const int *species);
/* rescale_cells, src/mpcd.f90:748-801 */
void orc_rescale_cells(const orc_grid *g, int N, const int *cell_count,
                       const int *cell_start, double *vel, const int *species,
                       double T);
/* mpcd_stream_periodic, src/mpcd.f90:440-457 */
void orc_mpcd_stream_periodic(const orc_grid *g, int N, double *pos, double *vel,
                              int *image, double dt);
/* mpcd_stream_xforce_yzwall + yzwall_collision, src/mpcd.f90:464-589 */
void orc_mpcd_stream_xforce_yzwall(const orc_grid *g, int N, double *pos,
                                   double *vel, int *flags, double dt, double gx);
/* mpcd_stream_nogravity_zwall, src/mpcd.f90:702-745 */
void orc_mpcd_stream_nogravity_zwall(const orc_grid *g, int N, double *pos,
                                     double *vel, const double *force, int *flags,
                                     double dt);
/* bulk_reaction, src/mpcd.f90:605-643 */
void orc_bulk_reaction(const orc_grid *g, int N, const int *cell_count,
                       const int *cell_start, const unsigned char *is_reac,
                       int *species, int from, int to, double rate, double tau,
                       uint64_t seed, uint64_t step);
/* bulk_reaction_endothermic, src/mpcd.f90:645-700 */
void orc_bulk_reaction_endothermic(const orc_grid *g, int N, const int *cell_count,
                                   const int *cell_start, const unsigned char *is_reac,
                                   int *species, double *vel, int from, int to,
                                   double rate, double tau, double delta_u,
                                   uint64_t seed, uint64_t step);

/* ---------------- MD (src/md.f90) ---------------- */
void orc_md_pos(int N, double *pos, const double *vel, const double *force, double dt);
void orc_md_vel(int N, double *vel, const double *force, const double *force_old,
                int *flags, double dt);
void orc_cell_md_pos(const orc_grid *g, const int *cell_count, const int *cell_start,
                     const unsigned char *is_md, double *pos, const double *vel,
                     const double *force, double dt, int md_flag);
void orc_cell_md_vel(const orc_grid *g, const int *cell_count, const int *cell_start,
                     const unsigned char *is_md, double *vel, const double *force,
                     const double *force_old, int *flags, double dt, int md_flag);
/* cell_md_pos_ywall (dim=1) / cell_md_pos_zwall (dim=2), src/md.f90:104-200 */
void orc_cell_md_pos_wall(const orc_grid *g, int dim, const int *cell_count,
                          const int *cell_start, const unsigned char *is_md,
                          double *pos, double *vel, const double *force, double dt,
                          int md_flag);
void orc_apply_pbc(int N, double *pos, int *image, const double edges[3]);
double orc_maximum_displacement(int N, const double *pos, const double *pos_old,
                                const int *species);
double orc_cell_maximum_displacement(const orc_grid *g, const int *cell_count,
                                     const int *cell_start, const unsigned char *is_md,
                                     const double *pos, const double *pos_old,
                                     const int *species, double delta_t);
void orc_rel_pos(const double x[3], const double y[3], const double L[3], double r[3]);
/* rattle_dimer_pos / rattle_dimer_vel, src/md.f90:265-319.  pos/vel/pos_rattle
 * hold the two dimer beads; mass1/mass2 are mass(species(1)), mass(species(2)) */
void orc_rattle_dimer_pos(double *pos, double *vel, const double *pos_rattle,
                          double mass1, double mass2, double d, double dt,
                          const double edges[3]);
void orc_rattle_dimer_vel(const double *pos, double *vel, double mass1, double mass2,
                          double d, double dt, const double edges[3]);
/* colloid velocity-Verlet halves, programs/single_dimer_pbc.f90:311-315,356-359;
 * mass[k] is the per-particle mass used there */
void orc_colloid_vv_pos(int C, double *pos, const double *vel, const double *force,
                        const double *mass, double dt);
void orc_colloid_vv_vel(int C, double *vel, const double *force,
                        const double *force_old, const double *mass, double dt);

/* ---------------- Lennard-Jones (src/interaction.f90) ---------------- */
#define ORC_MAX_SPECIES 4
typedef struct {
    int n1, n2;
    /* column-major (n1,n2): t[(s1-1) + n1*(s2-1)] */
    double epsilon[ORC_MAX_SPECIES * ORC_MAX_SPECIES];
    double sigma[ORC_MAX_SPECIES * ORC_MAX_SPECIES];
    double sigma_sq[ORC_MAX_SPECIES * ORC_MAX_SPECIES];
    double cut[ORC_MAX_SPECIES * ORC_MAX_SPECIES];
    double cut_sq[ORC_MAX_SPECIES * ORC_MAX_SPECIES];
    double cut_energy[ORC_MAX_SPECIES * ORC_MAX_SPECIES];
} orc_lj;
void orc_lj_init(orc_lj *lj, int n1, int n2, const double *epsilon,
                 const double *sigma, const double *cut);
double orc_sixth(double x);
void orc_lj_force(const double d[3], double r_sq, double epsilon, double sigma, double f[3]);
double orc_lj_energy(double r_sq, double epsilon, double sigma, double cut_energy);

/* ---------------- neighbor list (src/neighbor_list.f90) ---------------- */
/* make_stencil: writes up to cap offsets (3 ints each), returns the count */
int orc_make_stencil(double a, double cut, int *stencil, int cap);
/* update_list: list is (Nmax, C) column-major 1-based; n[C].  Returns 0, or
 * -1 when an entry would exceed Nmax (the reference's error stop). */
int orc_update_list(const orc_grid *g, int C, const double *cpos, const int *cspecies,
                    int N, const double *spos, const int *sspecies,
                    const int *cell_count, const int *cell_start,
                    const int *stencil, int n_stencil, double radius,
                    const orc_lj *lj, int Nmax, int *list, int *n,
                    unsigned char *is_md, unsigned char *is_reac);
/* compute_force, src/neighbor_list.f90:159-225.  Returns the energy. */
double orc_compute_force(int C, const double *cpos, const int *cspecies, double *cforce,
                         int N, const double *spos, const int *sspecies,
                         double *sforce, int *sflags, const int *list, const int *n,
                         int Nmax, const double L[3], const orc_lj *lj);
/* compute_force_n2, src/neighbor_list.f90:227-264 */
double orc_compute_force_n2(int C, const double *pos, const int *species, double *force,
                            const double L[3], const orc_lj *lj);

/* ---------------- program-local loops (programs/single_dimer_pbc.f90) ---------------- */
void orc_flag_particles_nl(int n1, const int *list1, const double *c1pos,
                           const double *spos, const int *species, int *flags,
                           const double edges[3], double cut_sq_11);
void orc_change_species(int N, const double *c1pos, const double *c2pos,
                        const double *spos, int *species, int *flags,
                        const double edges[3], double cut_sq_11, double cut_sq_12,
                        double prob, uint64_t seed, uint64_t step);
/* refuel with far = (L1*0.45)**2 evaluated in single precision as written */
void orc_refuel(int N, const double *c1pos, const double *c2pos, const double *spos,
                int *species, const double edges[3], int L1);
void orc_n_solvent(int N, const int *species, int n_species, int *counts);
void orc_cylindrical_shell_histogram(const double x1[3], const double x2[3],
                                     const double L[3], int bin_species, double r_min,
                                     double r_max, int N, const double *spos,
                                     const int *species, double xmin, double dx,
                                     int nbins, double *hist);
/* sums used by the per-interval observables: out = {sum v^2, sum vx, sum vy, sum vz} */
void orc_velocity_sums(int N, const double *vel, double out[4]);
/* random_placement, src/particle_system.f90:250-302 with the Philox stream */
void orc_random_placement(int N, double *pos, const int *species, const double L[3],
                          int C, const double *cpos, const int *cspecies,
                          const orc_lj *lj, uint64_t seed);
/* Maxwell velocities with zero total momentum (programs/single_dimer_pbc.f90:240-245) */
void orc_maxwell_velocities(int N, double *vel, double T, uint64_t seed);

/* ---------------- program drivers ---------------- */
/* bulk fluid loop of test/setup_bulk_decay.f90:112-121: per interval
 * simple_mpcd_step -> mpcd_stream_periodic(tau) -> random_shift -> sort.
 * step_base is the RNG step of the first interval; interval i uses
 * step_base + 2*i for the collision and step_base + 2*i + 1 for the shift. */
void orc_bulk_run(const orc_grid *g_in, int N, int n_intervals, double tau,
                  double alpha, int has_alpha, uint64_t seed, uint64_t step_base,
                  double *pos, int *image, double *vel, int *id, int *species,
                  int *flags, int *cell_count, int *cell_start, double origin_out[3]);

#ifdef __cplusplus
}
#endif
/* ---------------- rigid-body colloids (src/md.f90:321-700) ---------------- */
/* links: n_link pairs of 1-based particle numbers; im: 6 N ints of scratch.
 * Returns the reference's rattle_i at exit (1001: no convergence). */
int orc_rattle_body_pos(int N, double *pos, double *vel, double *pos_rattle, const int *species,
                        const double *mass, const int *links, const double *dist, int n_link, double dt,
                        const double *edges, double precision, int *im);
int orc_rattle_body_vel(int N, double *pos, double *vel, const int *species, const double *mass,
                        const int *links, const double *dist, int n_link, const double *edges,
                        double precision, int *im);
double orc_elastic_network(const double *pos, double *force, const int *links, const double *dist, int n_link,
                           double kel, const double *edges);
/* rigid body state st[26] = mass, pos3, vel3, force3, q4 (s,x,y,z), L3, torque3, I_body3, omega_body3 */
void orc_rigid_body_init(const double *pos, const double *vel, const int *image, const int *species,
                         const double *mass_table, int i_start, int i_stop, const double *edges, double *st,
                         double *pos_body);
void orc_rigid_body_force_torque(const double *force, int i_start, int i_stop, double *st, const double *pos_body);
int orc_rigid_body_vv1(double *pos, int i_start, int i_stop, double *st, const double *pos_body, double dt,
                       double treshold, const double *edges);
void orc_rigid_body_vv2(double *vel, int i_start, int i_stop, double *st, const double *pos_body, double dt);

#endif
