/*
 * Program-local solvent loops of programs/single_dimer_pbc.f90 (reactions,
 * observables), initial conditions, and the bulk-fluid interval loop of
 * test/setup_bulk_decay.f90.  Test infrastructure only (oracle).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "rmpcd_oracle.h"

static double dot3(const double a[3], const double b[3])
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* flag_particles_nl, programs/single_dimer_pbc.f90:493-509 */
void orc_flag_particles_nl(int n1, const int *list1, const double *c1pos,
                           const double *spos, const int *species, int *flags,
                           const double edges[3], double cut_sq_11)
{
    for (int s = 0; s < n1; s++) {
        int r = list1[s] - 1;
        if (species[r] == 1) {
            double x[3];
            orc_rel_pos(c1pos, spos + 3 * (size_t)r, edges, x);
            double d = dot3(x, x);
            if (d < cut_sq_11) flags[r] |= (1 << ORC_REAC_BIT);
        }
    }
}

/* change_species, programs/single_dimer_pbc.f90:511-542.  The uniform for
 * particle m is Philox(seed, step, m, REACT). */
void orc_change_species(int N, const double *c1pos, const double *c2pos,
                        const double *spos, int *species, int *flags,
                        const double edges[3], double cut_sq_11, double cut_sq_12,
                        double prob, uint64_t seed, uint64_t step)
{
#pragma omp parallel for schedule(static)
    for (int m = 0; m < N; m++) {
        if ((flags[m] >> ORC_REAC_BIT) & 1) {
            double x[3];
            orc_rel_pos(c1pos, spos + 3 * (size_t)m, edges, x);
            double dC = dot3(x, x);
            orc_rel_pos(c2pos, spos + 3 * (size_t)m, edges, x);
            double dN = dot3(x, x);
            if ((dC > cut_sq_11) && (dN > cut_sq_12)) {
                double u[2];
                orc_rng_u2(seed, step, (uint32_t)m, ORC_RNG_REACT, 0, u);
                if (u[0] <= prob) species[m] = 2;
                flags[m] &= ~(1 << ORC_REAC_BIT);
            }
        }
    }
}

/* refuel, programs/single_dimer_pbc.f90:544-565.  far = (L(1)*0.45)**2 is a
 * default-real (single precision) expression in the reference. */
void orc_refuel(int N, const double *c1pos, const double *c2pos, const double *spos,
                int *species, const double edges[3], int L1)
{
    volatile float lf = (float)L1 * 0.45f;
    volatile float farf = lf * lf;
    double far = (double)farf;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; n++) {
        if (species[n] == 2) {
            double x[3];
            orc_rel_pos(c1pos, spos + 3 * (size_t)n, edges, x);
            double dC = dot3(x, x);
            orc_rel_pos(c2pos, spos + 3 * (size_t)n, edges, x);
            double dN = dot3(x, x);
            if ((dC > far) && (dN > far)) species[n] = 1;
        }
    }
}

/* n_solvent count, programs/single_dimer_pbc.f90:432-437 */
void orc_n_solvent(int N, const int *species, int n_species, int *counts)
{
    for (int j = 0; j < n_species; j++) counts[j] = 0;
    for (int k = 0; k < N; k++) {
        int j = species[k];
        if (j >= 1 && j <= n_species) counts[j - 1]++;
    }
}

/* compute_cylindrical_shell_histogram, src/particle_system.f90:412-445, with
 * histogram_t%bin, src/common.f90:248-266 */
void orc_cylindrical_shell_histogram(const double x1[3], const double x2[3],
                                     const double L[3], int bin_species, double r_min,
                                     double r_max, int N, const double *spos,
                                     const int *species, double xmin, double dx,
                                     int nbins, double *hist)
{
    double r_min_sq = r_min * r_min, r_max_sq = r_max * r_max;
    double uz[3];
    orc_rel_pos(x2, x1, L, uz);
    double norm = sqrt(dot3(uz, uz));
    for (int k = 0; k < 3; k++) uz[k] = uz[k] / norm;
    for (int i = 0; i < N; i++) {
        if (species[i] != bin_species) continue;
        double dxv[3];
        orc_rel_pos(spos + 3 * (size_t)i, x1, L, dxv);
        double elevation = dot3(uz, dxv);
        for (int k = 0; k < 3; k++) dxv[k] = dxv[k] - elevation * uz[k];
        double nn = dot3(dxv, dxv);
        if ((nn > r_min_sq) && (nn < r_max_sq)) {
            int idx = (int)floor((elevation - xmin) / dx) + 1;
            if ((idx > 0) && (idx <= nbins)) hist[idx - 1] = hist[idx - 1] + 1;
        }
    }
}

void orc_velocity_sums(int N, const double *vel, double out[4])
{
    double s2 = 0, sx = 0, sy = 0, sz = 0;
    for (int i = 0; i < N; i++) {
        const double *v = vel + 3 * (size_t)i;
        s2 = s2 + v[0] * v[0];
        s2 = s2 + v[1] * v[1];
        s2 = s2 + v[2] * v[2];
        sx = sx + v[0];
        sy = sy + v[1];
        sz = sz + v[2];
    }
    out[0] = s2; out[1] = sx; out[2] = sy; out[3] = sz;
}

/* random_placement, src/particle_system.f90:250-302; attempt a of particle i
 * uses Philox(seed, 0, i, PLACE, 2a) for x,y and (.., 2a+1) for z */
void orc_random_placement(int N, double *pos, const int *species, const double L[3],
                          int C, const double *cpos, const int *cspecies,
                          const orc_lj *lj, uint64_t seed)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        int s1 = species ? species[i] : 1;
        double x[3] = {0, 0, 0};
        for (uint32_t a = 0; a < (1u << 20); a++) {
            double u[2], w[2];
            orc_rng_u2(seed, 0, (uint32_t)i, ORC_RNG_PLACE, 2 * a, u);
            orc_rng_u2(seed, 0, (uint32_t)i, ORC_RNG_PLACE, 2 * a + 1, w);
            x[0] = u[0] * L[0];
            x[1] = u[1] * L[1];
            x[2] = w[0] * L[2];
            int tooclose = 0;
            for (int j = 0; j < C && lj; j++) {
                int s2 = cspecies[j];
                double r[3];
                orc_rel_pos(x, cpos + 3 * (size_t)j, L, r);
                double rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                if (rsq < lj->cut_sq[(s1 - 1) + lj->n1 * (s2 - 1)]) {
                    tooclose = 1;
                    break;
                }
            }
            if (!tooclose) break;
        }
        for (int k = 0; k < 3; k++) pos[3 * (size_t)i + k] = x[k];
    }
}

/* Maxwell velocities, programs/single_dimer_pbc.f90:240-245: normal * sqrt(T)
 * then subtraction of sum(vel, dim=2)/Nmax.  Component k of particle i is
 * Leva-normal on Philox(seed, step=0, i, GAUSS, sub=k) -- the same mapping the
 * collision uses, on a different step. */
void orc_maxwell_velocities(int N, double *vel, double T, uint64_t seed)
{
    double st = sqrt(T);
    const uint64_t init_step = 0xFFFFFFFFFFFFFFFFull;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++)
            vel[3 * (size_t)i + k] = orc_normal(seed, init_step, (uint32_t)i, (uint32_t)k) * st;
    double s[3] = {0, 0, 0};
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++) s[k] = s[k] + vel[3 * (size_t)i + k];
    for (int k = 0; k < 3; k++) s[k] = s[k] / N;
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++) vel[3 * (size_t)i + k] = vel[3 * (size_t)i + k] - s[k];
}

void orc_bulk_run(const orc_grid *g_in, int N, int n_intervals, double tau,
                  double alpha, int has_alpha, uint64_t seed, uint64_t step_base,
                  double *pos, int *image, double *vel, int *id, int *species,
                  int *flags, int *cell_count, int *cell_start, double origin_out[3])
{
    orc_grid g = *g_in;
    for (int it = 0; it < n_intervals; it++) {
        uint64_t st = step_base + 2 * (uint64_t)it;
        orc_simple_mpcd_step(&g, N, cell_count, cell_start, vel, species, has_alpha,
                             alpha, 0, 0.0, 1, seed, st, NULL, NULL);
        orc_mpcd_stream_periodic(&g, N, pos, vel, image, tau);
        orc_random_shift_values(seed, st + 1, g.origin);
        orc_sort(&g, N, cell_count, cell_start, pos, NULL, image, vel, NULL, NULL,
                 id, species, flags, NULL);
    }
    for (int k = 0; k < 3; k++) origin_out[k] = g.origin[k];
}
