/*
 * Velocity-Verlet halves, PBC wrap, displacement bounds and dimer RATTLE,
 * restated from src/md.f90, src/particle_system.f90 and
 * programs/single_dimer_pbc.f90.  Test infrastructure only (oracle).
 */
#include <math.h>
#include "rmpcd_oracle.h"

/* rel_pos, src/common.f90:162-178 */
void orc_rel_pos(const double x[3], const double y[3], const double L[3], double r[3])
{
    for (int k = 0; k < 3; k++) {
        r[k] = x[k] - y[k];
        if (r[k] < -0.5 * L[k]) r[k] = r[k] + L[k];
        else if (r[k] > 0.5 * L[k]) r[k] = r[k] - L[k];
    }
}

/* md_pos, src/md.f90:61-77 */
void orc_md_pos(int N, double *pos, const double *vel, const double *force, double dt)
{
    double dt_sq = dt * dt / 2;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++) {
            size_t j = 3 * (size_t)i + k;
            pos[j] = pos[j] + dt * vel[j] + dt_sq * force[j];
        }
}

/* md_vel, src/md.f90:219-237 */
void orc_md_vel(int N, double *vel, const double *force, const double *force_old,
                int *flags, double dt)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        if (!((flags[i] >> ORC_WALL_BIT) & 1)) {
            for (int k = 0; k < 3; k++) {
                size_t j = 3 * (size_t)i + k;
                vel[j] = vel[j] + dt * (force[j] + force_old[j]) / 2;
            }
        } else {
            flags[i] &= ~(1 << ORC_WALL_BIT);
        }
    }
}

/* cell_md_pos, src/md.f90:79-102 */
void orc_cell_md_pos(const orc_grid *g, const int *cell_count, const int *cell_start,
                     const unsigned char *is_md, double *pos, const double *vel,
                     const double *force, double dt, int md_flag)
{
    double dt_sq = dt * dt / 2;
#pragma omp parallel for schedule(static)
    for (int s = 0; s < g->S; s++) {
        if ((is_md[s] != 0) == (md_flag != 0)) {
            for (int i = cell_start[s] - 1; i < cell_start[s] - 1 + cell_count[s]; i++)
                for (int k = 0; k < 3; k++) {
                    size_t j = 3 * (size_t)i + k;
                    pos[j] = pos[j] + dt * vel[j] + dt_sq * force[j];
                }
        }
    }
}

/* cell_md_vel, src/md.f90:239-263 */
void orc_cell_md_vel(const orc_grid *g, const int *cell_count, const int *cell_start,
                     const unsigned char *is_md, double *vel, const double *force,
                     const double *force_old, int *flags, double dt, int md_flag)
{
#pragma omp parallel for schedule(static)
    for (int s = 0; s < g->S; s++) {
        if ((is_md[s] != 0) == (md_flag != 0)) {
            for (int i = cell_start[s] - 1; i < cell_start[s] - 1 + cell_count[s]; i++) {
                if (!((flags[i] >> ORC_WALL_BIT) & 1)) {
                    for (int k = 0; k < 3; k++) {
                        size_t j = 3 * (size_t)i + k;
                        vel[j] = vel[j] + dt * (force[j] + force_old[j]) / 2;
                    }
                } else {
                    flags[i] &= ~(1 << ORC_WALL_BIT);
                }
            }
        }
    }
}

/* cell_md_pos_ywall / cell_md_pos_zwall, src/md.f90:104-200 */
void orc_cell_md_pos_wall(const orc_grid *g, int dim, const int *cell_count,
                          const int *cell_start, const unsigned char *is_md,
                          double *pos, double *vel, const double *force, double dt,
                          int md_flag)
{
    double dt_sq = dt * dt / 2;
    double Lw = g->edges[dim];
    int bc = g->bc[dim];
#pragma omp parallel for schedule(static)
    for (int s = 0; s < g->S; s++) {
        if ((is_md[s] != 0) != (md_flag != 0)) continue;
        for (int i = cell_start[s] - 1; i < cell_start[s] - 1 + cell_count[s]; i++) {
            double v[3], x[3];
            for (int k = 0; k < 3; k++) {
                size_t j = 3 * (size_t)i + k;
                v[k] = vel[j];
                x[k] = pos[j] + dt * v[k] + dt_sq * force[j];
            }
            int collide = 0;
            double overtime = 0;
            if (x[dim] < 0.0) {
                collide = 1;
                overtime = x[dim] / v[dim];
            } else if (x[dim] > Lw) {
                collide = 1;
                overtime = (x[dim] - Lw) / v[dim];
            }
            if (collide) {
                if (bc == ORC_BOUNCE_BACK_BC) {
                    for (int k = 0; k < 3; k++) v[k] = -v[k];
                    for (int k = 0; k < 3; k++) x[k] = x[k] + 2 * overtime * v[k];
                } else if (bc == ORC_SPECULAR_BC) {
                    v[dim] = -v[dim];
                    x[dim] = x[dim] + 2 * overtime * v[dim];
                }
                for (int k = 0; k < 3; k++) vel[3 * (size_t)i + k] = v[k];
            }
            for (int k = 0; k < 3; k++) pos[3 * (size_t)i + k] = x[k];
        }
    }
}

/* apply_pbc, src/md.f90:202-217 */
void orc_apply_pbc(int N, double *pos, int *image, const double edges[3])
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++)
        for (int k = 0; k < 3; k++) {
            size_t j = 3 * (size_t)i + k;
            int jump = (int)floor(pos[j] / edges[k]);
            image[j] = image[j] + jump;
            pos[j] = pos[j] - jump * edges[k];
        }
}

/* maximum_displacement, src/particle_system.f90:357-378 */
double orc_maximum_displacement(int N, const double *pos, const double *pos_old,
                                const int *species)
{
    double rmax_sq = 0;
#pragma omp parallel for reduction(max:rmax_sq) schedule(static)
    for (int i = 0; i < N; i++) {
        if (species[i] >= 0) {
            double d0 = pos[3 * (size_t)i] - pos_old[3 * (size_t)i];
            double d1 = pos[3 * (size_t)i + 1] - pos_old[3 * (size_t)i + 1];
            double d2 = pos[3 * (size_t)i + 2] - pos_old[3 * (size_t)i + 2];
            double r_sq = d0 * d0 + d1 * d1 + d2 * d2;
            rmax_sq = rmax_sq > r_sq ? rmax_sq : r_sq;
        }
    }
    return sqrt(rmax_sq);
}

/* cell_maximum_displacement, src/particle_system.f90:380-410 */
double orc_cell_maximum_displacement(const orc_grid *g, const int *cell_count,
                                     const int *cell_start, const unsigned char *is_md,
                                     const double *pos, const double *pos_old,
                                     const int *species, double delta_t)
{
    double rmax_sq = 0;
    for (int s = 0; s < g->S; s++) {
        if (!is_md[s]) continue;
        double local = 0;
        for (int i = cell_start[s] - 1; i < cell_start[s] - 1 + cell_count[s]; i++) {
            if (species[i] >= 0) {
                double d0 = pos[3 * (size_t)i] - pos_old[3 * (size_t)i];
                double d1 = pos[3 * (size_t)i + 1] - pos_old[3 * (size_t)i + 1];
                double d2 = pos[3 * (size_t)i + 2] - pos_old[3 * (size_t)i + 2];
                double r_sq = d0 * d0 + d1 * d1 + d2 * d2;
                if (r_sq > local) local = r_sq;
            }
        }
        rmax_sq = rmax_sq > local ? rmax_sq : local;
    }
    double a = sqrt(rmax_sq), b = g->max_v * delta_t;
    return a > b ? a : b;
}

static double dot3(const double a[3], const double b[3])
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* rattle_dimer_pos, src/md.f90:265-296 */
void orc_rattle_dimer_pos(double *pos, double *vel, const double *pos_rattle,
                          double mass1, double mass2, double d, double dt,
                          const double edges[3])
{
    double r[3], s[3];
    orc_rel_pos(pos_rattle, pos_rattle + 3, edges, r);
    orc_rel_pos(pos, pos + 3, edges, s);
    double inv_mass = 1 / mass1 + 1 / mass2;
    double rsq = dot3(r, r);
    double ssq = dot3(s, s);
    double rs = dot3(r, s);
    double g = rs - sqrt(rs * rs - rsq * (ssq - d * d));
    g = g / (dt * inv_mass * rsq);
    for (int k = 0; k < 3; k++) {
        pos[k] = pos[k] - g * dt * r[k] / mass1;
        pos[3 + k] = pos[3 + k] + g * dt * r[k] / mass2;
    }
    for (int k = 0; k < 3; k++) {
        vel[k] = vel[k] - g * r[k] / mass1;
        vel[3 + k] = vel[3 + k] + g * r[k] / mass2;
    }
}

/* rattle_dimer_vel, src/md.f90:298-319 */
void orc_rattle_dimer_vel(const double *pos, double *vel, double mass1, double mass2,
                          double d, double dt, const double edges[3])
{
    (void)dt;
    double s[3], dv[3];
    double inv_mass = 1 / mass1 + 1 / mass2;
    orc_rel_pos(pos, pos + 3, edges, s);
    for (int k = 0; k < 3; k++) dv[k] = vel[k] - vel[3 + k];
    double kk = dot3(dv, s) / (d * d * inv_mass);
    for (int k = 0; k < 3; k++) {
        vel[k] = vel[k] - kk * s[k] / mass1;
        vel[3 + k] = vel[3 + k] + kk * s[k] / mass2;
    }
}

/* colloid VV position half, programs/single_dimer_pbc.f90:312-315 */
void orc_colloid_vv_pos(int C, double *pos, const double *vel, const double *force,
                        const double *mass, double dt)
{
    for (int i = 0; i < C; i++)
        for (int k = 0; k < 3; k++) {
            size_t j = 3 * (size_t)i + k;
            pos[j] = pos[j] + dt * vel[j] + dt * dt * force[j] / (2 * mass[i]);
        }
}

/* colloid VV velocity half, programs/single_dimer_pbc.f90:356-359 */
void orc_colloid_vv_vel(int C, double *vel, const double *force,
                        const double *force_old, const double *mass, double dt)
{
    for (int i = 0; i < C; i++)
        for (int k = 0; k < 3; k++) {
            size_t j = 3 * (size_t)i + k;
            vel[j] = vel[j] + dt * (force[j] + force_old[j]) / (2 * mass[i]);
        }
}
