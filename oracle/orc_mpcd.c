/*
 * MPCD collision, temperature, rescaling, streaming and bulk reactions,
 * restated from src/mpcd.f90.  Test infrastructure only (oracle).
 * Expressions keep the Fortran association order; compile with
 * -ffp-contract=off.
 */
#include <math.h>
#include <float.h>
#include "rmpcd_oracle.h"

/* Rotation matrix of simple_mpcd_step, src/mpcd.f90:163-171.  The Fortran
 * reshape fills column-major, so om[r][c] below is omega(r+1, c+1). */
static void srd_omega(const double vec[3], double sin_a, double cos_a, double om[3][3])
{
    double omc = 1 - cos_a;
    om[0][0] = cos_a + vec[0] * vec[0] * omc;
    om[1][0] = vec[0] * vec[1] * omc - vec[2] * sin_a;
    om[2][0] = vec[0] * vec[2] * omc + vec[1] * sin_a;
    om[0][1] = vec[1] * vec[0] * omc + vec[2] * sin_a;
    om[1][1] = cos_a + vec[1] * vec[1] * omc;
    om[2][1] = vec[1] * vec[2] * omc - vec[0] * sin_a;
    om[0][2] = vec[2] * vec[0] * omc - vec[1] * sin_a;
    om[1][2] = vec[2] * vec[1] * omc + vec[0] * sin_a;
    om[2][2] = cos_a + vec[2] * vec[2] * omc;
}

/* vel = local_v + matmul(omega, vel - local_v), matmul accumulating k = 1..3 */
static void srd_rotate(double *v, const double lv[3], double om[3][3])
{
    double d0 = v[0] - lv[0], d1 = v[1] - lv[1], d2 = v[2] - lv[2];
    double r[3];
    for (int r_ = 0; r_ < 3; r_++) r[r_] = om[r_][0] * d0 + om[r_][1] * d1 + om[r_][2] * d2;
    v[0] = lv[0] + r[0];
    v[1] = lv[1] + r[1];
    v[2] = lv[2] + r[2];
}

int orc_simple_mpcd_step(const orc_grid *g, int N, const int *cell_count,
                         const int *cell_start, double *vel, const int *species,
                         int has_alpha, double alpha, int thermostat, double T,
                         int hydro, uint64_t seed, uint64_t step,
                         const double *axes, const double *gauss)
{
    (void)N;
    int do_thermostat = thermostat ? 1 : 0;
    int do_hydro = hydro ? 1 : 0;
    if (!do_hydro && !do_thermostat) return -1;
    double t_factor = do_thermostat ? sqrt(T) : 0.0;
    double sin_a = 1, cos_a = 0;
    if (has_alpha) {
        sin_a = sin(alpha);
        cos_a = cos(alpha);
    }

#pragma omp parallel for schedule(static)
    for (int s = 0; s < g->S; s++) {
        if (cell_count[s] <= 1) continue;
        int start = cell_start[s] - 1;
        int n = cell_count[s];
        int n_eff = 0;
        double lv[3] = {0, 0, 0};
        for (int i = start; i < start + n; i++) {
            if (species[i] > 0) {
                for (int k = 0; k < 3; k++) lv[k] = lv[k] + vel[3 * (size_t)i + k];
                n_eff++;
            }
        }
        if (n_eff <= 1) continue;
        for (int k = 0; k < 3; k++) lv[k] = lv[k] / n_eff;

        if (do_thermostat) {
            double vv[3] = {0, 0, 0};
            for (int i = start; i < start + n; i++) {
                if (species[i] <= 0) continue;
                for (int k = 0; k < 3; k++) {
                    double z = gauss ? gauss[3 * (size_t)i + k] : orc_normal(seed, step, (uint32_t)i, (uint32_t)k);
                    vel[3 * (size_t)i + k] = z * t_factor;
                    vv[k] = vv[k] + vel[3 * (size_t)i + k];
                }
            }
            for (int k = 0; k < 3; k++) vv[k] = lv[k] - vv[k] / n_eff;
            if (do_hydro) {
                for (int i = start; i < start + n; i++) {
                    if (species[i] <= 0) continue;
                    for (int k = 0; k < 3; k++) vel[3 * (size_t)i + k] = vel[3 * (size_t)i + k] + vv[k];
                }
            }
        } else {
            double vec[3], om[3][3];
            if (axes) {
                vec[0] = axes[3 * (size_t)s];
                vec[1] = axes[3 * (size_t)s + 1];
                vec[2] = axes[3 * (size_t)s + 2];
            } else {
                orc_rand_sphere(seed, step, (uint32_t)s, vec);
            }
            srd_omega(vec, sin_a, cos_a, om);
            for (int i = start; i < start + n; i++) srd_rotate(vel + 3 * (size_t)i, lv, om);
        }
    }
    return 0;
}

int orc_wall_mpcd_step(const orc_grid *g, int N, const int *cell_count,
                       const int *cell_start, double *vel,
                       int has_wall, const double wall_temperature[2],
                       const double wall_v[6], const int wall_n[2],
                       int thermostat, double bulk_temperature,
                       int has_alpha, double alpha, int keep_cell_v,
                       uint64_t seed, uint64_t step)
{
    (void)N;
    (void)wall_v; /* accepted but unused by the reference rule */
    int do_thermostat = thermostat ? 1 : 0;
    int do_cell_v = keep_cell_v ? 1 : 0;
    if (!do_cell_v && !do_thermostat) return -1;
    double t_factor = do_thermostat ? sqrt(bulk_temperature) : 0.0;
    double sin_a = 1, cos_a = 0;
    if (has_alpha) {
        sin_a = sin(alpha);
        cos_a = cos(alpha);
    }
    for (int s = 0; s < g->S; s++) {
        if (cell_count[s] <= 1) continue;
        int start = cell_start[s] - 1;
        int n = cell_count[s];
        int n_virtual = 0;
        int cell[3];
        orc_compact_h_to_p(s, g->M, cell);
        int wall_idx = -1;
        if (has_wall && cell[2] + 1 == 1) wall_idx = 0;
        else if (has_wall && cell[2] + 1 == g->L[2]) wall_idx = 1;
        double virtual_v[3] = {0, 0, 0};
        if (wall_idx >= 0 && n < wall_n[wall_idx]) {
            n_virtual = wall_n[wall_idx] - n;
            for (int k = 0; k < 3; k++) virtual_v[k] = orc_normal(seed, step, (uint32_t)s, (uint32_t)(3 + k));
            double f = sqrt(n_virtual * wall_temperature[wall_idx]);
            for (int k = 0; k < 3; k++) virtual_v[k] = virtual_v[k] * f;
        }
        double lv[3] = {0, 0, 0};
        for (int i = start; i < start + n; i++)
            for (int k = 0; k < 3; k++) lv[k] = lv[k] + vel[3 * (size_t)i + k];
        if (n_virtual > 0) {
            for (int k = 0; k < 3; k++) lv[k] = (lv[k] + virtual_v[k]) / wall_n[wall_idx];
        } else {
            for (int k = 0; k < 3; k++) lv[k] = lv[k] / n;
        }
        if (do_thermostat) {
            double vv[3] = {0, 0, 0};
            for (int i = start; i < start + n; i++) {
                for (int k = 0; k < 3; k++) {
                    double z = orc_normal(seed, step, (uint32_t)i, (uint32_t)k);
                    vel[3 * (size_t)i + k] = z * t_factor;
                    vv[k] = vv[k] + vel[3 * (size_t)i + k];
                }
            }
            if (do_cell_v) {
                for (int k = 0; k < 3; k++) vv[k] = lv[k] - vv[k] / (double)n;
                for (int i = start; i < start + n; i++)
                    for (int k = 0; k < 3; k++) vel[3 * (size_t)i + k] = vel[3 * (size_t)i + k] + vv[k];
            }
        } else {
            double vec[3], om[3][3];
            orc_rand_sphere(seed, step, (uint32_t)s, vec);
            srd_omega(vec, sin_a, cos_a, om);
            for (int i = start; i < start + n; i++) srd_rotate(vel + 3 * (size_t)i, lv, om);
        }
    }
    return 0;
}

double orc_compute_temperature(const orc_grid *g, int N, const int *cell_count,
                               const int *cell_start, const double *vel,
                               const int *species)
{
    (void)N;
    int count = 0;
    double te = 0;
#pragma omp parallel for reduction(+:count) reduction(+:te) schedule(static)
    for (int s = 0; s < g->S; s++) {
        if (cell_count[s] <= 1) continue;
        int start = cell_start[s] - 1;
        int n = cell_count[s];
        count = count + 1;
        int n_eff = 0;
        double lv[3] = {0, 0, 0};
        double kin = 0;
        for (int i = start; i < start + n; i++) {
            if (species[i] > 0) {
                for (int k = 0; k < 3; k++) lv[k] = lv[k] + vel[3 * (size_t)i + k];
                n_eff++;
            }
        }
        if (n_eff <= 1) continue;
        for (int k = 0; k < 3; k++) lv[k] = lv[k] / n;
        for (int i = start; i < start + n; i++) {
            if (species[i] > 0) {
                double d0 = vel[3 * (size_t)i] - lv[0];
                double d1 = vel[3 * (size_t)i + 1] - lv[1];
                double d2 = vel[3 * (size_t)i + 2] - lv[2];
                kin = kin + (d0 * d0 + d1 * d1 + d2 * d2);
            }
        }
        kin = kin / (double)(3 * (n_eff - 1));
        te = te + kin;
    }
    return te / count;
}

void orc_rescale_cells(const orc_grid *g, int N, const int *cell_count,
                       const int *cell_start, double *vel, const int *species,
                       double T)
{
    (void)N;
#pragma omp parallel for schedule(static)
    for (int s = 0; s < g->S; s++) {
        if (cell_count[s] <= 1) continue;
        int start = cell_start[s] - 1;
        int n = cell_count[s];
        int n_eff = 0;
        double lv[3] = {0, 0, 0};
        for (int i = start; i < start + n; i++) {
            if (species[i] > 0) {
                for (int k = 0; k < 3; k++) lv[k] = lv[k] + vel[3 * (size_t)i + k];
                n_eff++;
            }
        }
        if (n_eff <= 1) continue;
        for (int k = 0; k < 3; k++) lv[k] = lv[k] / n_eff;
        double kin = 0;
        for (int i = start; i < start + n; i++) {
            if (species[i] > 0) {
                double d0 = vel[3 * (size_t)i] - lv[0];
                double d1 = vel[3 * (size_t)i + 1] - lv[1];
                double d2 = vel[3 * (size_t)i + 2] - lv[2];
                kin = kin + (d0 * d0 + d1 * d1 + d2 * d2);
            }
        }
        double tf = sqrt((3 * (n_eff - 1)) * T / kin);
        for (int i = start; i < start + n; i++) {
            if (species[i] > 0)
                for (int k = 0; k < 3; k++)
                    vel[3 * (size_t)i + k] = lv[k] + tf * (vel[3 * (size_t)i + k] - lv[k]);
        }
    }
}

void orc_mpcd_stream_periodic(const orc_grid *g, int N, double *pos, double *vel,
                              int *image, double dt)
{
    const double *edges = g->edges;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        for (int k = 0; k < 3; k++) {
            double x = pos[3 * (size_t)i + k] + vel[3 * (size_t)i + k] * dt;
            int jump = (int)floor(x / edges[k]);
            image[3 * (size_t)i + k] += jump;
            pos[3 * (size_t)i + k] = x - jump * edges[k];
        }
    }
}

static int change_23(int i) { return i == 1 ? 2 : 1; } /* 0-based y=1, z=2 */

/* yzwall_collision, src/mpcd.f90:511-589 (0-based dims; the wall loop is
 * capped at 64 crossings so that degenerate NaN times cannot spin) */
static void yzwall_collision(const double x0[3], const double v0[3], double x[3],
                             double v[3], const double L[3], double t,
                             const int bc[3], double gx)
{
    double gvec[3] = {gx, 0, 0};
    int im[3] = {0, 0, 0};
    int coll_dim = -1;
    double t_collision = DBL_MAX;
    for (int i = 1; i <= 2; i++) {
        double tt;
        if (v0[i] > 0) {
            tt = (L[i] - x0[i]) / v0[i];
        } else {
            tt = -x0[i] / v0[i];
        }
        if ((tt > 0) && (tt < t_collision)) {
            t_collision = tt;
            coll_dim = i;
        }
    }
    if (coll_dim < 0) return;
    double t_remainder = t - t_collision;
    for (int k = 0; k < 3; k++) {
        x[k] = x0[k] + v0[k] * t_collision + gvec[k] * (t_collision * t_collision) / 2;
        v[k] = v0[k] + gvec[k] * t_collision;
    }
    for (int iter = 0; ; iter++) {
        if (bc[coll_dim] == ORC_BOUNCE_BACK_BC) {
            for (int k = 0; k < 3; k++) v[k] = -v[k];
        } else if (bc[coll_dim] == ORC_SPECULAR_BC) {
            v[coll_dim] = -v[coll_dim];
        } else if (bc[coll_dim] == ORC_PERIODIC_BC) {
            int jump = (int)floor(x[coll_dim] / L[coll_dim]);
            x[coll_dim] = x[coll_dim] - jump * L[coll_dim];
            im[coll_dim] = im[coll_dim] + jump;
        }
        if (iter >= 64) break;
        coll_dim = change_23(coll_dim);
        if (v[coll_dim] > 0) {
            t_collision = (L[coll_dim] - x[coll_dim]) / v[coll_dim];
        } else {
            t_collision = -x[coll_dim] / v[coll_dim];
        }
        if ((t_collision < 0) || (t_collision > t_remainder)) break;
        for (int k = 0; k < 3; k++) {
            x[k] = x[k] + v[k] * t_collision + gvec[k] * (t_collision * t_collision) / 2;
            v[k] = v[k] + gvec[k] * t_collision;
        }
        t_remainder = t_remainder - t_collision;
    }
    t_collision = t_remainder;
    for (int k = 0; k < 3; k++) {
        x[k] = x[k] + v[k] * t_collision + gvec[k] * (t_collision * t_collision) / 2 + im[k] * L[k];
        v[k] = v[k] + gvec[k] * t_collision;
    }
}

void orc_mpcd_stream_xforce_yzwall(const orc_grid *g, int N, double *pos,
                                   double *vel, int *flags, double dt, double gx)
{
    const double *L = g->edges;
    double gvec[3] = {gx, 0, 0};
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        double op[3], ov[3], np[3], nv[3];
        for (int k = 0; k < 3; k++) {
            op[k] = pos[3 * (size_t)i + k];
            ov[k] = vel[3 * (size_t)i + k];
        }
        for (int k = 0; k < 3; k++) {
            np[k] = op[k] + ov[k] * dt + gvec[k] * (dt * dt) / 2;
            nv[k] = ov[k];
        }
        int y_out = (np[1] < 0) || (np[1] > L[1]);
        int z_out = (np[2] < 0) || (np[2] > L[2]);
        if (((g->bc[1] == ORC_PERIODIC_BC) && z_out) ||
            ((g->bc[1] != ORC_PERIODIC_BC) && (y_out || z_out))) {
            yzwall_collision(op, ov, np, nv, L, dt, g->bc, gx);
            flags[i] |= (1 << ORC_WALL_BIT);
            for (int k = 0; k < 3; k++) vel[3 * (size_t)i + k] = nv[k];
        }
        for (int k = 0; k < 3; k++) pos[3 * (size_t)i + k] = np[k];
    }
}

void orc_mpcd_stream_nogravity_zwall(const orc_grid *g, int N, double *pos,
                                     double *vel, const double *force, int *flags,
                                     double dt)
{
    const double *L = g->edges;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        double op[3], ov[3], np[3], nv[3];
        for (int k = 0; k < 3; k++) {
            op[k] = pos[3 * (size_t)i + k];
            ov[k] = vel[3 * (size_t)i + k];
            np[k] = op[k] + ov[k] * dt + force[3 * (size_t)i + k] * (dt * dt) / 2;
        }
        int bounce = 0;
        double t_c = 0;
        if (np[2] < 0) {
            t_c = -op[2] / ov[2];
            bounce = 1;
        } else if (np[2] > L[2]) {
            t_c = (L[2] - op[2]) / ov[2];
            bounce = 1;
        } else {
            for (int k = 0; k < 3; k++) nv[k] = ov[k];
        }
        if (bounce) {
            for (int k = 0; k < 3; k++) {
                np[k] = np[k] - ov[k] * 2 * (dt - t_c);
                nv[k] = -ov[k];
            }
            flags[i] |= (1 << ORC_WALL_BIT);
        }
        for (int k = 0; k < 3; k++) {
            pos[3 * (size_t)i + k] = np[k];
            vel[3 * (size_t)i + k] = nv[k];
        }
    }
}

void orc_bulk_reaction(const orc_grid *g, int N, const int *cell_count,
                       const int *cell_start, const unsigned char *is_reac,
                       int *species, int from, int to, double rate, double tau,
                       uint64_t seed, uint64_t step)
{
    (void)N;
    for (int s = 0; s < g->S; s++) {
        if ((cell_count[s] <= 1) || !is_reac[s]) continue;
        int start = cell_start[s] - 1;
        int n = cell_count[s];
        double local_rate = 0;
        int pick = -1;
        for (int i = start; i < start + n; i++) {
            if (species[i] == from) {
                local_rate = local_rate + 1;
                pick = i;
            }
        }
        local_rate = local_rate * rate;
        double u[2];
        orc_rng_u2(seed, step, (uint32_t)s, ORC_RNG_BULK, 0, u);
        if (u[0] < (1 - exp(-local_rate * tau)) && pick >= 0) species[pick] = to;
    }
}

/* bulk_reaction_endothermic, src/mpcd.f90:645-700.  com_v is the plain mean of
 * the cell's velocities (:675-682), kin the sum of |v - com_v|^2 / 2 (:684-688),
 * with sum() over the three components taken left to right; the uniform is
 * drawn only when the cell can react (:690-692), and the rescale is
 * v = com_v + factor (v - com_v) with factor = sqrt((kin - delta_u) / kin)
 * (:693-698). */
void orc_bulk_reaction_endothermic(const orc_grid *g, int N, const int *cell_count,
                                   const int *cell_start, const unsigned char *is_reac,
                                   int *species, double *vel, int from, int to,
                                   double rate, double tau, double delta_u,
                                   uint64_t seed, uint64_t step)
{
    (void)N;
    for (int s = 0; s < g->S; s++) {
        if ((cell_count[s] <= 1) || !is_reac[s]) continue;
        int start = cell_start[s] - 1;
        int n = cell_count[s];
        double local_rate = 0;
        int pick = -1;
        double com_v[3] = {0, 0, 0};
        for (int i = start; i < start + n; i++) {
            if (species[i] == from) {
                local_rate = local_rate + 1;
                pick = i;
            }
            for (int k = 0; k < 3; k++) com_v[k] = com_v[k] + vel[3 * (size_t)i + k];
        }
        for (int k = 0; k < 3; k++) com_v[k] = com_v[k] / n;
        double kin = 0;
        for (int i = start; i < start + n; i++) {
            double d0 = vel[3 * (size_t)i] - com_v[0];
            double d1 = vel[3 * (size_t)i + 1] - com_v[1];
            double d2 = vel[3 * (size_t)i + 2] - com_v[2];
            kin = kin + ((d0 * d0 + d1 * d1) + d2 * d2);
        }
        kin = kin / 2;
        if ((local_rate > 0) && (kin > delta_u)) {
            local_rate = local_rate * rate;
            double u[2];
            orc_rng_u2(seed, step, (uint32_t)s, ORC_RNG_BULK, 0, u);
            if (u[0] < (1 - exp(-local_rate * tau))) {
                species[pick] = to;
                double factor = sqrt((kin - delta_u) / kin);
                for (int i = start; i < start + n; i++)
                    for (int k = 0; k < 3; k++)
                        vel[3 * (size_t)i + k] = com_v[k] + factor * (vel[3 * (size_t)i + k] - com_v[k]);
            }
        }
    }
}
