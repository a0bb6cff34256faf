/*
 * Lennard-Jones parameters and forces (src/interaction.f90) and the
 * colloid -> solvent neighbor list (src/neighbor_list.f90).  Test
 * infrastructure only (oracle).
 *
 * Integer powers follow gfortran's constant-exponent expansion (the addition
 * chain of gfc_conv_powi): x**6 = x**3 * x**3 with x**3 = x * (x*x), and
 * x**3 for r_sq.  Multiplication is commutative in IEEE arithmetic, so the
 * operand order inside each product does not matter.
 */
#include <math.h>
#include <string.h>
#include "rmpcd_oracle.h"

static double cube(double x) { return x * (x * x); }
double orc_sixth(double x)
{
    double x3 = cube(x);
    return x3 * x3;
}

/* lj_energy, src/interaction.f90:126-136 */
double orc_lj_energy(double r_sq, double epsilon, double sigma, double cut_energy)
{
    double s6 = orc_sixth(sigma) / cube(r_sq);
    return 4.0 * epsilon * (s6 * s6 - s6) - cut_energy;
}

/* lj_force, src/interaction.f90:83-96 */
void orc_lj_force(const double d[3], double r_sq, double epsilon, double sigma, double f[3])
{
    double s6 = orc_sixth(sigma) / cube(r_sq);
    double for_ = 24.0 * epsilon * s6 / r_sq * (2.0 * s6 - 1.0);
    for (int k = 0; k < 3; k++) f[k] = for_ * d[k];
}

/* lj_params_init, src/interaction.f90:38-80 */
void orc_lj_init(orc_lj *lj, int n1, int n2, const double *epsilon,
                 const double *sigma, const double *cut)
{
    memset(lj, 0, sizeof(*lj));
    lj->n1 = n1;
    lj->n2 = n2;
    for (int i = 0; i < n1 * n2; i++) {
        lj->epsilon[i] = epsilon[i];
        lj->sigma[i] = sigma[i];
        lj->sigma_sq[i] = sigma[i] * sigma[i];
        lj->cut[i] = cut[i];
        lj->cut_sq[i] = cut[i] * cut[i];
        lj->cut_energy[i] = orc_lj_energy(lj->cut_sq[i], lj->epsilon[i], lj->sigma[i], lj->sigma[i] * 0);
    }
}

/* closest, src/neighbor_list.f90:310-322 */
static double closest(const int x1[3])
{
    int dist_sq = 0;
    for (int i = 0; i < 3; i++) {
        int v = abs(x1[i]) - 1;
        if (v < 0) v = 0;
        dist_sq += v * v;
    }
    return sqrt((double)dist_sq);
}

/* make_stencil, src/neighbor_list.f90:271-308 */
int orc_make_stencil(double a, double cut, int *stencil, int cap)
{
    int max_i = (int)floor(cut / a) + 1;
    int count = 0;
    for (int i = -max_i; i <= max_i; i++)
        for (int j = -max_i; j <= max_i; j++)
            for (int k = -max_i; k <= max_i; k++) {
                int o[3] = {i, j, k};
                if (closest(o) < cut) {
                    if (count < cap) {
                        stencil[3 * count] = i;
                        stencil[3 * count + 1] = j;
                        stencil[3 * count + 2] = k;
                    }
                    count++;
                }
            }
    return count;
}

static int imodulo(int a, int p)
{
    int r = a % p;
    if (r != 0 && ((r < 0) != (p < 0))) r += p;
    return r;
}

#define LJT(lj, s1, s2) ((s1) - 1 + (lj)->n1 * ((s2) - 1))

/* update_list, src/neighbor_list.f90:76-157 */
int orc_update_list(const orc_grid *g, int C, const double *cpos, const int *cspecies,
                    int N, const double *spos, const int *sspecies,
                    const int *cell_count, const int *cell_start,
                    const int *stencil, int n_stencil, double radius,
                    const orc_lj *lj, int Nmax, int *list, int *n,
                    unsigned char *is_md, unsigned char *is_reac)
{
    (void)N;
    double L[3];
    for (int k = 0; k < 3; k++) L[k] = g->L[k] * g->a;
    double radiussq = radius * radius;
    for (int s = 0; s < g->S; s++) {
        is_md[s] = 0;
        is_reac[s] = 1;
    }
    int status = 0;
    for (int i = 0; i < C; i++) {
        const double *x = cpos + 3 * (size_t)i;
        int si = cspecies[i];
        int cell[3];
        orc_cartesian_indices(g, x, cell);
        int list_idx = 0;
        for (int j = 0; j < n_stencil; j++) {
            int actual[3];
            for (int k = 0; k < 3; k++) actual[k] = imodulo(cell[k] + stencil[3 * j + k], g->L[k]);
            int md = 0, noreac = 0;
            int slot = orc_compact_p_to_h(actual, g->M);
            int cn = cell_count[slot];
            int cs = cell_start[slot];
            for (int ci = cs - 1; ci < cs - 1 + cn; ci++) {
                int s = sspecies[ci];
                if (s <= 0) continue;
                double r[3];
                orc_rel_pos(x, spos + 3 * (size_t)ci, L, r);
                double rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                if (rsq < radiussq) {
                    list_idx++;
                    md = 1;
                    if (lj && rsq <= lj->cut_sq[LJT(lj, s, si)]) noreac = 1;
                    if (list_idx > Nmax) {
                        status = -1;
                        list_idx = Nmax;
                        continue;
                    }
                    list[(size_t)i * (size_t)Nmax + (list_idx - 1)] = ci + 1;
                }
            }
            if (md) {
                is_md[slot] = 1;
                if (noreac) is_reac[slot] = 0;
            }
        }
        n[i] = list_idx;
    }
    return status;
}

/* compute_force, src/neighbor_list.f90:159-225 */
double orc_compute_force(int C, const double *cpos, const int *cspecies, double *cforce,
                         int N, const double *spos, const int *sspecies,
                         double *sforce, int *sflags, const int *list, const int *n,
                         int Nmax, const double L[3], const orc_lj *lj)
{
    double e = 0;
    for (int i = 0; i < N; i++) {
        if ((sflags[i] >> ORC_MD_BIT) & 1) sflags[i] |= (1 << ORC_PAST_MD_BIT);
        else sflags[i] &= ~(1 << ORC_PAST_MD_BIT);
        sflags[i] &= ~(1 << ORC_MD_BIT);
    }
    for (int i = 0; i < C; i++) {
        /* if (species(i) <= 0) continue  -- a no-op in the reference */
        const double *x = cpos + 3 * (size_t)i;
        int s1 = cspecies[i];
        double f1[3] = {0, 0, 0};
        for (int j = 0; j < n[i]; j++) {
            int idx = list[(size_t)i * (size_t)Nmax + j] - 1;
            int s2 = sspecies[idx];
            if (s2 <= 0) continue;
            double d[3];
            orc_rel_pos(x, spos + 3 * (size_t)idx, L, d);
            double r_sq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            int t = LJT(lj, s2, s1);
            if (r_sq <= lj->cut_sq[t]) {
                double f[3];
                orc_lj_force(d, r_sq, lj->epsilon[t], lj->sigma[t], f);
                e = e + orc_lj_energy(r_sq, lj->epsilon[t], lj->sigma[t], lj->cut_energy[t]);
                for (int k = 0; k < 3; k++) {
                    f1[k] = f1[k] + f[k];
                    sforce[3 * (size_t)idx + k] = sforce[3 * (size_t)idx + k] - f[k];
                }
                int mask = 1 << ORC_MD_BIT;
                if (s1 == 1) mask |= (1 << ORC_CATALYZED_BIT);
                sflags[idx] |= mask;
            }
        }
        for (int k = 0; k < 3; k++) cforce[3 * (size_t)i + k] = cforce[3 * (size_t)i + k] + f1[k];
    }
    return e;
}

/* compute_force_n2, src/neighbor_list.f90:227-264 */
double orc_compute_force_n2(int C, const double *pos, const int *species, double *force,
                            const double L[3], const orc_lj *lj)
{
    double e = 0;
    for (int i = 0; i < C; i++) {
        int s1 = species[i];
        const double *x = pos + 3 * (size_t)i;
        for (int j = i + 1; j < C; j++) {
            int s2 = species[j];
            double d[3];
            orc_rel_pos(x, pos + 3 * (size_t)j, L, d);
            double r_sq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r_sq <= lj->cut_sq[LJT(lj, s1, s2)]) {
                int t = LJT(lj, s2, s1);
                double f[3];
                orc_lj_force(d, r_sq, lj->epsilon[t], lj->sigma[t], f);
                for (int k = 0; k < 3; k++) {
                    force[3 * (size_t)i + k] = force[3 * (size_t)i + k] + f[k];
                    force[3 * (size_t)j + k] = force[3 * (size_t)j + k] - f[k];
                }
                e = e + orc_lj_energy(r_sq, lj->epsilon[t], lj->sigma[t], lj->cut_energy[t]);
            }
        }
    }
    return e;
}
