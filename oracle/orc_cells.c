/*
 * Cell system and particle sort, restated from src/cell_system.f90 and
 * src/particle_system.f90.  Test infrastructure only (oracle).
 *
 * With one thread the scatter follows the reference's single-thread order
 * (stable in the old particle index).  With more threads it uses the same
 * OpenMP atomic-capture scatter as the reference, whose in-cell order is then
 * schedule dependent; that mode exists only for timing the CPU baseline.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "rmpcd_oracle.h"

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* cell_system_t%init, src/cell_system.f90:49-84 */
void orc_grid_init(orc_grid *g, const int L[3], double a, int has_walls)
{
    memset(g, 0, sizeof(*g));
    for (int i = 0; i < 3; i++) {
        g->L[i] = L[i];
        g->edges[i] = L[i] * a;
    }
    g->has_walls = has_walls ? 1 : 0;
    if (g->has_walls) g->L[2] = L[2] + 1;
    g->a = a;
    for (int i = 0; i < 3; i++) {
        g->M[i] = 1;
        g->origin[i] = 0.0;
        g->bc[i] = ORC_PERIODIC_BC;
        while ((1 << g->M[i]) < g->L[i]) g->M[i]++;
    }
    g->S = (1 << g->M[0]) * (1 << g->M[1]) * (1 << g->M[2]);
    g->max_v = 0.0;
}

/* cartesian_indices, src/cell_system.f90:165-175 */
void orc_cartesian_indices(const orc_grid *g, const double x[3], int p[3])
{
    for (int k = 0; k < 3; k++) p[k] = (int)floor((x[k] / g->a) - g->origin[k]);
    if (p[0] == g->L[0]) p[0] = 0;
    if (p[1] == g->L[1]) p[1] = 0;
    if ((!g->has_walls) && (p[2] == g->L[2])) p[2] = 0;
}

static int slot_of(const orc_grid *g, const double *x)
{
    int p[3];
    orc_cartesian_indices(g, x, p);
    return orc_compact_p_to_h(p, g->M);
}

/* count_particles, src/cell_system.f90:86-129 (per-thread histograms, merge,
 * serial prefix with cell_start(1) = 1) */
void orc_count_particles(const orc_grid *g, int N, const double *pos,
                         int *cell_count, int *cell_start)
{
    int S = g->S;
    int nt = orc_num_threads();
    if (nt <= 1) {
        memset(cell_count, 0, sizeof(int) * (size_t)S);
        for (int i = 0; i < N; i++) cell_count[slot_of(g, pos + 3 * (size_t)i)]++;
    } else {
        int *tmp = (int *)calloc((size_t)S * (size_t)nt, sizeof(int));
#pragma omp parallel
        {
#ifdef _OPENMP
            int tid = omp_get_thread_num();
#else
            int tid = 0;
#endif
            int *mine = tmp + (size_t)tid * (size_t)S;
#pragma omp for
            for (int i = 0; i < N; i++) mine[slot_of(g, pos + 3 * (size_t)i)]++;
        }
#pragma omp parallel for
        for (int s = 0; s < S; s++) {
            int c = 0;
            for (int t = 0; t < nt; t++) c += tmp[(size_t)t * (size_t)S + s];
            cell_count[s] = c;
        }
        free(tmp);
    }
    cell_start[0] = 1;
    for (int s = 1; s < S; s++) cell_start[s] = cell_start[s - 1] + cell_count[s - 1];
}

/* particle_system_t%sort, src/particle_system.f90:304-355 */
void orc_sort(const orc_grid *g, int N, int *cell_count, int *cell_start,
              double *pos, double *pos_old, int *image, double *vel,
              double *force, double *force_old, int *id, int *species,
              int *flags, int *id_to_idx)
{
    size_t n3 = 3 * (size_t)N;
    orc_count_particles(g, N, pos, cell_count, cell_start);

    int *dest = (int *)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
    if (orc_num_threads() <= 1) {
        for (int i = 0; i < N; i++) {
            /* if (species(i) == 0) continue  -- a no-op in the reference */
            int s = slot_of(g, pos + 3 * (size_t)i);
            dest[i] = cell_start[s] - 1;
            cell_start[s]++;
        }
    } else {
#pragma omp parallel for
        for (int i = 0; i < N; i++) {
            int s = slot_of(g, pos + 3 * (size_t)i);
            int start;
#pragma omp atomic capture
            { start = cell_start[s]; cell_start[s]++; }
            dest[i] = start - 1;
        }
    }
    for (int s = 0; s < g->S; s++) cell_start[s] -= cell_count[s];

    double *dtmp = (double *)malloc(sizeof(double) * (n3 > 0 ? n3 : 1));
    int *itmp = (int *)malloc(sizeof(int) * (n3 > 0 ? n3 : 1));
#define PERMUTE3(T, arr, tmp) do { if (arr) { \
        for (int i = 0; i < N; i++) for (int k = 0; k < 3; k++) \
            tmp[3 * (size_t)dest[i] + k] = arr[3 * (size_t)i + k]; \
        memcpy(arr, tmp, sizeof(T) * n3); } } while (0)
#define PERMUTE1(T, arr, tmp) do { if (arr) { \
        for (int i = 0; i < N; i++) tmp[dest[i]] = arr[i]; \
        memcpy(arr, tmp, sizeof(T) * (size_t)N); } } while (0)

    if (pos_old) memcpy(pos_old, pos, sizeof(double) * n3);
    if (id_to_idx && id)
        for (int i = 0; i < N; i++) id_to_idx[id[i] - 1] = dest[i] + 1;
    PERMUTE3(double, pos, dtmp);
    PERMUTE3(int, image, itmp);
    PERMUTE3(double, vel, dtmp);
    PERMUTE3(double, force, dtmp);
    PERMUTE3(double, force_old, dtmp);
    PERMUTE1(int, id, itmp);
    PERMUTE1(int, species, itmp);
    PERMUTE1(int, flags, itmp);
#undef PERMUTE3
#undef PERMUTE1
    free(dtmp);
    free(itmp);
    free(dest);
}

/* sort_particles, src/cell_system.f90:131-151 */
void orc_sort_particles(const orc_grid *g, int N, int *cell_start,
                        const double *pos_in, double *pos_out)
{
    for (int i = 0; i < N; i++) {
        int s = slot_of(g, pos_in + 3 * (size_t)i);
        int start = cell_start[s];
        cell_start[s]++;
        for (int k = 0; k < 3; k++) pos_out[3 * (size_t)(start - 1) + k] = pos_in[3 * (size_t)i + k];
    }
}
