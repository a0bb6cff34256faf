/*
 * A plain-C user of include/rmpcd.h: builds a bulk SRD fluid of 12 x 10 x 8
 * cells at density 10, sorts it, runs three MPCD intervals and a collision
 * through the C entry points (the calls a C or Fortran program makes), and
 * checks what must hold: the particle ids are still a permutation of 1..N,
 * the cell counts add up to N, every position is inside the box, and the
 * total momentum is unchanged (SRD conserves it cell by cell; streaming does
 * not change velocities).  Exit status 0 on success, 1 with a message on
 * failure.  Build: see tests/test_c_program.py.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rmpcd.h"

#define CHECK(call)                                                                  \
    do {                                                                             \
        int rc_ = (call);                                                            \
        if (rc_ != RMPCD_OK) {                                                       \
            fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, rmpcd_last_error_string()); \
            return 1;                                                                \
        }                                                                            \
    } while (0)

/* deterministic uniform numbers in [0, 1) (64-bit LCG, top 53 bits) */
static double uniform(uint64_t *s)
{
    *s = *s * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(*s >> 11) * (1.0 / 9007199254740992.0);
}

int main(int argc, char **argv)
{
    const int precision = (argc > 1 && strcmp(argv[1], "32") == 0) ? RMPCD_FP32 : RMPCD_FP64;
    const int L[3] = {12, 10, 8};
    const int N = 10 * L[0] * L[1] * L[2];
    rmpcd_cells *cells = NULL;
    rmpcd_particles *p = NULL;
    CHECK(rmpcd_cells_init(&cells, L, 1.0, 0));
    int Lo[3], M[3], S;
    double edges[3];
    CHECK(rmpcd_cells_info(cells, Lo, M, &S, edges));
    CHECK(rmpcd_particles_init(&p, N, 1, NULL, precision));

    double *pos = malloc(sizeof(double) * 3 * N), *vel = malloc(sizeof(double) * 3 * N);
    int *species = malloc(sizeof(int) * N), *id = malloc(sizeof(int) * N), *count = malloc(sizeof(int) * S);
    char *seen = calloc(N + 1, 1);
    uint64_t s = 12345;
    double mom0[3] = {0, 0, 0};
    for (int i = 0; i < N; i++) {
        for (int k = 0; k < 3; k++) {
            pos[3 * i + k] = uniform(&s) * edges[k];
            vel[3 * i + k] = uniform(&s) - 0.5;
            mom0[k] += vel[3 * i + k];
        }
        species[i] = 1;
    }
    CHECK(rmpcd_particles_upload(p, "pos", pos));
    CHECK(rmpcd_particles_upload(p, "vel", vel));
    CHECK(rmpcd_particles_upload(p, "species", species));
    const double origin[3] = {-0.25, -0.5, -0.75};
    CHECK(rmpcd_cells_set_origin(cells, origin));
    CHECK(rmpcd_particles_sort(p, cells));
    rmpcd_rng rng = {2024, 0};
    CHECK(rmpcd_bulk_run(p, cells, &rng, 1.0, 0, 0.0, 3));
    CHECK(rmpcd_simple_mpcd_step(p, cells, &rng, 0, 0.0, 0, 0.0, 1));
    CHECK(rmpcd_particles_download(p, "pos", pos));
    CHECK(rmpcd_particles_download(p, "vel", vel));
    CHECK(rmpcd_particles_download(p, "id", id));
    CHECK(rmpcd_cells_download_count(cells, count));

    int bad = 0;
    long long total = 0;
    for (int c = 0; c < S; c++) total += count[c];
    if (total != N) {
        fprintf(stderr, "cell counts add up to %lld, not %d\n", total, N);
        bad = 1;
    }
    double mom[3] = {0, 0, 0};
    for (int i = 0; i < N; i++) {
        if (id[i] < 1 || id[i] > N || seen[id[i]]) {
            fprintf(stderr, "id %d at %d is not part of a permutation\n", id[i], i);
            bad = 1;
            break;
        }
        seen[id[i]] = 1;
        for (int k = 0; k < 3; k++) {
            if (!(pos[3 * i + k] >= 0 && pos[3 * i + k] < edges[k])) {
                fprintf(stderr, "position %d,%d = %g outside the box\n", i, k, pos[3 * i + k]);
                bad = 1;
            }
            mom[k] += vel[3 * i + k];
        }
    }
    const double tol = precision == RMPCD_FP32 ? 1e-2 : 1e-9;
    for (int k = 0; k < 3; k++)
        if (fabs(mom[k] - mom0[k]) > tol) {
            fprintf(stderr, "momentum %d changed: %.17g -> %.17g\n", k, mom0[k], mom[k]);
            bad = 1;
        }
    if (rng.step != 7) {
        fprintf(stderr, "rng step %llu, expected 7\n", (unsigned long long)rng.step);
        bad = 1;
    }
    /* sort_particles (src/cell_system.f90:131-151): the current positions of p,
     * counted, scattered in cell order into a second system q; the compact
     * Hilbert index of each scattered position must not decrease */
    rmpcd_particles *q = NULL;
    CHECK(rmpcd_particles_init(&q, N, 1, NULL, precision));
    CHECK(rmpcd_cells_count_particles(cells, p));
    CHECK(rmpcd_cells_sort_particles(cells, p, q));
    double *qpos = malloc(sizeof(double) * 3 * N), o[3];
    CHECK(rmpcd_particles_download(q, "pos", qpos));
    CHECK(rmpcd_cells_get_origin(cells, o));
    int prev = -1;
    for (int i = 0; i < N && !bad; i++) {
        int pc[3], h = 0;
        for (int k = 0; k < 3; k++) {
            pc[k] = (int)floor(qpos[3 * i + k] - o[k]);
            if (pc[k] == Lo[k]) pc[k] = 0;
        }
        CHECK(rmpcd_compact_p_to_h(pc, M, &h));
        if (h < prev) {
            fprintf(stderr, "sort_particles: position %d in slot %d after slot %d\n", i, h, prev);
            bad = 1;
        }
        prev = h;
    }
    /* random_placement keyed by the state's seed; the step stays */
    CHECK(rmpcd_particles_random_placement(q, edges, NULL, NULL, &rng));
    CHECK(rmpcd_particles_download(q, "pos", qpos));
    for (int i = 0; i < 3 * N && !bad; i++)
        if (!(qpos[i] >= 0 && qpos[i] < edges[i % 3])) {
            fprintf(stderr, "random_placement: coordinate %d = %g outside the box\n", i, qpos[i]);
            bad = 1;
        }
    if (rng.step != 7) {
        fprintf(stderr, "random_placement moved the rng step to %llu\n", (unsigned long long)rng.step);
        bad = 1;
    }
    free(qpos);
    CHECK(rmpcd_particles_destroy(q));
    CHECK(rmpcd_particles_destroy(p));
    CHECK(rmpcd_cells_destroy(cells));
    free(pos);
    free(vel);
    free(species);
    free(id);
    free(count);
    free(seen);
    if (!bad) printf("bulk_fluid (FP%d): %d particles, 4 intervals, ok\n", precision, N);
    return bad;
}
