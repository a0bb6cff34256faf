// The main loops of programs/n_colloids_pbc.f90 (:221-276 thermalisation,
// :304-324 production) as one native call: passive LJ colloids in an SRD
// fluid with lazy, cell-wise solvent streaming.  The loop issues the same
// module entry points, in the same order, as a program calling them one by
// one (and as rmpcdmd_b200.programs.NColloidsPBC.interval does), so the
// results are identical; it removes the per-call host overhead and reads the
// two displacement maxima of each MD step with a single synchronisation.
#include <cmath>
#include <cstring>
#include <vector>

#include "rmpcd_common.cuh"
#include "sortcore.cuh"
#include "state.cuh"
#include "timers.cuh"

namespace rmpcd {

struct NcLoop {
    rmpcd_particles *s, *c;
    rmpcd_cells *cells;
    rmpcd_nlist *nl;
    const rmpcd_lj *lj_sc, *lj_cc;
    rmpcd_rng *rng;
    const rmpcd_ncolloids_params *prm;
    rmpcd_ncolloids_state *st;
    std::vector<double> vv_mass;
    double dt;
};

// the displacement maxima of the MD step: solvent over is_md cells (floored
// at max_v * delta_t) and colloids, read with one synchronisation
static int displacements(NcLoop &L, double delta_t, double *so_max, double *co_max)
{
    int rc = launch_cell_max_disp(L.cells, L.s);
    if (!rc) rc = launch_max_disp(L.c);
    if (rc) return rc;
    unsigned long long bits[2] = {0, 0};
    RMPCD_CUDA_TRY(cudaMemcpyAsync(bits, L.s->d_max, 8, cudaMemcpyDeviceToHost, stream()));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(bits + 1, L.c->d_max, 8, cudaMemcpyDeviceToHost, stream()));
    rc = sync();
    if (rc) return rc;
    double m0, m1;
    memcpy(&m0, bits, 8);
    memcpy(&m1, bits + 1, 8);
    const double a = sqrt(m0), b = L.cells->max_v * delta_t;
    *so_max = a > b ? a : b;
    *co_max = sqrt(m1);
    return RMPCD_OK;
}

// stream the non-MD cells over the time since the last sort, wrap, sort,
// rebuild the list (programs/n_colloids_pbc.f90:230-241)
static int catch_up_and_sort(NcLoop &L)
{
    const double dtl = (L.st->t - L.st->last_sort) * L.dt;
    int rc = rmpcd_cell_md_pos(L.cells, L.s, dtl, 0);
    if (!rc) rc = rmpcd_cell_md_vel(L.cells, L.s, dtl, 0);
    if (!rc) rc = rmpcd_apply_pbc(L.s, L.cells->edges);
    if (!rc) rc = rmpcd_apply_pbc(L.c, L.cells->edges);
    if (!rc) rc = rmpcd_particles_sort(L.s, L.cells);
    L.st->last_sort = L.st->t;
    if (!rc) rc = rmpcd_nlist_update(L.nl, L.c, L.s, L.prm->list_radius, L.cells, nullptr);
    if (!rc) rc = rmpcd_particles_copy_pos_old(L.s);
    if (!rc) rc = rmpcd_particles_copy_pos_old(L.c);
    return rc;
}

// one pass of md_loop (programs/n_colloids_pbc.f90:221-254)
static int md_step(NcLoop &L, bool want_energy)
{
    const double dt = L.dt;
    L.st->t += 1;
    int rc = rmpcd_cell_md_pos(L.cells, L.s, dt, 1);
    if (!rc) rc = rmpcd_colloid_vv_pos(L.c, dt, L.vv_mass.data());
    double so_max = 0, co_max = 0;
    if (!rc) rc = displacements(L, dt * (L.st->t - L.st->last_sort), &so_max, &co_max);
    if (rc) return rc;
    if ((co_max >= L.prm->skin * 0.1) || (so_max >= L.prm->skin * 0.9)) {
        rc = catch_up_and_sort(L);
        if (rc) return rc;
        L.st->n_extra_sorting += 1;
    }
    rc = rmpcd_particles_switch_force(L.s);
    if (!rc) rc = rmpcd_particles_switch_force(L.c);
    if (!rc) rc = rmpcd_particles_zero_force(L.s);
    if (!rc) rc = rmpcd_particles_zero_force(L.c);
    double e1 = 0, e2 = 0;
    if (!rc) rc = rmpcd_compute_force(L.c, L.s, L.nl, L.cells->edges, L.lj_sc, want_energy ? &e1 : nullptr);
    if (!rc) rc = rmpcd_compute_force_n2(L.c, L.cells->edges, L.lj_cc, want_energy ? &e2 : nullptr);
    if (!rc && want_energy) {
        L.st->e1 = e1;
        L.st->e2 = e2;
    }
    if (!rc) rc = rmpcd_cell_md_vel(L.cells, L.s, dt, 1);
    if (!rc) rc = rmpcd_colloid_vv_vel(L.c, dt, L.vv_mass.data());
    return rc;
}

}  // namespace rmpcd

using namespace rmpcd;

extern "C" int rmpcd_ncolloids_run(rmpcd_particles *solvent, rmpcd_particles *colloids, rmpcd_cells *cells,
                                   rmpcd_nlist *nl, const rmpcd_lj *solvent_colloid, const rmpcd_lj *colloid_colloid,
                                   rmpcd_rng *rng, const rmpcd_ncolloids_params *params, int n_intervals,
                                   int thermostat, const double *T, int first_interval, int rescale_every,
                                   double T_rescale, rmpcd_ncolloids_state *state)
{
    RMPCD_ARG(solvent && colloids && cells && nl && solvent_colloid && colloid_colloid && rng && params && state,
              "null argument");
    RMPCD_ARG(n_intervals >= 0 && params->N_MD >= 1 && params->tau > 0, "n_intervals >= 0, N_MD >= 1, tau > 0");
    RMPCD_ARG(!thermostat || T, "a thermostatted run needs the temperatures T");
    RMPCD_ARG(colloids->precision == RMPCD_FP64, "colloids must be FP64");
    NcLoop L;
    L.s = solvent;
    L.c = colloids;
    L.cells = cells;
    L.nl = nl;
    L.lj_sc = solvent_colloid;
    L.lj_cc = colloid_colloid;
    L.rng = rng;
    L.prm = params;
    L.st = state;
    L.vv_mass.assign((size_t)colloids->N, params->mass);
    L.dt = params->tau / params->N_MD;
    PhaseTimer timer("ncolloids_run");
    for (int k = 0; k < n_intervals; k++) {
        const int i = first_interval + k;
        for (int j = 0; j < params->N_MD; j++) {
            int rc = md_step(L, j == params->N_MD - 1);
            if (rc) return rc;
        }
        int rc = rmpcd_cells_random_shift(cells, rng);
        if (!rc) rc = catch_up_and_sort(L);
        if (!rc)
            rc = rmpcd_simple_mpcd_step(solvent, cells, rng, 0, 0.0, thermostat, T ? T[k] : 0.0, params->do_hydro);
        if (!rc && rescale_every > 0 && i % rescale_every == 0) rc = rmpcd_rescale_cells(solvent, cells, T_rescale);
        if (rc) return rc;
    }
    return check_dev_error(nullptr);
}
