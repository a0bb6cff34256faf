// Program-local solvent loops of programs/single_dimer_pbc.f90 on the GPU:
// reaction flagging, A -> B conversion, B -> A refuelling and the
// per-interval observables.
#include <cmath>
#include <cstring>
#include <vector>

#include "rmpcd_common.cuh"
#include "rng.cuh"
#include "state.cuh"
#include "stepops.cuh"
#include "timers.cuh"

namespace rmpcd {

// flag_particles_nl, programs/single_dimer_pbc.f90:493-509
template <typename R>
__global__ void k_flag_nl(const int *list, const int *n, int point, int Nmax, const double *cx,
                          const double *cy, const double *cz, const R *sx, const R *sy, const R *sz,
                          const int *species, int *flags, double L0, double L1, double L2, double cut_sq)
{
    int n1 = n[point];
    double x[3] = {cx[point], cy[point], cz[point]};
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n1; s += gridDim.x * blockDim.x)
        flag_nl_one(list[(size_t)point * Nmax + s], x, sx, sy, sz, species, flags, L0, L1, L2, cut_sq);
}

// change_species, programs/single_dimer_pbc.f90:511-542
template <typename R>
__global__ void k_change_species(PView<R> v, const double *cx, const double *cy, const double *cz,
                                 double L0, double L1, double L2, double cut_c, double cut_n, double prob,
                                 uint64_t seed, uint64_t step)
{
    double a[3] = {cx[0], cy[0], cz[0]}, b[3] = {cx[1], cy[1], cz[1]};
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < v.N;
         m += (long long)gridDim.x * blockDim.x)
        change_species_one(v, m, m, a, b, L0, L1, L2, cut_c, cut_n, prob, seed, step);
}

// refuel, programs/single_dimer_pbc.f90:544-565
template <typename R>
__global__ void k_refuel(PView<R> v, const double *cx, const double *cy, const double *cz, double L0,
                         double L1, double L2, double far)
{
    double a[3] = {cx[0], cy[0], cz[0]}, b[3] = {cx[1], cy[1], cz[1]};
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < v.N;
         m += (long long)gridDim.x * blockDim.x)
        refuel_one(v, m, a, b, L0, L1, L2, far);
}

__global__ void k_n_solvent(const int *species, int N, int n_species, int *counts)
{
    __shared__ int c[RMPCD_MAX_SPECIES];
    if (threadIdx.x < RMPCD_MAX_SPECIES) c[threadIdx.x] = 0;
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        int j = species[i];
        if (j >= 1 && j <= n_species) atomicAdd(c + (j - 1), 1);
    }
    __syncthreads();
    if (threadIdx.x < n_species) atomicAdd(counts + threadIdx.x, c[threadIdx.x]);
}

// compute_cylindrical_shell_histogram, src/particle_system.f90:412-445
template <typename R>
__global__ void k_cyl_hist(PView<R> v, double x1_0, double x1_1, double x1_2, double u0, double u1, double u2,
                           double L0, double L1, double L2, int bin_species, double rmin_sq, double rmax_sq,
                           double xmin, double dx, int nbins, unsigned long long *hist)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x) {
        if (v.species[i] != bin_species) continue;
        double d0 = min_image_d((double)v.pos.x[i] - x1_0, L0);
        double d1 = min_image_d((double)v.pos.y[i] - x1_1, L1);
        double d2 = min_image_d((double)v.pos.z[i] - x1_2, L2);
        double el = u0 * d0 + u1 * d1 + u2 * d2;
        d0 = d0 - el * u0;
        d1 = d1 - el * u1;
        d2 = d2 - el * u2;
        double nn = d0 * d0 + d1 * d1 + d2 * d2;
        if ((nn > rmin_sq) && (nn < rmax_sq)) {
            int idx = ifloor((el - xmin) / dx) + 1;
            if ((idx > 0) && (idx <= nbins)) atomicAdd(hist + (idx - 1), 1ull);
        }
    }
}

// sum(vel**2) and sum(vel, dim=2): per-block partials in a fixed partition,
// then a fixed-order final sum
template <typename R>
__global__ void k_vel_sums(PView<R> v, double *part)
{
    double s2 = 0, sx = 0, sy = 0, sz = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x) {
        double a = (double)v.vel.x[i], b = (double)v.vel.y[i], c = (double)v.vel.z[i];
        s2 = s2 + a * a + b * b + c * c;
        sx += a;
        sy += b;
        sz += c;
    }
    __shared__ double sh[4][256];
    sh[0][threadIdx.x] = s2;
    sh[1][threadIdx.x] = sx;
    sh[2][threadIdx.x] = sy;
    sh[3][threadIdx.x] = sz;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; k++) part[4 * blockIdx.x + k] = sh[k][0];
}

__global__ void k_vel_sums_final(const double *part, int nb, double *out)
{
    if (threadIdx.x != 0) return;
    double a[4] = {0, 0, 0, 0};
    for (int b = 0; b < nb; b++)
        for (int k = 0; k < 4; k++) a[k] = a[k] + part[4 * b + k];
    for (int k = 0; k < 4; k++) out[k] = a[k];
}

}  // namespace rmpcd

using namespace rmpcd;

#define DISPATCH_R(p, CALL_F, CALL_D)        \
    do {                                      \
        if ((p)->precision == RMPCD_FP32) {   \
            CALL_F;                           \
        } else {                              \
            CALL_D;                           \
        }                                     \
    } while (0)

static bool colloid_ok(const rmpcd_particles *c, int need)
{
    return c && c->precision == RMPCD_FP64 && c->N >= need;
}

extern "C" {

int rmpcd_flag_particles_nl(rmpcd_nlist *nl, int point, rmpcd_particles *col, rmpcd_particles *sol,
                            const double edges[3], double cut_sq)
{
    RMPCD_ARG(nl && col && sol && edges, "null argument");
    RMPCD_ARG(colloid_ok(col, point + 1) && point >= 0 && point < nl->Npoints, "flag_particles_nl: bad point");
    PhaseTimer t("flag");
    PView<double> c = cur<double>(col);
    int g = grid_for(nl->Nmax, 256);
    DISPATCH_R(sol,
               ({ PView<float> v = cur<float>(sol);
                  k_flag_nl<float><<<g, 256, 0, stream()>>>(nl->list, nl->n, point, nl->Nmax, c.pos.x, c.pos.y, c.pos.z,
                                                            v.pos.x, v.pos.y, v.pos.z, v.species, v.flags, edges[0], edges[1], edges[2], cut_sq); }),
               ({ PView<double> v = cur<double>(sol);
                  k_flag_nl<double><<<g, 256, 0, stream()>>>(nl->list, nl->n, point, nl->Nmax, c.pos.x, c.pos.y, c.pos.z,
                                                             v.pos.x, v.pos.y, v.pos.z, v.species, v.flags, edges[0], edges[1], edges[2], cut_sq); }));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_change_species(rmpcd_particles *sol, rmpcd_particles *col, const double edges[3], double cut_sq_C,
                         double cut_sq_N, double prob, rmpcd_rng *r)
{
    RMPCD_ARG(sol && col && edges && r, "null argument");
    RMPCD_ARG(colloid_ok(col, 2), "change_species: needs a 2-colloid FP64 system");
    PhaseTimer t("change");
    PView<double> c = cur<double>(col);
    if (sol->N > 0) {
        int g = grid_for(sol->N, 256);
        DISPATCH_R(sol,
                   (k_change_species<float><<<g, 256, 0, stream()>>>(cur<float>(sol), c.pos.x, c.pos.y, c.pos.z, edges[0],
                                                                     edges[1], edges[2], cut_sq_C, cut_sq_N, prob, r->seed, r->step)),
                   (k_change_species<double><<<g, 256, 0, stream()>>>(cur<double>(sol), c.pos.x, c.pos.y, c.pos.z, edges[0],
                                                                      edges[1], edges[2], cut_sq_C, cut_sq_N, prob, r->seed, r->step)));
        RMPCD_CHECK_LAUNCH();
    }
    r->step++;
    return RMPCD_OK;
}

int rmpcd_refuel(rmpcd_particles *sol, rmpcd_particles *col, const double edges[3], int L1)
{
    RMPCD_ARG(sol && col && edges, "null argument");
    RMPCD_ARG(colloid_ok(col, 2), "refuel: needs a 2-colloid FP64 system");
    PhaseTimer t("refuel");
    // far = (L(1)*0.45)**2 is a default-real expression in the reference
    volatile float lf = (float)L1 * 0.45f;
    volatile float ff = lf * lf;
    double far = (double)ff;
    PView<double> c = cur<double>(col);
    if (sol->N > 0) {
        int g = grid_for(sol->N, 256);
        DISPATCH_R(sol,
                   (k_refuel<float><<<g, 256, 0, stream()>>>(cur<float>(sol), c.pos.x, c.pos.y, c.pos.z, edges[0], edges[1], edges[2], far)),
                   (k_refuel<double><<<g, 256, 0, stream()>>>(cur<double>(sol), c.pos.x, c.pos.y, c.pos.z, edges[0], edges[1], edges[2], far)));
        RMPCD_CHECK_LAUNCH();
    }
    return RMPCD_OK;
}

int rmpcd_n_solvent(rmpcd_particles *sol, int n_species, int *counts)
{
    RMPCD_ARG(sol && counts, "null argument");
    RMPCD_ARG(n_species >= 1 && n_species <= RMPCD_MAX_SPECIES, "n_species must be in 1..4");
    int *d = sol->d_ints + 8;
    RMPCD_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(int) * RMPCD_MAX_SPECIES, stream()));
    if (sol->N > 0)
        k_n_solvent<<<grid_for(sol->N, 256), 256, 0, stream()>>>(sol->species[sol->cur], sol->N, n_species, d);
    RMPCD_CHECK_LAUNCH();
    RMPCD_CUDA_TRY(cudaMemcpyAsync(counts, d, sizeof(int) * n_species, cudaMemcpyDeviceToHost, stream()));
    return sync();
}

int rmpcd_cylindrical_shell_histogram(rmpcd_particles *sol, const double x1[3], const double x2[3],
                                      const double L[3], int bin_species, double r_min, double r_max,
                                      double xmin, double dx, int nbins, double *hist)
{
    RMPCD_ARG(sol && x1 && x2 && L && hist, "null argument");
    RMPCD_ARG(nbins >= 1 && nbins <= 4096, "nbins must be in 1..4096");
    double uz[3];
    for (int k = 0; k < 3; k++) uz[k] = min_image_d(x2[k] - x1[k], L[k]);
    double norm = sqrt(uz[0] * uz[0] + uz[1] * uz[1] + uz[2] * uz[2]);
    for (int k = 0; k < 3; k++) uz[k] = uz[k] / norm;
    unsigned long long *d = nullptr;
    RMPCD_CUDA_TRY(cudaMalloc(&d, sizeof(unsigned long long) * (size_t)nbins));
    RMPCD_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long) * (size_t)nbins, stream()));
    if (sol->N > 0) {
        int g = grid_for(sol->N, 256);
        DISPATCH_R(sol,
                   (k_cyl_hist<float><<<g, 256, 0, stream()>>>(cur<float>(sol), x1[0], x1[1], x1[2], uz[0], uz[1], uz[2], L[0], L[1], L[2],
                                                               bin_species, r_min * r_min, r_max * r_max, xmin, dx, nbins, d)),
                   (k_cyl_hist<double><<<g, 256, 0, stream()>>>(cur<double>(sol), x1[0], x1[1], x1[2], uz[0], uz[1], uz[2], L[0], L[1], L[2],
                                                                bin_species, r_min * r_min, r_max * r_max, xmin, dx, nbins, d)));
    }
    std::vector<unsigned long long> h((size_t)nbins);
    cudaError_t e = cudaMemcpyAsync(h.data(), d, sizeof(unsigned long long) * (size_t)nbins, cudaMemcpyDeviceToHost, stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream());
    cudaFree(d);
    if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "cylindrical histogram: %s", cudaGetErrorString(e));
    for (int b = 0; b < nbins; b++) hist[b] = hist[b] + (double)h[b];
    return RMPCD_OK;
}

int rmpcd_velocity_sums(rmpcd_particles *p, double out[4])
{
    RMPCD_ARG(p && out, "null argument");
    const int nb = 256;
    double *part = p->d_sums;
    if (p->N > 0) {
        DISPATCH_R(p, (k_vel_sums<float><<<nb, 256, 0, stream()>>>(cur<float>(p), part)),
                   (k_vel_sums<double><<<nb, 256, 0, stream()>>>(cur<double>(p), part)));
        k_vel_sums_final<<<1, 32, 0, stream()>>>(part, nb, part + 4 * nb);
        RMPCD_CHECK_LAUNCH();
        RMPCD_CUDA_TRY(cudaMemcpyAsync(out, part + 4 * nb, 4 * sizeof(double), cudaMemcpyDeviceToHost, stream()));
        return sync();
    }
    for (int k = 0; k < 4; k++) out[k] = 0;
    return RMPCD_OK;
}

}  // extern "C"
