// Velocity-Verlet halves, lazy cell-wise streaming with walls, PBC wrap,
// dimer RATTLE and the colloid integrator (src/md.f90,
// programs/single_dimer_pbc.f90).
#include <cmath>
#include <cstring>
#include <vector>

#include "rmpcd_common.cuh"
#include "state.cuh"
#include "stepops.cuh"
#include "timers.cuh"

namespace rmpcd {

// md_pos, src/md.f90:61-77
template <typename R>
__global__ void k_md_pos(PView<R> v, R dt, R dt_sq)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x)
        md_pos_one(v, i, dt, dt_sq);
}

// md_vel, src/md.f90:219-237
template <typename R>
__global__ void k_md_vel(PView<R> v, R dt)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x)
        md_vel_one(v, i, dt);
}

// cell_md_pos, src/md.f90:79-102
template <typename R>
__global__ void k_cell_md_pos(const int *count, const int *start, const unsigned char *is_md, int S,
                              PView<R> v, R dt, R dt_sq, int md_flag)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        if ((is_md[s] != 0) != (md_flag != 0)) continue;
        int a = start[s], n = count[s];
        for (int i = a; i < a + n; i++) {
            v.pos.x[i] = v.pos.x[i] + dt * v.vel.x[i] + dt_sq * v.force.x[i];
            v.pos.y[i] = v.pos.y[i] + dt * v.vel.y[i] + dt_sq * v.force.y[i];
            v.pos.z[i] = v.pos.z[i] + dt * v.vel.z[i] + dt_sq * v.force.z[i];
        }
    }
}

// cell_md_vel, src/md.f90:239-263
template <typename R>
__global__ void k_cell_md_vel(const int *count, const int *start, const unsigned char *is_md, int S,
                              PView<R> v, R dt, int md_flag)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        if ((is_md[s] != 0) != (md_flag != 0)) continue;
        int a = start[s], n = count[s];
        for (int i = a; i < a + n; i++) {
            int f = v.flags[i];
            if (!((f >> WALL_BIT) & 1)) {
                v.vel.x[i] = v.vel.x[i] + dt * (v.force.x[i] + v.force_old.x[i]) / 2;
                v.vel.y[i] = v.vel.y[i] + dt * (v.force.y[i] + v.force_old.y[i]) / 2;
                v.vel.z[i] = v.vel.z[i] + dt * (v.force.z[i] + v.force_old.z[i]) / 2;
            } else {
                v.flags[i] = f & ~(1 << WALL_BIT);
            }
        }
    }
}

// cell_md_pos_ywall / cell_md_pos_zwall, src/md.f90:104-200 (dim 1 or 2)
template <typename R>
__global__ void k_cell_md_pos_wall(const int *count, const int *start, const unsigned char *is_md, int S,
                                   PView<R> v, R dt, R dt_sq, int md_flag, int dim, double Lw, int bc)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        if ((is_md[s] != 0) != (md_flag != 0)) continue;
        int a = start[s], n = count[s];
        for (int i = a; i < a + n; i++) {
            R vv[3] = {v.vel.x[i], v.vel.y[i], v.vel.z[i]};
            R x[3] = {v.pos.x[i] + dt * vv[0] + dt_sq * v.force.x[i],
                      v.pos.y[i] + dt * vv[1] + dt_sq * v.force.y[i],
                      v.pos.z[i] + dt * vv[2] + dt_sq * v.force.z[i]};
            bool collide = false;
            R overtime = 0;
            if (x[dim] < (R)0) {
                collide = true;
                overtime = x[dim] / vv[dim];
            } else if ((double)x[dim] > Lw) {
                collide = true;
                overtime = (x[dim] - (R)Lw) / vv[dim];
            }
            if (collide) {
                if (bc == BOUNCE_BACK_BC) {
                    for (int k = 0; k < 3; k++) vv[k] = -vv[k];
                    for (int k = 0; k < 3; k++) x[k] = x[k] + (R)2 * overtime * vv[k];
                } else if (bc == SPECULAR_BC) {
                    vv[dim] = -vv[dim];
                    x[dim] = x[dim] + (R)2 * overtime * vv[dim];
                }
                v.vel.x[i] = vv[0];
                v.vel.y[i] = vv[1];
                v.vel.z[i] = vv[2];
            }
            v.pos.x[i] = x[0];
            v.pos.y[i] = x[1];
            v.pos.z[i] = x[2];
        }
    }
}

// apply_pbc, src/md.f90:202-217
template <typename R>
__global__ void k_apply_pbc(PView<R> v, double e0, double e1, double e2)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x)
        apply_pbc_one(v, i, e0, e1, e2);
}

// rattle_dimer_pos, src/md.f90:265-296
__global__ void k_rattle_pos(PView<double> v, const double *rx, const double *ry, const double *rz,
                             Masses ms, double d, double dt, E3 L, unsigned *err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    rattle_pos_dimer(v, rx, ry, rz, ms, d, dt, L, err);
}

// rattle_dimer_vel, src/md.f90:298-319
__global__ void k_rattle_vel(PView<double> v, Masses ms, double d, E3 L, unsigned *err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    rattle_vel_dimer(v, ms, d, L, err);
}

// colloid VV halves, programs/single_dimer_pbc.f90:312-315 and :356-359
__global__ void k_colloid_vv_pos(PView<double> v, const double *mass, double dt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.N; i += gridDim.x * blockDim.x)
        colloid_vv_pos_one(v, i, mass[i], dt);
}

__global__ void k_colloid_vv_vel(PView<double> v, const double *mass, double dt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < v.N; i += gridDim.x * blockDim.x)
        colloid_vv_vel_one(v, i, mass[i], dt);
}

// per-particle masses cached on the device (re-uploaded only on change)
struct MassCache {
    const rmpcd_particles *owner = nullptr;
    std::vector<double> host;
    double *dev = nullptr;
    int cap = 0;
};
static MassCache g_mass;

static int mass_on_device(const rmpcd_particles *p, const double *mass, const double **out)
{
    int N = p->N;
    bool same = g_mass.owner == p && (int)g_mass.host.size() == N &&
                memcmp(g_mass.host.data(), mass, sizeof(double) * (size_t)N) == 0;
    if (!same) {
        if (g_mass.cap < N) {
            cudaStreamSynchronize(stream());
            cudaFree(g_mass.dev);
            g_mass.dev = nullptr;
            RMPCD_CUDA_TRY(cudaMalloc(&g_mass.dev, sizeof(double) * (size_t)(N > 0 ? N : 1)));
            g_mass.cap = N;
        }
        g_mass.host.assign(mass, mass + N);
        g_mass.owner = p;
        RMPCD_CUDA_TRY(cudaMemcpyAsync(g_mass.dev, g_mass.host.data(), sizeof(double) * (size_t)N,
                                       cudaMemcpyHostToDevice, stream()));
    }
    *out = g_mass.dev;
    return RMPCD_OK;
}

// Fixed device scratch of rmpcd_colloid_vv_pos_noalloc: the masses of at most
// kNoAllocMaxParticles particles (64 KB), part of the library image, so the
// entry point never calls the allocator.  Nothing in it has to start at zero:
// every call writes the first N entries before its kernel reads them.
constexpr int kNoAllocMaxParticles = 8192;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_noalloc_mass[kNoAllocMaxParticles];

// address of g_noalloc_mass on the current device, looked up once per device
static int noalloc_mass_scratch(double **out)
{
    static double *addr[kNoAllocMaxDevices] = {};
    int dev = 0;
    RMPCD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return fail(RMPCD_ERR_CAPACITY, "rmpcd_colloid_vv_pos_noalloc: device %d is above the %d devices it tracks",
                    dev, kNoAllocMaxDevices);
    if (!addr[dev]) {
        double *a = nullptr;
        RMPCD_CUDA_TRY(cudaGetSymbolAddress((void **)&a, g_noalloc_mass));
        addr[dev] = a;
    }
    *out = addr[dev];
    return RMPCD_OK;
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

extern "C" {

int rmpcd_md_pos(rmpcd_particles *p, double dt)
{
    RMPCD_ARG(p, "null argument");
    if (p->N == 0) return RMPCD_OK;
    PhaseTimer t("md_pos");
    double dt_sq = dt * dt / 2;
    int g = grid_for(p->N, 256);
    DISPATCH_R(p, (k_md_pos<float><<<g, 256, 0, stream()>>>(cur<float>(p), (float)dt, (float)dt_sq)),
               (k_md_pos<double><<<g, 256, 0, stream()>>>(cur<double>(p), dt, dt_sq)));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_md_vel(rmpcd_particles *p, double dt)
{
    RMPCD_ARG(p, "null argument");
    if (p->N == 0) return RMPCD_OK;
    PhaseTimer t("md_vel");
    int g = grid_for(p->N, 256);
    DISPATCH_R(p, (k_md_vel<float><<<g, 256, 0, stream()>>>(cur<float>(p), (float)dt)),
               (k_md_vel<double><<<g, 256, 0, stream()>>>(cur<double>(p), dt)));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_cell_md_pos(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag)
{
    RMPCD_ARG(c && p, "null argument");
    PhaseTimer t("md_pos");
    double dt_sq = dt * dt / 2;
    int g = grid_full(c->S, 128);
    DISPATCH_R(p,
               (k_cell_md_pos<float><<<g, 128, 0, stream()>>>(c->count, c->start, c->is_md, c->S, cur<float>(p),
                                                               (float)dt, (float)dt_sq, md_flag)),
               (k_cell_md_pos<double><<<g, 128, 0, stream()>>>(c->count, c->start, c->is_md, c->S, cur<double>(p),
                                                                dt, dt_sq, md_flag)));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_cell_md_vel(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag)
{
    RMPCD_ARG(c && p, "null argument");
    PhaseTimer t("md_vel");
    int g = grid_full(c->S, 128);
    DISPATCH_R(p,
               (k_cell_md_vel<float><<<g, 128, 0, stream()>>>(c->count, c->start, c->is_md, c->S, cur<float>(p),
                                                               (float)dt, md_flag)),
               (k_cell_md_vel<double><<<g, 128, 0, stream()>>>(c->count, c->start, c->is_md, c->S, cur<double>(p),
                                                                dt, md_flag)));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

static int cell_md_pos_wall(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag, int dim)
{
    RMPCD_ARG(c && p, "null argument");
    PhaseTimer t("md_pos");
    double dt_sq = dt * dt / 2;
    int g = grid_full(c->S, 128);
    DISPATCH_R(p,
               (k_cell_md_pos_wall<float><<<g, 128, 0, stream()>>>(c->count, c->start, c->is_md, c->S,
                                                                    cur<float>(p), (float)dt, (float)dt_sq,
                                                                    md_flag, dim, c->edges[dim], c->bc[dim])),
               (k_cell_md_pos_wall<double><<<g, 128, 0, stream()>>>(c->count, c->start, c->is_md, c->S,
                                                                     cur<double>(p), dt, dt_sq, md_flag, dim,
                                                                     c->edges[dim], c->bc[dim])));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_cell_md_pos_ywall(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag)
{
    return cell_md_pos_wall(c, p, dt, md_flag, 1);
}

int rmpcd_cell_md_pos_zwall(rmpcd_cells *c, rmpcd_particles *p, double dt, int md_flag)
{
    return cell_md_pos_wall(c, p, dt, md_flag, 2);
}

int rmpcd_apply_pbc(rmpcd_particles *p, const double edges[3])
{
    RMPCD_ARG(p && edges, "null argument");
    if (p->N == 0) return RMPCD_OK;
    PhaseTimer t("apply_pbc");
    int g = grid_for(p->N, 256);
    DISPATCH_R(p, (k_apply_pbc<float><<<g, 256, 0, stream()>>>(cur<float>(p), edges[0], edges[1], edges[2])),
               (k_apply_pbc<double><<<g, 256, 0, stream()>>>(cur<double>(p), edges[0], edges[1], edges[2])));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

static Masses masses_of(const rmpcd_particles *p)
{
    Masses ms;
    for (int k = 0; k < RMPCD_MAX_SPECIES; k++) ms.m[k] = p->mass[k];
    ms.n = p->n_species;
    return ms;
}

// rattle_dimer_pos, src/md.f90:265-296; masses are mass(species(1)) and
// mass(species(2)), read on the device
int rmpcd_rattle_dimer_pos(rmpcd_particles *p, double d, double dt, const double edges[3])
{
    RMPCD_ARG(p && edges, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64 && p->N >= 2, "rattle_dimer_pos: needs an FP64 system of >= 2 particles");
    RMPCD_ARG(p->pos_rattle[0] != nullptr, "rattle_dimer_pos: pos_rattle was never set");
    E3 L = {{edges[0], edges[1], edges[2]}};
    PhaseTimer t("rattle_pos");
    k_rattle_pos<<<1, 32, 0, stream()>>>(cur<double>(p), (const double *)p->pos_rattle[0],
                                         (const double *)p->pos_rattle[1], (const double *)p->pos_rattle[2],
                                         masses_of(p), d, dt, L, dev_error_word());
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

// rattle_dimer_vel, src/md.f90:298-319
int rmpcd_rattle_dimer_vel(rmpcd_particles *p, double d, double dt, const double edges[3])
{
    (void)dt;
    RMPCD_ARG(p && edges, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64 && p->N >= 2, "rattle_dimer_vel: needs an FP64 system of >= 2 particles");
    E3 L = {{edges[0], edges[1], edges[2]}};
    PhaseTimer t("rattle_vel");
    k_rattle_vel<<<1, 32, 0, stream()>>>(cur<double>(p), masses_of(p), d, L, dev_error_word());
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_colloid_vv_pos(rmpcd_particles *p, double dt, const double *mass)
{
    RMPCD_ARG(p && mass, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64, "colloid integrator needs an FP64 system");
    if (p->N == 0) return RMPCD_OK;
    const double *dm = nullptr;
    int rc = mass_on_device(p, mass, &dm);
    if (rc) return rc;
    k_colloid_vv_pos<<<grid_for(p->N, 128), 128, 0, stream()>>>(cur<double>(p), dm, dt);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_colloid_vv_vel(rmpcd_particles *p, double dt, const double *mass)
{
    RMPCD_ARG(p && mass, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64, "colloid integrator needs an FP64 system");
    if (p->N == 0) return RMPCD_OK;
    const double *dm = nullptr;
    int rc = mass_on_device(p, mass, &dm);
    if (rc) return rc;
    k_colloid_vv_vel<<<grid_for(p->N, 128), 128, 0, stream()>>>(cur<double>(p), dm, dt);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_colloid_vv_pos_noalloc(rmpcd_particles *p, double dt, const double *mass)
{
    RMPCD_ARG(p && mass, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64, "colloid integrator needs an FP64 system");
    if (p->N > kNoAllocMaxParticles)
        return fail(RMPCD_ERR_CAPACITY,
                    "rmpcd_colloid_vv_pos_noalloc: N = %d is above its fixed scratch of %d particles "
                    "(use rmpcd_colloid_vv_pos)",
                    p->N, kNoAllocMaxParticles);
    double *dm = nullptr;
    int rc = noalloc_mass_scratch(&dm);
    if (rc) return rc;
    if (p->N == 0) return RMPCD_OK;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(dm, mass, sizeof(double) * (size_t)p->N, cudaMemcpyHostToDevice, stream()));
    k_colloid_vv_pos<<<grid_for(p->N, 128), 128, 0, stream()>>>(cur<double>(p), dm, dt);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

}  // extern "C"
