// cell_system_t on the GPU (src/cell_system.f90): slot tables, the key
// lookup table, counting and the random grid shift.
#include <cstring>
#include <vector>

#include "keys.cuh"
#include "rng.cuh"
#include "scan.cuh"
#include "sortcore.cuh"
#include "timers.cuh"

namespace rmpcd {

__global__ void k_build_lut(int *lut, int L0, int L1, int L2, int M0, int M1, int M2)
{
    int n = L0 * L1 * L2;
    int M[3] = {M0, M1, M2};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int p[3] = {c % L0, (c / L0) % L1, c / (L0 * L1)};
        lut[c] = hilbert::compact_index(p, M);
    }
}

}  // namespace rmpcd

using namespace rmpcd;

static void free_cells(rmpcd_cells *c)
{
    if (!c) return;
    cudaFree(c->count);
    cudaFree(c->start);
    cudaFree(c->cursor);
    cudaFree(c->count_next);
    cudaFree(c->start_next);
    cudaFree(c->is_md);
    cudaFree(c->is_reac);
    cudaFree(c->lut);
    cudaFree(c->scan_tmp);
    cudaFree(c->axes);
    cudaFree(c->d_red);
    delete c;
}

extern "C" {

// cell_system_t%init, src/cell_system.f90:49-84
int rmpcd_cells_init(rmpcd_cells **out, const int L[3], double a, int has_walls)
{
    RMPCD_ARG(out && L, "null argument");
    RMPCD_ARG(L[0] > 0 && L[1] > 0 && L[2] > 0, "cell_system_t%init: L must be positive");
    RMPCD_ARG(a > 0, "cell_system_t%init: a must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(RMPCD_ERR_NO_DEVICE, "no CUDA device visible");
    rmpcd_cells *c = new rmpcd_cells();
    for (int k = 0; k < 3; k++) {
        c->L[k] = L[k];
        c->edges[k] = L[k] * a;
        c->origin[k] = 0.0;
        c->bc[k] = RMPCD_PERIODIC_BC;
    }
    c->has_walls = has_walls ? 1 : 0;
    if (c->has_walls) c->L[2] = L[2] + 1;
    c->a = a;
    c->max_v = 0.0;
    for (int k = 0; k < 3; k++) {
        c->M[k] = 1;
        while ((1LL << c->M[k]) < c->L[k]) c->M[k]++;
    }
    if (c->M[0] + c->M[1] + c->M[2] > 27) {
        delete c;
        return fail(RMPCD_ERR_CAPACITY, "cell_system_t%%init: 2^(M1+M2+M3) above 2^27 slots");
    }
    c->S = (1 << c->M[0]) * (1 << c->M[1]) * (1 << c->M[2]);
    c->n_lut = c->L[0] * c->L[1] * c->L[2];
    c->scan_blocks = scan_blocks_for(c->S);
    c->red_cap = 4 * 4096;
    size_t S = (size_t)c->S;
    cudaStream_t s = stream();
    if (cudaMalloc(&c->count, S * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->start, S * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->cursor, S * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->count_next, S * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->start_next, S * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->is_md, S) != cudaSuccess || cudaMalloc(&c->is_reac, S) != cudaSuccess ||
        cudaMalloc(&c->lut, (size_t)c->n_lut * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->scan_tmp, (size_t)c->scan_blocks * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->d_red, (size_t)c->red_cap * sizeof(double)) != cudaSuccess) {
        free_cells(c);
        return fail(RMPCD_ERR_CUDA, "cell_system_t%%init: device allocation failed (S=%d)", (int)S);
    }
    cudaMemsetAsync(c->count, 0, S * sizeof(int), s);
    cudaMemsetAsync(c->start, 0, S * sizeof(int), s);
    cudaMemsetAsync(c->cursor, 0, S * sizeof(int), s);
    cudaMemsetAsync(c->count_next, 0, S * sizeof(int), s);
    cudaMemsetAsync(c->start_next, 0, S * sizeof(int), s);
    cudaMemsetAsync(c->is_md, 0, S, s);
    cudaMemsetAsync(c->is_reac, 0, S, s);
    k_build_lut<<<grid_for(c->n_lut, 256), 256, 0, s>>>(c->lut, c->L[0], c->L[1], c->L[2], c->M[0],
                                                        c->M[1], c->M[2]);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_cells(c);
        return fail(RMPCD_ERR_CUDA, "cell_system_t%%init: %s", cudaGetErrorString(e));
    }
    *out = c;
    return RMPCD_OK;
}

int rmpcd_cells_destroy(rmpcd_cells *c)
{
    if (!c) return RMPCD_OK;
    ncolloids_forget(c);
    cudaStreamSynchronize(stream());
    free_cells(c);
    return RMPCD_OK;
}

int rmpcd_cells_info(const rmpcd_cells *c, int L[3], int M[3], int *S, double edges[3])
{
    RMPCD_ARG(c, "null cell system");
    for (int k = 0; k < 3; k++) {
        if (L) L[k] = c->L[k];
        if (M) M[k] = c->M[k];
        if (edges) edges[k] = c->edges[k];
    }
    if (S) *S = c->S;
    return RMPCD_OK;
}

int rmpcd_cells_set_origin(rmpcd_cells *c, const double origin[3])
{
    RMPCD_ARG(c && origin, "null argument");
    for (int k = 0; k < 3; k++) c->origin[k] = origin[k];
    return RMPCD_OK;
}

int rmpcd_cells_get_origin(const rmpcd_cells *c, double origin[3])
{
    RMPCD_ARG(c && origin, "null argument");
    for (int k = 0; k < 3; k++) origin[k] = c->origin[k];
    return RMPCD_OK;
}

int rmpcd_cells_set_bc(rmpcd_cells *c, const int bc[3])
{
    RMPCD_ARG(c && bc, "null argument");
    for (int k = 0; k < 3; k++) {
        RMPCD_ARG(bc[k] >= 1 && bc[k] <= 3, "boundary condition must be 1, 2 or 3");
        c->bc[k] = bc[k];
    }
    return RMPCD_OK;
}

int rmpcd_cells_set_max_v(rmpcd_cells *c, double max_v)
{
    RMPCD_ARG(c, "null argument");
    c->max_v = max_v;
    return RMPCD_OK;
}

// random_shift, src/cell_system.f90:153-163: origin(k) = u_k - 1
int rmpcd_cells_random_shift(rmpcd_cells *c, rmpcd_rng *r)
{
    RMPCD_ARG(c && r, "null argument");
    double u0, u1, u2, u3;
    rng::uniform2(r->seed, r->step, 0, rng::SHIFT, 0, u0, u1);
    rng::uniform2(r->seed, r->step, 1, rng::SHIFT, 0, u2, u3);
    c->origin[0] = u0 - 1;
    c->origin[1] = u1 - 1;
    c->origin[2] = u2 - 1;
    r->step++;
    return RMPCD_OK;
}

// count_particles, src/cell_system.f90:86-129
int rmpcd_cells_count_particles(rmpcd_cells *c, rmpcd_particles *p)
{
    RMPCD_ARG(c && p, "null argument");
    PhaseTimer t("count");
    return count_and_scan(c, p, false);
}

// sort_particles, src/cell_system.f90:131-151
int rmpcd_cells_sort_particles(rmpcd_cells *c, const rmpcd_particles *position_old, rmpcd_particles *position_new)
{
    RMPCD_ARG(c && position_old && position_new, "null argument");
    RMPCD_ARG(position_old != position_new, "sort_particles: position_old and position_new must be different systems");
    RMPCD_ARG(position_old->N == position_new->N && position_old->precision == position_new->precision,
              "sort_particles: both systems need the same size and precision");
    PhaseTimer t("sort");
    return sort_positions(c, position_old, position_new);
}

static int dl(const void *src, void *dst, size_t bytes)
{
    RMPCD_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream()));
    RMPCD_CUDA_TRY(cudaStreamSynchronize(stream()));
    return RMPCD_OK;
}

int rmpcd_cells_download_count(const rmpcd_cells *c, int *count)
{
    RMPCD_ARG(c && count, "null argument");
    return dl(c->count, count, (size_t)c->S * sizeof(int));
}

int rmpcd_cells_download_start(const rmpcd_cells *c, int *start)
{
    RMPCD_ARG(c && start, "null argument");
    int rc = dl(c->start, start, (size_t)c->S * sizeof(int));
    if (rc) return rc;
    for (int s = 0; s < c->S; s++) start[s] += 1;
    return RMPCD_OK;
}

int rmpcd_cells_download_is_md(const rmpcd_cells *c, unsigned char *v)
{
    RMPCD_ARG(c && v, "null argument");
    return dl(c->is_md, v, (size_t)c->S);
}

int rmpcd_cells_download_is_reac(const rmpcd_cells *c, unsigned char *v)
{
    RMPCD_ARG(c && v, "null argument");
    return dl(c->is_reac, v, (size_t)c->S);
}

int rmpcd_cells_upload_is_md(rmpcd_cells *c, const unsigned char *v)
{
    RMPCD_ARG(c && v, "null argument");
    RMPCD_CUDA_TRY(cudaMemcpyAsync(c->is_md, v, (size_t)c->S, cudaMemcpyHostToDevice, stream()));
    return sync();
}

int rmpcd_cells_upload_is_reac(rmpcd_cells *c, const unsigned char *v)
{
    RMPCD_ARG(c && v, "null argument");
    RMPCD_CUDA_TRY(cudaMemcpyAsync(c->is_reac, v, (size_t)c->S, cudaMemcpyHostToDevice, stream()));
    return sync();
}

int rmpcd_cells_set_axes(rmpcd_cells *c, const double *axes)
{
    RMPCD_ARG(c, "null cell system");
    if (!axes) {
        if (c->axes) {
            cudaStreamSynchronize(stream());
            cudaFree(c->axes);
        }
        c->axes = nullptr;
        return RMPCD_OK;
    }
    if (!c->axes) RMPCD_CUDA_TRY(cudaMalloc(&c->axes, 3 * (size_t)c->S * sizeof(double)));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(c->axes, axes, 3 * (size_t)c->S * sizeof(double),
                                   cudaMemcpyHostToDevice, stream()));
    return sync();
}

}  // extern "C"
