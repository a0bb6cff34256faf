// particle_system_t on the GPU (src/particle_system.f90): allocation, host
// transfers in the reference (3,N) layout, sort, displacement bounds, random
// placement and Maxwell initial velocities.
#include <cstring>
#include <string>
#include <vector>

#include "keys.cuh"
#include "rng.cuh"
#include "sortcore.cuh"
#include "stepops.cuh"
#include "timers.cuh"

namespace rmpcd {

// (3,N) host layout <-> SoA device layout through a device staging buffer
template <typename R, typename H>
__global__ void k_deinterleave(const H *__restrict__ in, int N, R *x, R *y, R *z)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        x[i] = (R)in[3 * i];
        y[i] = (R)in[3 * i + 1];
        z[i] = (R)in[3 * i + 2];
    }
}

template <typename R, typename H>
__global__ void k_interleave(const R *x, const R *y, const R *z, int N, H *__restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        out[3 * i] = (H)x[i];
        out[3 * i + 1] = (H)y[i];
        out[3 * i + 2] = (H)z[i];
    }
}

__global__ void k_iota1(int *a, int N)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        a[i] = (int)i + 1;
}

__global__ void k_id_to_idx(const int *id, int N, int *out)
{
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < N;
         j += (long long)gridDim.x * blockDim.x) {
        int v = id[j];
        if (v >= 1 && v <= N) out[v - 1] = (int)j + 1;
    }
}

// particles with a non-finite position or velocity component (one atomic
// per warp that found any)
template <typename R>
__global__ void k_count_nonfinite(Vec3<R> pos, Vec3<R> vel, long long N, unsigned long long *out)
{
    for (long long base = (long long)blockIdx.x * blockDim.x; base < N; base += (long long)gridDim.x * blockDim.x) {
        const long long i = base + threadIdx.x;
        bool bad = false;
        if (i < N)
            bad = !(isfinite(pos.x[i]) && isfinite(pos.y[i]) && isfinite(pos.z[i]) && isfinite(vel.x[i]) &&
                    isfinite(vel.y[i]) && isfinite(vel.z[i]));
        const unsigned b = __ballot_sync(0xffffffffu, bad);
        if (b && (threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)__popc(b));
    }
}

// maximum_displacement, src/particle_system.f90:357-378
template <typename R>
__global__ void k_max_disp(Vec3<R> pos, Vec3<R> old, const int *species, int N,
                           unsigned long long *out)
{
    double m = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        double r = disp_sq_one(pos, old, species, i);
        m = m > r ? m : r;
    }
    warp_max_into(out, m);
}

// cell_maximum_displacement, src/particle_system.f90:380-410
template <typename R>
__global__ void k_cell_max_disp(const int *count, const int *start, const unsigned char *is_md,
                                int S, Vec3<R> pos, Vec3<R> old, const int *species,
                                unsigned long long *out)
{
    double m = 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        if (!is_md[s]) continue;
        int a = start[s], n = count[s];
        for (int i = a; i < a + n; i++) {
            if (species[i] >= 0) {
                double d0 = (double)pos.x[i] - (double)old.x[i];
                double d1 = (double)pos.y[i] - (double)old.y[i];
                double d2 = (double)pos.z[i] - (double)old.z[i];
                double r = d0 * d0 + d1 * d1 + d2 * d2;
                m = m > r ? m : r;
            }
        }
    }
    warp_max_into(out, m);
}

// random_placement, src/particle_system.f90:250-302: uniform positions,
// rejected within cut_sq(s1, s2) of any obstacle; attempt a of particle i
// draws Philox(seed, 0, i, PLACE, 2a) and (.., 2a+1)
template <typename R>
__global__ void k_place(Vec3<R> pos, const int *species, int N, double L0, double L1, double L2,
                        const double *cx, const double *cy, const double *cz, const int *cs,
                        int C, const double *cut_sq, int n1, uint64_t seed)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        int s1 = species ? species[i] : 1;
        double x0 = 0, x1 = 0, x2 = 0;
        for (uint32_t a = 0; a < (1u << 20); a++) {
            double u0, u1, w0, w1;
            rng::uniform2(seed, 0, (uint32_t)i, rng::PLACE, 2 * a, u0, u1);
            rng::uniform2(seed, 0, (uint32_t)i, rng::PLACE, 2 * a + 1, w0, w1);
            x0 = u0 * L0;
            x1 = u1 * L1;
            x2 = w0 * L2;
            bool tooclose = false;
            for (int j = 0; j < C; j++) {
                // species outside the LJ table have no exclusion radius
                if (s1 < 1 || s1 > n1 || cs[j] < 1 || cs[j] > RMPCD_MAX_SPECIES) continue;
                double r0 = min_image_d(x0 - cx[j], L0);
                double r1 = min_image_d(x1 - cy[j], L1);
                double r2 = min_image_d(x2 - cz[j], L2);
                double rsq = r0 * r0 + r1 * r1 + r2 * r2;
                if (rsq < cut_sq[(s1 - 1) + n1 * (cs[j] - 1)]) {
                    tooclose = true;
                    break;
                }
            }
            if (!tooclose) break;
        }
        pos.x[i] = (R)x0;
        pos.y[i] = (R)x1;
        pos.z[i] = (R)x2;
    }
}

// normal * sqrt(T) per component (programs/single_dimer_pbc.f90:240-244)
__global__ void k_maxwell(double *vx, double *vy, double *vz, int N, double st, uint64_t seed)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        vx[i] = rng::normal(seed, rng::kInitStep, (uint32_t)i, 0) * st;
        vy[i] = rng::normal(seed, rng::kInitStep, (uint32_t)i, 1) * st;
        vz[i] = rng::normal(seed, rng::kInitStep, (uint32_t)i, 2) * st;
    }
}

template <typename R>
__global__ void k_sub_mean(R *v, int N, const double *sum)
{
    double m = *sum / N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        v[i] = (R)((double)v[i] - m);
}

template <typename A, typename B>
__global__ void k_convert(const A *a, B *b, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = (B)a[i];
}

// sum(vel, dim=2) in the reference's sequential order.  Initialisation only:
// the column is summed on the host, where a dependent chain of N adds runs
// at full clock, and the result goes back to d_out.
int fixed_order_sum(const double *a, int N, double *d_out)
{
    std::vector<double> h((size_t)(N > 0 ? N : 1));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(h.data(), a, sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost, stream()));
    RMPCD_CUDA_TRY(cudaStreamSynchronize(stream()));
    double s = 0;
    for (int i = 0; i < N; i++) s = s + h[(size_t)i];
    RMPCD_CUDA_TRY(cudaMemcpyAsync(d_out, &s, sizeof(double), cudaMemcpyHostToDevice, stream()));
    RMPCD_CUDA_TRY(cudaStreamSynchronize(stream()));
    return RMPCD_OK;
}

int launch_max_disp(rmpcd_particles *p)
{
    cudaStream_t s = stream();
    RMPCD_CUDA_TRY(cudaMemsetAsync(p->d_max, 0, 8, s));
    if (p->N > 0) {
        if (p->precision == RMPCD_FP32) {
            PView<float> a = cur<float>(p), b = alt<float>(p);
            k_max_disp<float><<<grid_for(p->N, 256), 256, 0, s>>>(a.pos, b.pos, a.species, p->N, p->d_max);
        } else {
            PView<double> a = cur<double>(p), b = alt<double>(p);
            k_max_disp<double><<<grid_for(p->N, 256), 256, 0, s>>>(a.pos, b.pos, a.species, p->N, p->d_max);
        }
        RMPCD_CHECK_LAUNCH();
    }
    return RMPCD_OK;
}

int launch_cell_max_disp(rmpcd_cells *c, rmpcd_particles *p)
{
    cudaStream_t s = stream();
    RMPCD_CUDA_TRY(cudaMemsetAsync(p->d_max, 0, 8, s));
    if (p->precision == RMPCD_FP32) {
        PView<float> a = cur<float>(p), b = alt<float>(p);
        k_cell_max_disp<float><<<grid_full(c->S, 256), 256, 0, s>>>(c->count, c->start, c->is_md, c->S, a.pos,
                                                                   b.pos, a.species, p->d_max);
    } else {
        PView<double> a = cur<double>(p), b = alt<double>(p);
        k_cell_max_disp<double><<<grid_full(c->S, 256), 256, 0, s>>>(c->count, c->start, c->is_md, c->S, a.pos,
                                                                    b.pos, a.species, p->d_max);
    }
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

}  // namespace rmpcd

using namespace rmpcd;

static void free_particles(rmpcd_particles *p)
{
    if (!p) return;
    for (int b = 0; b < 2; b++) {
        for (int k = 0; k < 3; k++) {
            cudaFree(p->pos[b][k]);
            cudaFree(p->vel[b][k]);
            cudaFree(p->force[b][k]);
            cudaFree(p->force_old[b][k]);
            cudaFree(p->image[b][k]);
        }
        cudaFree(p->id[b]);
        cudaFree(p->species[b]);
        cudaFree(p->flags[b]);
    }
    for (int k = 0; k < 3; k++) cudaFree(p->pos_rattle[k]);
    cudaFree(p->key);
    cudaFree(p->perm);
    cudaFree(p->id_to_idx);
    cudaFree(p->gauss);
    cudaFree(p->d_max);
    cudaFree(p->d_sums);
    cudaFree(p->d_ints);
    cudaFree(p->stage);
    cudaFree(p->rec[0]);
    cudaFree(p->rec[1]);
    cudaFree(p->n2_terms);
    delete p;
}

static bool is_real_field(const std::string &f)
{
    return f == "pos" || f == "pos_old" || f == "vel" || f == "force" || f == "force_old" ||
           f == "pos_rattle";
}

template <typename R>
static R *const *real_arrays(rmpcd_particles *p, const std::string &f)
{
    int c = p->cur;
    if (f == "pos") return (R *const *)p->pos[c];
    if (f == "pos_old") return (R *const *)p->pos[1 - c];
    if (f == "vel") return (R *const *)p->vel[c];
    if (f == "force") return (R *const *)p->force[c];
    if (f == "force_old") return (R *const *)p->force_old[c];
    if (f == "pos_rattle") return (R *const *)p->pos_rattle;
    return nullptr;
}

// staging buffer for the (3,N) host layout, allocated on first transfer
static int stage_of(rmpcd_particles *p, void **out)
{
    size_t need = 3 * (size_t)p->N * sizeof(double) + 16;
    if (p->stage_bytes < need) {
        cudaStreamSynchronize(stream());
        cudaFree(p->stage);
        p->stage = nullptr;
        p->stage_bytes = 0;
        RMPCD_CUDA_TRY(cudaMalloc(&p->stage, need));
        p->stage_bytes = need;
    }
    *out = p->stage;
    return RMPCD_OK;
}

template <typename R>
static int upload_real(rmpcd_particles *p, const std::string &f, const double *host)
{
    size_t n3 = 3 * (size_t)p->N;
    double *stage = nullptr;
    int rc = stage_of(p, (void **)&stage);
    if (rc) return rc;
    cudaStream_t s = stream();
    RMPCD_CUDA_TRY(cudaMemcpyAsync(stage, host, n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    R *const *a = real_arrays<R>(p, f);
    k_deinterleave<R, double><<<grid_for(p->N, 256), 256, 0, s>>>(stage, p->N, a[0], a[1], a[2]);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "upload %s: %s", f.c_str(), cudaGetErrorString(e));
    if (f == "force") p->force_zero = false;
    if (f == "force_old") p->force_old_zero = false;
    return RMPCD_OK;
}

template <typename R>
static int download_real(rmpcd_particles *p, const std::string &f, double *host)
{
    size_t n3 = 3 * (size_t)p->N;
    double *stage = nullptr;
    int rc = stage_of(p, (void **)&stage);
    if (rc) return rc;
    cudaStream_t s = stream();
    R *const *a = real_arrays<R>(p, f);
    k_interleave<R, double><<<grid_for(p->N, 256), 256, 0, s>>>(a[0], a[1], a[2], p->N, stage);
    cudaError_t e = cudaMemcpyAsync(host, stage, n3 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "download %s: %s", f.c_str(), cudaGetErrorString(e));
    return RMPCD_OK;
}

extern "C" {

// particle_system_t%init, src/particle_system.f90:81-184
int rmpcd_particles_init(rmpcd_particles **out, int Nmax, int n_species, const double *mass,
                         int precision)
{
    RMPCD_ARG(out, "null argument");
    RMPCD_ARG(Nmax >= 0, "particle_system_t%init: Nmax must be >= 0");
    RMPCD_ARG(n_species >= 1 && n_species <= RMPCD_MAX_SPECIES, "n_species must be in 1..4");
    RMPCD_ARG(precision == RMPCD_FP64 || precision == RMPCD_FP32, "precision must be 32 or 64");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(RMPCD_ERR_NO_DEVICE, "no CUDA device visible");
    rmpcd_particles *p = new rmpcd_particles();
    p->N = Nmax;
    p->n_species = n_species;
    p->precision = precision;
    p->rsize = precision == RMPCD_FP32 ? 4 : 8;
    if (mass)
        for (int s = 0; s < n_species; s++) p->mass[s] = mass[s];
    // every array is allocated to a multiple of 4 elements: bulk copies read
    // 16-byte windows rounded outward
    size_t n = ((size_t)(Nmax > 0 ? Nmax : 1) + 3) & ~(size_t)3;
    size_t rb = n * p->rsize, ib = n * sizeof(int);
    bool ok = true;
    cudaStream_t st = stream();
    for (int b = 0; b < 2 && ok; b++) {
        for (int k = 0; k < 3 && ok; k++) {
            ok = ok && cudaMalloc(&p->pos[b][k], rb) == cudaSuccess;
            ok = ok && cudaMalloc(&p->vel[b][k], rb) == cudaSuccess;
            ok = ok && cudaMalloc(&p->force[b][k], rb) == cudaSuccess;
            ok = ok && cudaMalloc(&p->force_old[b][k], rb) == cudaSuccess;
            ok = ok && cudaMalloc(&p->image[b][k], ib) == cudaSuccess;
        }
        ok = ok && cudaMalloc(&p->id[b], ib) == cudaSuccess;
        ok = ok && cudaMalloc(&p->species[b], ib) == cudaSuccess;
        ok = ok && cudaMalloc(&p->flags[b], ib) == cudaSuccess;
    }
    ok = ok && cudaMalloc(&p->key, ib) == cudaSuccess;
    ok = ok && cudaMalloc(&p->perm, ib) == cudaSuccess;
    p->sums_cap = 8192;
    ok = ok && cudaMalloc(&p->d_max, 64) == cudaSuccess;
    ok = ok && cudaMalloc(&p->d_sums, (size_t)p->sums_cap * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&p->d_ints, 64 * sizeof(int)) == cudaSuccess;
    if (!ok) {
        free_particles(p);
        return fail(RMPCD_ERR_CUDA, "particle_system_t%%init: device allocation failed (N=%d)", Nmax);
    }
    for (int b = 0; b < 2; b++) {
        for (int k = 0; k < 3; k++) {
            cudaMemsetAsync(p->pos[b][k], 0, rb, st);
            cudaMemsetAsync(p->vel[b][k], 0, rb, st);
            cudaMemsetAsync(p->force[b][k], 0, rb, st);
            cudaMemsetAsync(p->force_old[b][k], 0, rb, st);
            cudaMemsetAsync(p->image[b][k], 0, ib, st);
        }
        cudaMemsetAsync(p->species[b], 0, ib, st);
        cudaMemsetAsync(p->flags[b], 0, ib, st);
        if (Nmax > 0) k_iota1<<<grid_for(Nmax, 256), 256, 0, st>>>(p->id[b], Nmax);
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        free_particles(p);
        return fail(RMPCD_ERR_CUDA, "particle_system_t%%init: %s", cudaGetErrorString(e));
    }
    *out = p;
    return RMPCD_OK;
}

int rmpcd_particles_destroy(rmpcd_particles *p)
{
    if (!p) return RMPCD_OK;
    ncolloids_forget(p);
    cudaStreamSynchronize(stream());
    free_particles(p);
    return RMPCD_OK;
}

int rmpcd_particles_info(const rmpcd_particles *p, int *Nmax, int *n_species, int *precision)
{
    RMPCD_ARG(p, "null particle system");
    if (Nmax) *Nmax = p->N;
    if (n_species) *n_species = p->n_species;
    if (precision) *precision = p->precision;
    return RMPCD_OK;
}

int rmpcd_particles_upload(rmpcd_particles *p, const char *field, const void *host)
{
    RMPCD_ARG(p && field && host, "null argument");
    std::string f(field);
    if (p->N == 0) return RMPCD_OK;
    if (f == "pos_rattle" && !p->pos_rattle[0]) {
        for (int k = 0; k < 3; k++) RMPCD_CUDA_TRY(cudaMalloc(&p->pos_rattle[k], (size_t)p->N * p->rsize));
    }
    if (is_real_field(f)) {
        if (p->precision == RMPCD_FP32) return upload_real<float>(p, f, (const double *)host);
        return upload_real<double>(p, f, (const double *)host);
    }
    cudaStream_t s = stream();
    size_t ib = (size_t)p->N * sizeof(int);
    if (f == "image") {
        int *stage = nullptr;
        int rc = stage_of(p, (void **)&stage);
        if (rc) return rc;
        RMPCD_CUDA_TRY(cudaMemcpyAsync(stage, host, 3 * ib, cudaMemcpyHostToDevice, s));
        k_deinterleave<int, int><<<grid_for(p->N, 256), 256, 0, s>>>(
            stage, p->N, p->image[p->cur][0], p->image[p->cur][1], p->image[p->cur][2]);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "upload image: %s", cudaGetErrorString(e));
        return RMPCD_OK;
    }
    int *dst = nullptr;
    if (f == "id") dst = p->id[p->cur];
    else if (f == "species") dst = p->species[p->cur];
    else if (f == "flags") dst = p->flags[p->cur];
    else return fail(RMPCD_ERR_INVALID, "unknown or read-only particle field '%s'", field);
    RMPCD_CUDA_TRY(cudaMemcpyAsync(dst, host, ib, cudaMemcpyHostToDevice, s));
    return sync();
}

int rmpcd_particles_download(const rmpcd_particles *pc, const char *field, void *host)
{
    RMPCD_ARG(pc && field && host, "null argument");
    rmpcd_particles *p = const_cast<rmpcd_particles *>(pc);
    std::string f(field);
    if (p->N == 0) return RMPCD_OK;
    if (f == "pos_rattle" && !p->pos_rattle[0])
        return fail(RMPCD_ERR_INVALID, "pos_rattle was never set");
    if (is_real_field(f)) {
        if (p->precision == RMPCD_FP32) return download_real<float>(p, f, (double *)host);
        return download_real<double>(p, f, (double *)host);
    }
    cudaStream_t s = stream();
    size_t ib = (size_t)p->N * sizeof(int);
    if (f == "image") {
        int *stage = nullptr;
        int rc = stage_of(p, (void **)&stage);
        if (rc) return rc;
        k_interleave<int, int><<<grid_for(p->N, 256), 256, 0, s>>>(
            p->image[p->cur][0], p->image[p->cur][1], p->image[p->cur][2], p->N, stage);
        cudaError_t e = cudaMemcpyAsync(host, stage, 3 * ib, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "download image: %s", cudaGetErrorString(e));
        return RMPCD_OK;
    }
    const int *src = nullptr;
    if (f == "id") src = p->id[p->cur];
    else if (f == "species") src = p->species[p->cur];
    else if (f == "flags") src = p->flags[p->cur];
    else if (f == "id_to_idx") {
        if (!p->id_to_idx) RMPCD_CUDA_TRY(cudaMalloc(&p->id_to_idx, ib));
        RMPCD_CUDA_TRY(cudaMemsetAsync(p->id_to_idx, 0, ib, s));
        k_id_to_idx<<<grid_for(p->N, 256), 256, 0, s>>>(p->id[p->cur], p->N, p->id_to_idx);
        src = p->id_to_idx;
    } else
        return fail(RMPCD_ERR_INVALID, "unknown particle field '%s'", field);
    RMPCD_CUDA_TRY(cudaMemcpyAsync(host, src, ib, cudaMemcpyDeviceToHost, s));
    return sync();
}

// particle_system_t%sort, src/particle_system.f90:304-355
int rmpcd_particles_sort(rmpcd_particles *p, rmpcd_cells *c)
{
    RMPCD_ARG(p && c, "null argument");
    return sort_particles(c, p);
}

int rmpcd_particles_maximum_displacement(rmpcd_particles *p, double *r)
{
    RMPCD_ARG(p && r, "null argument");
    PhaseTimer t("maximum disp");
    cudaStream_t s = stream();
    int rc0 = launch_max_disp(p);
    if (rc0) return rc0;
    unsigned long long bits = 0;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(&bits, p->d_max, 8, cudaMemcpyDeviceToHost, s));
    int rc = sync();
    if (rc) return rc;
    double m;
    memcpy(&m, &bits, 8);
    *r = sqrt(m);
    return RMPCD_OK;
}

int rmpcd_cell_maximum_displacement(rmpcd_cells *c, rmpcd_particles *p, double delta_t, double *r)
{
    RMPCD_ARG(c && p && r, "null argument");
    cudaStream_t s = stream();
    int rc0 = launch_cell_max_disp(c, p);
    if (rc0) return rc0;
    unsigned long long bits = 0;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(&bits, p->d_max, 8, cudaMemcpyDeviceToHost, s));
    int rc = sync();
    if (rc) return rc;
    double m;
    memcpy(&m, &bits, 8);
    double a = sqrt(m), b = c->max_v * delta_t;
    *r = a > b ? a : b;
    return RMPCD_OK;
}

int rmpcd_particles_random_placement(rmpcd_particles *p, const double L[3], rmpcd_particles *other,
                                     const rmpcd_lj *lj, const rmpcd_rng *state)
{
    RMPCD_ARG(p && L && state, "null argument");
    const uint64_t seed = state->seed;
    RMPCD_ARG((other == nullptr) == (lj == nullptr),
              "other and lj_params must be present/absent together");
    if (p->N == 0) return RMPCD_OK;
    cudaStream_t s = stream();
    const double *cx = nullptr, *cy = nullptr, *cz = nullptr;
    const int *cs = nullptr;
    double *cut = nullptr;
    int C = 0, n1 = 1;
    if (other) {
        RMPCD_ARG(other->precision == RMPCD_FP64, "obstacles must be an FP64 particle system");
        C = other->N;
        cx = (const double *)other->pos[other->cur][0];
        cy = (const double *)other->pos[other->cur][1];
        cz = (const double *)other->pos[other->cur][2];
        cs = other->species[other->cur];
        n1 = lj->n1;
        RMPCD_CUDA_TRY(cudaMalloc(&cut, sizeof(lj->cut_sq)));
        RMPCD_CUDA_TRY(cudaMemcpyAsync(cut, lj->cut_sq, sizeof(lj->cut_sq), cudaMemcpyHostToDevice, s));
    }
    const int *sp = p->species[p->cur];
    if (p->precision == RMPCD_FP32)
        k_place<float><<<grid_for(p->N, 128), 128, 0, s>>>(cur<float>(p).pos, other ? sp : nullptr, p->N,
                                                            L[0], L[1], L[2], cx, cy, cz, cs, C, cut, n1, seed);
    else
        k_place<double><<<grid_for(p->N, 128), 128, 0, s>>>(cur<double>(p).pos, other ? sp : nullptr, p->N,
                                                             L[0], L[1], L[2], cx, cy, cz, cs, C, cut, n1, seed);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(cut);
    if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "random_placement: %s", cudaGetErrorString(e));
    return RMPCD_OK;
}

int rmpcd_particles_maxwell(rmpcd_particles *p, double T, uint64_t seed)
{
    RMPCD_ARG(p, "null argument");
    if (p->N == 0) return RMPCD_OK;
    cudaStream_t s = stream();
    double *tmp = nullptr;
    size_t n = (size_t)p->N;
    RMPCD_CUDA_TRY(cudaMalloc(&tmp, 3 * n * sizeof(double) + 4 * sizeof(double)));
    double *vx = tmp, *vy = tmp + n, *vz = tmp + 2 * n, *sums = tmp + 3 * n;
    k_maxwell<<<grid_for(p->N, 128), 128, 0, s>>>(vx, vy, vz, p->N, sqrt(T), seed);
    int rc = RMPCD_OK;
    double *comp[3] = {vx, vy, vz};
    for (int k = 0; k < 3 && !rc; k++) rc = fixed_order_sum(comp[k], p->N, sums + k);
    for (int k = 0; k < 3 && !rc; k++)
        k_sub_mean<double><<<grid_for(p->N, 256), 256, 0, s>>>(comp[k], p->N, sums + k);
    if (!rc) {
        if (p->precision == RMPCD_FP32) {
            PView<float> v = cur<float>(p);
            float *dst[3] = {v.vel.x, v.vel.y, v.vel.z};
            for (int k = 0; k < 3; k++)
                k_convert<double, float><<<grid_for(p->N, 256), 256, 0, s>>>(comp[k], dst[k], p->N);
        } else {
            PView<double> v = cur<double>(p);
            double *dst[3] = {v.vel.x, v.vel.y, v.vel.z};
            for (int k = 0; k < 3; k++)
                RMPCD_CUDA_TRY(cudaMemcpyAsync(dst[k], comp[k], n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        }
    }
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(tmp);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(RMPCD_ERR_CUDA, "maxwell: %s", cudaGetErrorString(e));
    return RMPCD_OK;
}

int rmpcd_particles_switch_force(rmpcd_particles *p)
{
    RMPCD_ARG(p, "null argument");
    int c = p->cur;
    for (int k = 0; k < 3; k++) {
        void *t = p->force[c][k];
        p->force[c][k] = p->force_old[c][k];
        p->force_old[c][k] = t;
    }
    bool z = p->force_zero;
    p->force_zero = p->force_old_zero;
    p->force_old_zero = z;
    return RMPCD_OK;
}

int rmpcd_particles_zero_force(rmpcd_particles *p)
{
    RMPCD_ARG(p, "null argument");
    if (p->N > 0)
        for (int k = 0; k < 3; k++)
            RMPCD_CUDA_TRY(cudaMemsetAsync(p->force[p->cur][k], 0, (size_t)p->N * p->rsize, stream()));
    p->force_zero = true;
    return RMPCD_OK;
}

int rmpcd_particles_count_nonfinite(const rmpcd_particles *p, long long *n_bad)
{
    RMPCD_ARG(p && n_bad, "null argument");
    *n_bad = 0;
    if (p->N == 0) return RMPCD_OK;
    cudaStream_t s = stream();
    unsigned long long *d = p->d_max;  // the reduction word, free between calls
    RMPCD_CUDA_TRY(cudaMemsetAsync(d, 0, 8, s));
    if (p->precision == RMPCD_FP32) {
        PView<float> v = cur<float>(p);
        k_count_nonfinite<float><<<grid_for(p->N, 256), 256, 0, s>>>(v.pos, v.vel, p->N, d);
    } else {
        PView<double> v = cur<double>(p);
        k_count_nonfinite<double><<<grid_for(p->N, 256), 256, 0, s>>>(v.pos, v.vel, p->N, d);
    }
    RMPCD_CHECK_LAUNCH();
    unsigned long long h = 0;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, s));
    int rc = sync();
    if (!rc) *n_bad = (long long)h;
    return rc;
}

int rmpcd_particles_copy_pos_old(rmpcd_particles *p)
{
    RMPCD_ARG(p, "null argument");
    if (p->N > 0)
        for (int k = 0; k < 3; k++)
            RMPCD_CUDA_TRY(cudaMemcpyAsync(p->pos[1 - p->cur][k], p->pos[p->cur][k], (size_t)p->N * p->rsize,
                                           cudaMemcpyDeviceToDevice, stream()));
    return RMPCD_OK;
}

// force_old = force (programs/single_dimer_pbc.f90:295)
int rmpcd_particles_copy_force_old(rmpcd_particles *p)
{
    RMPCD_ARG(p, "null argument");
    if (p->N > 0)
        for (int k = 0; k < 3; k++)
            RMPCD_CUDA_TRY(cudaMemcpyAsync(p->force_old[p->cur][k], p->force[p->cur][k], (size_t)p->N * p->rsize,
                                           cudaMemcpyDeviceToDevice, stream()));
    p->force_old_zero = p->force_zero;
    return RMPCD_OK;
}

int rmpcd_particles_copy_pos_rattle(rmpcd_particles *p)
{
    RMPCD_ARG(p, "null argument");
    if (p->N == 0) return RMPCD_OK;
    if (!p->pos_rattle[0])
        for (int k = 0; k < 3; k++) RMPCD_CUDA_TRY(cudaMalloc(&p->pos_rattle[k], (size_t)p->N * p->rsize));
    for (int k = 0; k < 3; k++)
        RMPCD_CUDA_TRY(cudaMemcpyAsync(p->pos_rattle[k], p->pos[p->cur][k], (size_t)p->N * p->rsize,
                                       cudaMemcpyDeviceToDevice, stream()));
    return RMPCD_OK;
}

int rmpcd_particles_set_gauss(rmpcd_particles *p, const double *gauss)
{
    RMPCD_ARG(p, "null argument");
    if (!gauss) {
        if (p->gauss) {
            cudaStreamSynchronize(stream());
            cudaFree(p->gauss);
        }
        p->gauss = nullptr;
        return RMPCD_OK;
    }
    if (!p->gauss) RMPCD_CUDA_TRY(cudaMalloc(&p->gauss, 3 * (size_t)p->N * sizeof(double) + 8));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(p->gauss, gauss, 3 * (size_t)p->N * sizeof(double),
                                   cudaMemcpyHostToDevice, stream()));
    return sync();
}

}  // extern "C"
