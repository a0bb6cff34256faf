// neighbor_list_t on the GPU (src/neighbor_list.f90): the cell stencil, the
// colloid -> solvent list built from the sorted cell lists, the list-based
// Lennard-Jones forces and the O(C^2) colloid-colloid forces.
//
// Order fidelity: list entries follow the reference's single-thread order
// (stencil order, then in-cell order); colloid force sums and energies are
// accumulated sequentially in list order; a solvent particle touched by one
// list entry gets force - f directly, one touched by several gets its
// subtractions in (colloid, entry) order.
#include <cmath>
#include <cstring>
#include <vector>

#include "keys.cuh"
#include "nlist_ops.cuh"
#include "sortcore.cuh"
#include "rmpcd_common.cuh"
#include "state.cuh"
#include "stepops.cuh"
#include "timers.cuh"

namespace rmpcd {

constexpr int kNlThreads = kNlBlockThreads;

// one block per colloid; the candidate cells of each stencil chunk are staged
// in nl_stage_bytes<R>() of dynamic shared memory by bulk copies
template <typename R>
__global__ void __launch_bounds__(kNlThreads)
    k_update_list(Grid g, const double *cx, const double *cy, const double *cz, const int *cs, const R *sx,
                  const R *sy, const R *sz, const int *sspec, const int *count, const int *start,
                  const int *stencil, int n_stencil, double radiussq, LJDev lj, int do_lj, int Nmax, int *list,
                  int *n_out, unsigned char *is_md, unsigned char *is_reac, unsigned *err)
{
    extern __shared__ __align__(16) unsigned char nl_stage[];
    __shared__ __align__(8) unsigned long long bar;
    update_list_block<R>(blockIdx.x, g, cx, cy, cz, cs, sx, sy, sz, sspec, count, start, stencil, n_stencil,
                         radiussq, lj, do_lj, Nmax, list, n_out, is_md, is_reac, err, NlStage{nl_stage, &bar});
}

template <typename R>
static int update_list_smem(size_t *bytes)
{
    static bool set = false;
    *bytes = nl_stage_bytes<R>();
    if (!set) {
        RMPCD_CUDA_TRY(cudaFuncSetAttribute(k_update_list<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)*bytes));
        set = true;
    }
    return RMPCD_OK;
}

// PAST_MD <- MD, MD cleared, for every solvent particle (src/neighbor_list.f90:180-188)
__global__ void k_flag_roll(int *flags, int N)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        flag_roll_one(flags, i);
}

// pair forces of every list entry (src/neighbor_list.f90:198-219)
template <typename R>
__global__ void k_pair_forces(const double *cx, const double *cy, const double *cz, const int *cs,
                              const R *sx, const R *sy, const R *sz, const int *sspec, int *sflags,
                              const int *list, const int *n, int Nmax, double L0, double L1, double L2,
                              LJDev lj, double *pf, double *pe, unsigned char *contrib, int *ncontrib,
                              int *max_contrib, const int *gate)
{
    if (gate && *gate) return;
    const int i = blockIdx.y;
    const int ni = n[i];
    const double x[3] = {cx[i], cy[i], cz[i]};
    const int s1 = cs[i];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ni; e += gridDim.x * blockDim.x)
        pair_force_entry((size_t)i * Nmax + e, x, s1, sx, sy, sz, sspec, sflags, list, L0, L1, L2, lj, pf, pe,
                         contrib, ncontrib, max_contrib);
}

// solvent force - f for particles with exactly one contribution; the others
// are collected for k_apply_multi
template <typename R>
__global__ void k_apply_single(const int *list, const int *n, int Nmax, const unsigned char *contrib,
                               const double *pf, const int *ncontrib, R *fx, R *fy, R *fz,
                               unsigned long long *mkeys, int *m_count, const int *gate)
{
    if (gate && *gate) return;
    const int i = blockIdx.y;
    const int ni = n[i];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ni; e += gridDim.x * blockDim.x)
        apply_single_or_collect((size_t)i * Nmax + e, list, contrib, pf, ncontrib, fx, fy, fz, mkeys, m_count);
}

template <typename R>
__global__ void k_apply_multi(const int *list, const int *n, int C, int Nmax, const unsigned char *contrib,
                              const double *pf, const int *ncontrib, int *max_contrib, int serial,
                              R *fx, R *fy, R *fz, const unsigned long long *mkeys, int *m_count,
                              const int *gate)
{
    if (gate && *gate) return;
    // the largest contribution count, read by every thread before thread 0
    // clears it for the next evaluation
    const int mc = *max_contrib;
    __syncthreads();
    if (threadIdx.x == 0) *max_contrib = 0;
    if (mc < 2) return;
    const int m = *m_count;
    if (!apply_multi_sorted_block(mkeys, m, pf, fx, fy, fz))
        apply_multi_block(list, n, C, Nmax, contrib, pf, ncontrib, serial, fx, fy, fz);
    __syncthreads();
    if (threadIdx.x == 0) *m_count = 0;
}

// f1 = sum of the pair forces in list order; force(:,i) = force(:,i) + f1
// (kSum = false: only the contributing entries compacted into clist / cn)
template <bool kSum>
__global__ void k_colloid_sum(const int *n, int Nmax, const unsigned char *contrib, const double *pf,
                              double *cfx, double *cfy, double *cfz, int *clist, int *cn, const int *gate)
{
    if (gate && *gate) return;
    colloid_sum_block<kSum>(blockIdx.x, n, Nmax, contrib, pf, cfx, cfy, cfz, clist, cn);
}

// the FP32 form: f1 by the fixed tree of colloid_tree_block
__global__ void __launch_bounds__(kNlBlockThreads) k_colloid_tree(const int *n, int Nmax, const unsigned char *contrib,
                                                                  const double *pf, double *cfx, double *cfy,
                                                                  double *cfz, const int *gate)
{
    if (gate && *gate) return;
    colloid_tree_block(blockIdx.x, n, Nmax, contrib, pf, cfx, cfy, cfz);
}

// Sequential sum e = (((0 + t_0) + t_1) + ...) of `total` terms, one block:
// thread 0 adds a chunk held in shared memory while warps 1.. load the next
// chunk, so the add chain never waits on a global load.
constexpr int kSumChunk = 2048;

template <typename Get>
__device__ void ordered_sum_block(Get get, long long total, double *out)
{
    __shared__ double buf[2][kSumChunk];
    const int t = threadIdx.x, nt = blockDim.x;
    const long long nch = (total + kSumChunk - 1) / kSumChunk;
    auto load = [&](long long c, double *dst, int t0, int nthr) {
        const long long b = c * kSumChunk;
        const int m = (int)(total - b < kSumChunk ? total - b : kSumChunk);
        for (int j = t0; j < m; j += nthr) dst[j] = get(b + j);
    };
    double e = 0;
    if (nch > 0) load(0, buf[0], t, nt);
    __syncthreads();
    for (long long c = 0; c < nch; c++) {
        if (t == 0) {
            const long long b = c * kSumChunk;
            const int m = (int)(total - b < kSumChunk ? total - b : kSumChunk);
            const double *x = buf[c & 1];
#pragma unroll 8
            for (int j = 0; j < m; j++) e = e + x[j];
        } else if (t >= 32 && c + 1 < nch) {
            load(c + 1, buf[(c + 1) & 1], t - 32, nt - 32);
        }
        __syncthreads();
    }
    if (t == 0) *out = e;
}

// e = sum of pair energies in (colloid, entry) order: the contributing
// entries of colloid i are clist[i*Nmax + 0 .. cn[i]-1]; an exclusive scan of
// cn (into pre, C + 1 ints) turns a position in that order into (i, k).
__global__ void __launch_bounds__(1024) k_energy(const int *cn, const int *clist, int C, int Nmax, const double *pe,
                                                 int *pre, double *out)
{
    __shared__ int wsum[32];
    __shared__ int carry;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int b = 0; b < C; b += blockDim.x) {
        const int i = b + t;
        const int v = i < C ? cn[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            int z = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, z, o);
                if (lane >= o) z += y;
            }
            wsum[lane] = z;
        }
        __syncthreads();
        const int incl = x + (w > 0 ? wsum[w - 1] : 0) + carry;
        if (i < C) pre[i] = incl - v;
        __syncthreads();
        if (t == (int)blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (t == 0) pre[C] = carry;
    __syncthreads();
    const long long total = pre[C];
    ordered_sum_block(
        [&](long long f) {
            int lo = 0, hi = C;  // largest i with pre[i] <= f
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (pre[mid] <= f) lo = mid;
                else hi = mid;
            }
            const size_t q = (size_t)lo * Nmax;
            return pe[q + clist[q + (f - pre[lo])]];
        },
        total, out);
}

__global__ void k_reset_contrib(const int *list, const int *n, int Nmax, const unsigned char *contrib,
                                int *ncontrib, const int *gate)
{
    if (gate && *gate) return;
    const int i = blockIdx.y;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n[i]; e += gridDim.x * blockDim.x) {
        size_t q = (size_t)i * Nmax + e;
        if (contrib[q]) ncontrib[list[q]] = 0;
    }
}

// compute_force_n2, src/neighbor_list.f90:227-264: a thread per colloid for
// a few colloids, a block per colloid for many
__global__ void k_force_n2(const double *px, const double *py, const double *pz, const int *sp, int C,
                           double L0, double L1, double L2, LJDev lj, double *fx, double *fy, double *fz,
                           const int *gate)
{
    if (gate && *gate) return;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < C; m += gridDim.x * blockDim.x)
        force_n2_one(m, px, py, pz, sp, C, L0, L1, L2, lj, fx, fy, fz);
}

__global__ void __launch_bounds__(kNlBlockThreads)
    k_force_n2_blocks(const double *px, const double *py, const double *pz, const int *sp, int C, double L0,
                      double L1, double L2, LJDev lj, double *fx, double *fy, double *fz, const int *gate)
{
    if (gate && *gate) return;
    force_n2_block(blockIdx.x, px, py, pz, sp, C, L0, L1, L2, lj, fx, fy, fz);
}

// the pair energies of compute_force_n2 in the reference's (i, j > i) order,
// 0 for pairs beyond the cut (adding +0.0 leaves the sum unchanged: a
// round-to-nearest sum starting at +0.0 is never -0.0), block i writes row i
__global__ void k_energy_n2_terms(const double *px, const double *py, const double *pz, const int *sp, int C,
                                  double L0, double L1, double L2, LJDev lj, double *terms)
{
    const int i = blockIdx.x;
    const long long row = (long long)i * C - (long long)i * (i + 1) / 2;
    for (int j = i + 1 + threadIdx.x; j < C; j += blockDim.x) {
        double d0 = min_image_d(px[i] - px[j], L0);
        double d1 = min_image_d(py[i] - py[j], L1);
        double d2 = min_image_d(pz[i] - pz[j], L2);
        double r_sq = d0 * d0 + d1 * d1 + d2 * d2;
        int s1 = sp[i], s2 = sp[j];
        double e = 0;
        if (r_sq <= lj.cut_sq[(s1 - 1) + lj.n1 * (s2 - 1)]) {
            int tt = (s2 - 1) + lj.n1 * (s1 - 1);
            e = lj_energy(r_sq, lj.epsilon[tt], lj.sigma[tt], lj.cut_energy[tt]);
        }
        terms[row + (j - i - 1)] = e;
    }
}

__global__ void __launch_bounds__(1024) k_energy_sum(const double *terms, long long total, double *out)
{
    ordered_sum_block([&](long long f) { return terms[f]; }, total, out);
}

// a single thread for a few colloids
__global__ void k_energy_n2(const double *px, const double *py, const double *pz, const int *sp, int C,
                            double L0, double L1, double L2, LJDev lj, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double e = 0;
    for (int i = 0; i < C; i++)
        for (int j = i + 1; j < C; j++) {
            double d0 = min_image_d(px[i] - px[j], L0);
            double d1 = min_image_d(py[i] - py[j], L1);
            double d2 = min_image_d(pz[i] - pz[j], L2);
            double r_sq = d0 * d0 + d1 * d1 + d2 * d2;
            int s1 = sp[i], s2 = sp[j];
            if (r_sq <= lj.cut_sq[(s1 - 1) + lj.n1 * (s2 - 1)]) {
                int tt = (s2 - 1) + lj.n1 * (s1 - 1);
                e = e + lj_energy(r_sq, lj.epsilon[tt], lj.sigma[tt], lj.cut_energy[tt]);
            }
        }
    *out = e;
}

static int ensure_force_scratch(rmpcd_nlist *nl, int N2)
{
    if (!nl->pair_f) {
        size_t ne = (size_t)nl->Npoints * nl->Nmax;
        RMPCD_CUDA_TRY(cudaMalloc(&nl->pair_f, 3 * ne * sizeof(double) + 8));
        RMPCD_CUDA_TRY(cudaMalloc(&nl->pair_e, ne * sizeof(double) + 8));
        RMPCD_CUDA_TRY(cudaMalloc(&nl->contrib, ne + 8));
        RMPCD_CUDA_TRY(cudaMalloc(&nl->d_status, (2 * nl->Npoints + 16 + ne) * sizeof(int)));
        RMPCD_CUDA_TRY(cudaMalloc(&nl->mkeys, kMultiSortMax * sizeof(unsigned long long)));
        RMPCD_CUDA_TRY(cudaMalloc(&nl->e_pre, ((size_t)nl->Npoints + 1) * sizeof(int)));
        RMPCD_CUDA_TRY(cudaMemsetAsync(nl->d_status, 0, 16 * sizeof(int), stream()));
    }
    if (nl->ncontrib_cap < N2) {
        cudaStreamSynchronize(stream());
        cudaFree(nl->ncontrib);
        RMPCD_CUDA_TRY(cudaMalloc(&nl->ncontrib, (size_t)(N2 > 0 ? N2 : 1) * sizeof(int)));
        RMPCD_CUDA_TRY(cudaMemsetAsync(nl->ncontrib, 0, (size_t)(N2 > 0 ? N2 : 1) * sizeof(int), stream()));
        nl->ncontrib_cap = N2;
    }
    return RMPCD_OK;
}

}  // namespace rmpcd

using namespace rmpcd;

extern "C" {

int rmpcd_nlist_init(rmpcd_nlist **out, int Npoints, int Nmax)
{
    RMPCD_ARG(out, "null argument");
    RMPCD_ARG(Npoints >= 0 && Nmax >= 1, "neighbor_list_t%init: Npoints >= 0 and Nmax >= 1 required");
    rmpcd_nlist *nl = new rmpcd_nlist();
    nl->Npoints = Npoints;
    nl->Nmax = Nmax;
    size_t ne = (size_t)(Npoints > 0 ? Npoints : 1) * Nmax;
    if (cudaMalloc(&nl->list, ne * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&nl->n, (size_t)(Npoints > 0 ? Npoints : 1) * sizeof(int)) != cudaSuccess) {
        cudaFree(nl->list);
        delete nl;
        return fail(RMPCD_ERR_CUDA, "neighbor_list_t%%init: device allocation failed");
    }
    cudaMemsetAsync(nl->list, 0xff, ne * sizeof(int), stream());
    cudaMemsetAsync(nl->n, 0, (size_t)(Npoints > 0 ? Npoints : 1) * sizeof(int), stream());
    *out = nl;
    return sync();
}

int rmpcd_nlist_destroy(rmpcd_nlist *nl)
{
    if (!nl) return RMPCD_OK;
    ncolloids_forget(nl);
    cudaStreamSynchronize(stream());
    cudaFree(nl->list);
    cudaFree(nl->n);
    cudaFree(nl->stencil);
    cudaFree(nl->pair_f);
    cudaFree(nl->pair_e);
    cudaFree(nl->contrib);
    cudaFree(nl->ncontrib);
    cudaFree(nl->d_status);
    cudaFree(nl->mkeys);
    cudaFree(nl->e_pre);
    delete nl;
    return RMPCD_OK;
}

// make_stencil, src/neighbor_list.f90:271-308 (closest, :310-322)
int rmpcd_nlist_make_stencil(rmpcd_nlist *nl, rmpcd_cells *c, double cut)
{
    RMPCD_ARG(nl && c, "null argument");
    int max_i = (int)floor(cut / c->a) + 1;
    std::vector<int> st;
    for (int i = -max_i; i <= max_i; i++)
        for (int j = -max_i; j <= max_i; j++)
            for (int k = -max_i; k <= max_i; k++) {
                int o[3] = {i, j, k};
                int dist_sq = 0;
                for (int d = 0; d < 3; d++) {
                    int v = abs(o[d]) - 1;
                    if (v < 0) v = 0;
                    dist_sq += v * v;
                }
                if (sqrt((double)dist_sq) < cut) {
                    st.push_back(i);
                    st.push_back(j);
                    st.push_back(k);
                }
            }
    cudaStreamSynchronize(stream());
    cudaFree(nl->stencil);
    nl->stencil = nullptr;
    nl->n_stencil = (int)(st.size() / 3);
    nl->max_i = max_i;
    for (int k = 0; k < 3; k++) nl->box_cells[k] = c->L[k];
    RMPCD_CUDA_TRY(cudaMalloc(&nl->stencil, st.size() * sizeof(int) + 4));
    RMPCD_CUDA_TRY(cudaMemcpyAsync(nl->stencil, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice,
                                   stream()));
    return sync();
}

int rmpcd_nlist_stencil_size(const rmpcd_nlist *nl, int *n)
{
    RMPCD_ARG(nl && n, "null argument");
    *n = nl->n_stencil;
    return RMPCD_OK;
}

int rmpcd_nlist_update(rmpcd_nlist *nl, rmpcd_particles *s1, rmpcd_particles *s2, double radius,
                       rmpcd_cells *c, const rmpcd_lj *lj)
{
    RMPCD_ARG(nl && s1 && s2 && c, "null argument");
    RMPCD_ARG(s1->precision == RMPCD_FP64, "update_list: system1 (colloids) must be FP64");
    RMPCD_ARG(s1->N == nl->Npoints, "update_list: system1 size differs from Npoints");
    RMPCD_ARG(nl->stencil != nullptr, "update_list: make_stencil was not called");
    PhaseTimer t("neigh list update");
    cudaStream_t s = stream();
    RMPCD_CUDA_TRY(cudaMemsetAsync(c->is_md, 0, (size_t)c->S, s));
    RMPCD_CUDA_TRY(cudaMemsetAsync(c->is_reac, 1, (size_t)c->S, s));
    if (s1->N == 0) return RMPCD_OK;
    PView<double> cv = cur<double>(s1);
    LJDev ld = lj_dev(lj);
    size_t smem = 0;
    if (s2->precision == RMPCD_FP32) {
        int rc = update_list_smem<float>(&smem);
        if (rc) return rc;
        PView<float> v = cur<float>(s2);
        k_update_list<float><<<s1->N, kNlThreads, smem, s>>>(grid_of(c), cv.pos.x, cv.pos.y, cv.pos.z, cv.species,
                                                          v.pos.x, v.pos.y, v.pos.z, v.species, c->count, c->start,
                                                          nl->stencil, nl->n_stencil, radius * radius, ld,
                                                          lj ? 1 : 0, nl->Nmax, nl->list, nl->n, c->is_md,
                                                          c->is_reac, dev_error_word());
    } else {
        int rc = update_list_smem<double>(&smem);
        if (rc) return rc;
        PView<double> v = cur<double>(s2);
        k_update_list<double><<<s1->N, kNlThreads, smem, s>>>(grid_of(c), cv.pos.x, cv.pos.y, cv.pos.z, cv.species,
                                                           v.pos.x, v.pos.y, v.pos.z, v.species, c->count, c->start,
                                                           nl->stencil, nl->n_stencil, radius * radius, ld,
                                                           lj ? 1 : 0, nl->Nmax, nl->list, nl->n, c->is_md,
                                                           c->is_reac, dev_error_word());
    }
    RMPCD_CHECK_LAUNCH();
    return check_dev_error(nullptr);
}

int rmpcd_nlist_download(const rmpcd_nlist *nl, int *list, int *n)
{
    RMPCD_ARG(nl, "null argument");
    size_t ne = (size_t)nl->Npoints * nl->Nmax;
    if (list && ne) {
        RMPCD_CUDA_TRY(cudaMemcpyAsync(list, nl->list, ne * sizeof(int), cudaMemcpyDeviceToHost, stream()));
    }
    if (n && nl->Npoints)
        RMPCD_CUDA_TRY(cudaMemcpyAsync(n, nl->n, (size_t)nl->Npoints * sizeof(int), cudaMemcpyDeviceToHost, stream()));
    int rc = sync();
    if (rc) return rc;
    if (list && n)
        for (int i = 0; i < nl->Npoints; i++)
            for (int e = 0; e < nl->Nmax; e++) {
                size_t q = (size_t)i * nl->Nmax + e;
                list[q] = e < n[i] ? list[q] + 1 : 0;
            }
    return RMPCD_OK;
}

// compute_force, src/neighbor_list.f90:159-225
int rmpcd_compute_force(rmpcd_particles *ps1, rmpcd_particles *ps2, rmpcd_nlist *nl, const double L[3],
                        const rmpcd_lj *lj, double *energy)
{
    return compute_force_impl(ps1, ps2, nl, L, lj, energy, true);
}

}  // extern "C"

namespace rmpcd {

// the force kernels of compute_force_n2 (src/neighbor_list.f90:227-264) on st
static void launch_force_n2(rmpcd_particles *ps, const double L[3], const rmpcd_lj *lj, cudaStream_t st,
                            const int *gate = nullptr)
{
    const int C = ps->N;
    PView<double> v = cur<double>(ps);
    LJDev ld = lj_dev(lj);
    if (C <= 32)
        k_force_n2<<<1, 32, 0, st>>>(v.pos.x, v.pos.y, v.pos.z, v.species, C, L[0], L[1], L[2], ld, v.force.x,
                                     v.force.y, v.force.z, gate);
    else
        k_force_n2_blocks<<<C, kNlBlockThreads, 0, st>>>(v.pos.x, v.pos.y, v.pos.z, v.species, C, L[0], L[1], L[2],
                                                         ld, v.force.x, v.force.y, v.force.z, gate);
}

int compute_force_impl(rmpcd_particles *ps1, rmpcd_particles *ps2, rmpcd_nlist *nl, const double L[3],
                       const rmpcd_lj *lj, double *energy, bool roll_flags, const ForceN2Branch *n2)
{
    RMPCD_ARG(ps1 && ps2 && nl && L && lj, "null argument");
    RMPCD_ARG(ps1->precision == RMPCD_FP64, "compute_force: ps1 (colloids) must be FP64");
    RMPCD_ARG(ps1->N == nl->Npoints, "compute_force: ps1 size differs from Npoints");
    int rc = ensure_force_scratch(nl, ps2->N);
    if (rc) return rc;
    PhaseTimer tm("neigh list force");
    cudaStream_t s = stream();
    int C = ps1->N;
    const int *gate = n2 ? n2->gate : nullptr;
    if (roll_flags && ps2->N > 0) k_flag_roll<<<grid_for(ps2->N, 256), 256, 0, s>>>(ps2->flags[ps2->cur], ps2->N);
    int *max_contrib = nl->d_status;
    int *m_count = nl->d_status + 1;  // multi-contribution keys collected (reset by k_apply_multi)
    int *cn = nl->d_status + 16;
    int *clist = nl->d_status + 16 + 2 * nl->Npoints;
    double *e_out = (double *)ps1->d_sums;
    // k_apply_multi leaves max_contrib at zero and the scratch starts at zero,
    // so the n_colloids loop (n2 given) skips this clear; other callers keep it
    if (!n2) RMPCD_CUDA_TRY(cudaMemsetAsync(max_contrib, 0, sizeof(int), s));
    ps2->force_zero = false;
    ps1->force_zero = false;
    if (C > 0) {
        PView<double> cv = cur<double>(ps1);
        LJDev ld = lj_dev(lj);
        int gx = (nl->Nmax + 255) / 256;
        if (gx > 64) gx = 64;
        dim3 grid(gx, C);
        // duplicates inside one list exist only when the stencil wraps the box
        int serial = 0;
        for (int k = 0; k < 3; k++)
            if (2 * nl->max_i + 1 > nl->box_cells[k]) serial = 1;
        if (ps2->precision == RMPCD_FP32) {
            PView<float> v = cur<float>(ps2);
            k_pair_forces<float><<<grid, 256, 0, s>>>(cv.pos.x, cv.pos.y, cv.pos.z, cv.species, v.pos.x, v.pos.y,
                                                      v.pos.z, v.species, v.flags, nl->list, nl->n, nl->Nmax, L[0],
                                                      L[1], L[2], ld, nl->pair_f, nl->pair_e, nl->contrib,
                                                      nl->ncontrib, max_contrib, gate);
        } else {
            PView<double> v = cur<double>(ps2);
            k_pair_forces<double><<<grid, 256, 0, s>>>(cv.pos.x, cv.pos.y, cv.pos.z, cv.species, v.pos.x, v.pos.y,
                                                       v.pos.z, v.species, v.flags, nl->list, nl->n, nl->Nmax, L[0],
                                                       L[1], L[2], ld, nl->pair_f, nl->pair_e, nl->contrib,
                                                       nl->ncontrib, max_contrib, gate);
        }
        // the colloid sums (and with n2 the colloid-colloid forces after them)
        // only read the pair terms and write the colloid forces: with n2 they
        // run on the second stream while the solvent forces are applied
        const bool fork = n2 && !energy;
        cudaStream_t sc = s;
        if (fork) {
            RMPCD_CUDA_TRY(cudaEventRecord(n2->ev_fork, s));
            RMPCD_CUDA_TRY(cudaStreamWaitEvent(n2->side, n2->ev_fork, 0));
            sc = n2->side;
        }
        // the colloid sums: list order in the FP64 form, the fixed tree in the
        // FP32 form (whose energy still needs the compacted entries)
        if (ps2->precision == RMPCD_FP32) {
            k_colloid_tree<<<C, kNlBlockThreads, 0, sc>>>(nl->n, nl->Nmax, nl->contrib, nl->pair_f, cv.force.x,
                                                          cv.force.y, cv.force.z, gate);
            if (energy)
                k_colloid_sum<false><<<C, kNlThreads, 0, sc>>>(nl->n, nl->Nmax, nl->contrib, nl->pair_f, cv.force.x,
                                                               cv.force.y, cv.force.z, clist, cn, gate);
        } else {
            k_colloid_sum<true><<<C, kNlThreads, 0, sc>>>(nl->n, nl->Nmax, nl->contrib, nl->pair_f, cv.force.x,
                                                          cv.force.y, cv.force.z, clist, cn, gate);
        }
        if (fork) {
            launch_force_n2(ps1, L, n2->lj_cc, sc, gate);
            RMPCD_CUDA_TRY(cudaEventRecord(n2->ev_join, sc));
        }
        if (ps2->precision == RMPCD_FP32) {
            PView<float> v = cur<float>(ps2);
            k_apply_single<float><<<grid, 256, 0, s>>>(nl->list, nl->n, nl->Nmax, nl->contrib, nl->pair_f,
                                                       nl->ncontrib, v.force.x, v.force.y, v.force.z, nl->mkeys, m_count,
                                                       gate);
            k_apply_multi<float><<<1, 1024, 0, s>>>(nl->list, nl->n, C, nl->Nmax, nl->contrib, nl->pair_f,
                                                   nl->ncontrib, max_contrib, serial, v.force.x, v.force.y, v.force.z, nl->mkeys,
                                                   m_count, gate);
        } else {
            PView<double> v = cur<double>(ps2);
            k_apply_single<double><<<grid, 256, 0, s>>>(nl->list, nl->n, nl->Nmax, nl->contrib, nl->pair_f,
                                                        nl->ncontrib, v.force.x, v.force.y, v.force.z, nl->mkeys, m_count,
                                                       gate);
            k_apply_multi<double><<<1, 1024, 0, s>>>(nl->list, nl->n, C, nl->Nmax, nl->contrib, nl->pair_f,
                                                    nl->ncontrib, max_contrib, serial, v.force.x, v.force.y, v.force.z, nl->mkeys,
                                                   m_count, gate);
        }
        k_reset_contrib<<<grid, 256, 0, s>>>(nl->list, nl->n, nl->Nmax, nl->contrib, nl->ncontrib, gate);
        if (energy) k_energy<<<1, 1024, 0, s>>>(cn, clist, C, nl->Nmax, nl->pair_e, nl->e_pre, e_out);
        if (fork) RMPCD_CUDA_TRY(cudaStreamWaitEvent(s, n2->ev_join, 0));
        RMPCD_CHECK_LAUNCH();
    }
    if (energy) {
        if (C > 0) {
            RMPCD_CUDA_TRY(cudaMemcpyAsync(energy, e_out, sizeof(double), cudaMemcpyDeviceToHost, s));
            return sync();
        }
        *energy = 0;
    }
    return RMPCD_OK;
}

}  // namespace rmpcd

extern "C" {

// compute_force_n2, src/neighbor_list.f90:227-264
int rmpcd_compute_force_n2(rmpcd_particles *ps, const double L[3], const rmpcd_lj *lj, double *energy)
{
    RMPCD_ARG(ps && L && lj, "null argument");
    RMPCD_ARG(ps->precision == RMPCD_FP64, "compute_force_n2: needs an FP64 system");
    PhaseTimer tm("self force");
    cudaStream_t s = stream();
    int C = ps->N;
    ps->force_zero = false;
    double *e_out = ps->d_sums + 1;
    if (C > 0) {
        PView<double> v = cur<double>(ps);
        LJDev ld = lj_dev(lj);
        if (energy && C <= 32) {
            k_energy_n2<<<1, 32, 0, s>>>(v.pos.x, v.pos.y, v.pos.z, v.species, C, L[0], L[1], L[2], ld, e_out);
        } else if (energy) {
            const long long np = (long long)C * (C - 1) / 2;
            if (ps->n2_cap < np) {
                cudaStreamSynchronize(s);
                cudaFree(ps->n2_terms);
                ps->n2_terms = nullptr;
                ps->n2_cap = 0;
                RMPCD_CUDA_TRY(cudaMalloc(&ps->n2_terms, (size_t)np * sizeof(double)));
                ps->n2_cap = np;
            }
            k_energy_n2_terms<<<C, 128, 0, s>>>(v.pos.x, v.pos.y, v.pos.z, v.species, C, L[0], L[1], L[2], ld,
                                                ps->n2_terms);
            k_energy_sum<<<1, 1024, 0, s>>>(ps->n2_terms, np, e_out);
        }
        launch_force_n2(ps, L, lj, s);
        RMPCD_CHECK_LAUNCH();
    }
    if (energy) {
        if (C > 0) {
            RMPCD_CUDA_TRY(cudaMemcpyAsync(energy, e_out, sizeof(double), cudaMemcpyDeviceToHost, s));
            return sync();
        }
        *energy = 0;
    }
    return RMPCD_OK;
}

}  // extern "C"
