// MPCD on the GPU (src/mpcd.f90): SRD and MPC-AT collisions, the Lamura wall
// rule, temperature, cell rescaling, streaming with periodic and wall
// boundaries, and bulk reactions.  Collisions run one thread per Hilbert
// slot over the sorted particle ranges (cells hold ~10 particles).
#include <cmath>

#include "cellops.cuh"
#include "hilbert.cuh"
#include "keys.cuh"
#include "rng.cuh"
#include "stepops.cuh"
#include "timers.cuh"

namespace rmpcd {

// simple_mpcd_step, src/mpcd.f90:71-183
template <typename R>
__global__ void k_simple_mpcd(const int *__restrict__ count, const int *__restrict__ start, int S,
                              R *vx, R *vy, R *vz, const int *__restrict__ species, SrdParams q)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x)
        srd_slot<R>(count[s], start[s], s, 0, vx, vy, vz, species, q);
}

// The MPC-AT normals of simple_mpcd_step (src/mpcd.f90:144-160): for every
// particle i with species > 0, (R)(rng::normal(seed, step, i, k) * t_factor)
// for k = 0, 1, 2 into n[k][i].  Each deviate is the first accepted of the
// attempts t = 0, 1, ... of rng::normal, so the values are rng::normal's.  A
// warp takes kAtChunks chunks of 32 particles at a time and deals the
// attempts of their deviates to its lanes: first every lane's attempt 0 of
// its particles' deviates, then the attempts that rejections queue in a ring
// in shared memory, 32 at a time, so no lane waits while another repeats a
// rejection (a deviate drawn by one thread costs its warp the slowest lane's
// attempts) and the last few rejections of a pass leave few lanes idle.
constexpr int kAtThreads = 256;
constexpr int kAtChunks = 8;    // 32-particle chunks per warp pass
constexpr int kAtQueue = 1024;  // ring of queued attempts per warp: at least 96 * kAtChunks

__device__ inline unsigned at_job(int p, int k, int t) { return (unsigned)p | ((unsigned)k << 8) | ((unsigned)t << 10); }

template <typename R>
__global__ void __launch_bounds__(kAtThreads) k_at_normals(const int *__restrict__ species, long long N, SrdParams q,
                                                           R *nx, R *ny, R *nz)
{
    static_assert(kAtChunks * 32 <= 256 && 96 * kAtChunks <= kAtQueue && (kAtQueue & (kAtQueue - 1)) == 0,
                  "job fields and ring size");
    __shared__ unsigned ring[kAtThreads / 32][kAtQueue];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned below = lanemask_lt();
    unsigned *qr = ring[w];
    R *out[3] = {nx, ny, nz};
    const long long warps = (long long)gridDim.x * (kAtThreads / 32);
    const long long span = 32LL * kAtChunks;
    for (long long base = ((long long)blockIdx.x * (kAtThreads / 32) + w) * span; base < N; base += warps * span) {
        // round 0: every lane the attempt 0 of its own particles' deviates
        int tail = 0;
        for (int c = 0; c < kAtChunks; c++) {
            const long long i = base + c * 32 + lane;
            const bool act = i < N && species[i] > 0;
            for (int k = 0; k < 3; k++) {
                double z = 0;
                const bool ok = act && rng::normal_attempt(q.seed, q.step, (uint32_t)i, (uint32_t)k, 0u, &z);
                if (ok) out[k][i] = (R)(z * q.t_factor);
                const unsigned rej = __ballot_sync(0xffffffffu, act && !ok);
                if (act && !ok) qr[(tail + __popc(rej & below)) & (kAtQueue - 1)] = at_job(c * 32 + lane, k, 1);
                tail += __popc(rej);
            }
        }
        __syncwarp();
        // then the queued attempts, 32 at a time; a rejected one queues the
        // deviate's next attempt behind the others (at most 96 * kAtChunks
        // are queued at once, so the ring never overwrites an unread one)
        int head = 0;
        while (head < tail) {
            const int n = min(32, tail - head);
            const bool have = lane < n;
            const unsigned jb = have ? qr[(head + lane) & (kAtQueue - 1)] : 0u;
            head += n;
            const int p = jb & 255, k = (jb >> 8) & 3, t = (int)(jb >> 10);
            const long long ii = base + p;
            double z = 0;
            bool ok = false;
            if (have) {
                // rng::normal gives 0 once its attempts are spent
                ok = t >= (int)rng::kNormalAttempts ||
                     rng::normal_attempt(q.seed, q.step, (uint32_t)ii, (uint32_t)k, (uint32_t)t, &z);
                if (ok) out[k][ii] = (R)(z * q.t_factor);
            }
            const unsigned rej = __ballot_sync(0xffffffffu, have && !ok);
            if (have && !ok) qr[(tail + __popc(rej & below)) & (kAtQueue - 1)] = at_job(p, k, t + 1);
            tail += __popc(rej);
            __syncwarp();
        }
    }
}

// simple_mpcd_step with the MPC-AT thermostat given the normals of
// k_at_normals: the thermostat branch of srd_slot (src/mpcd.f90:126-160) with
// each normal read instead of drawn; vel = normal + dv (hydro) or the normal,
// as srd_slot's store and later add.
template <typename R>
__global__ void k_at_cells(const int *__restrict__ count, const int *__restrict__ start, int S, R *vx, R *vy, R *vz,
                           const int *__restrict__ species, int hydro, const R *__restrict__ nx,
                           const R *__restrict__ ny, const R *__restrict__ nz)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        const int n = count[s];
        if (n <= 1) continue;
        const long long a = start[s];
        int n_eff = 0;
        CellSum<R> sx, sy, sz, wx, wy, wz;
        for (long long i = a; i < a + n; i++) {
            if (species[i] > 0) {
                sx.add(vx[i]);
                sy.add(vy[i]);
                sz.add(vz[i]);
                wx.add(nx[i]);
                wy.add(ny[i]);
                wz.add(nz[i]);
                n_eff++;
            }
        }
        if (n_eff <= 1) continue;
        const R lv[3] = {sx.value() / n_eff, sy.value() / n_eff, sz.value() / n_eff};
        const R dv[3] = {lv[0] - wx.value() / n_eff, lv[1] - wy.value() / n_eff, lv[2] - wz.value() / n_eff};
        for (long long i = a; i < a + n; i++) {
            if (species[i] <= 0) continue;
            if (hydro) {
                vx[i] = nx[i] + dv[0];
                vy[i] = ny[i] + dv[1];
                vz[i] = nz[i] + dv[2];
            } else {
                vx[i] = nx[i];
                vy[i] = ny[i];
                vz[i] = nz[i];
            }
        }
    }
}

// wall_mpcd_step, src/mpcd.f90:193-337
template <typename R>
__global__ void k_wall_mpcd(const int *__restrict__ count, const int *__restrict__ start, int S,
                            int M0, int M1, int M2, int L2, R *vx, R *vy, R *vz, SrdParams q,
                            int has_wall, double wt0, double wt1, int wn0, int wn1, int do_cell_v)
{
    int M[3] = {M0, M1, M2};
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        int n = count[s];
        if (n <= 1) continue;
        int a = start[s];
        int cell[3];
        hilbert::compact_point(s, M, cell);
        int wall_idx = -1;
        if (has_wall && cell[2] + 1 == 1) wall_idx = 0;
        else if (has_wall && cell[2] + 1 == L2) wall_idx = 1;
        int n_virtual = 0;
        double vv[3] = {0, 0, 0};
        int wn = wall_idx == 0 ? wn0 : wn1;
        if (wall_idx >= 0 && n < wn) {
            n_virtual = wn - n;
            for (int k = 0; k < 3; k++) vv[k] = rng::normal(q.seed, q.step, (uint32_t)s, (uint32_t)(3 + k));
            double f = sqrt(n_virtual * (wall_idx == 0 ? wt0 : wt1));
            for (int k = 0; k < 3; k++) vv[k] = vv[k] * f;
        }
        CellSum<R> sx, sy, sz;
        for (int i = a; i < a + n; i++) {
            sx.add(vx[i]);
            sy.add(vy[i]);
            sz.add(vz[i]);
        }
        R lv[3];
        if (n_virtual > 0) {
            lv[0] = (R)(((double)sx.value() + vv[0]) / wn);
            lv[1] = (R)(((double)sy.value() + vv[1]) / wn);
            lv[2] = (R)(((double)sz.value() + vv[2]) / wn);
        } else {
            lv[0] = sx.value() / n;
            lv[1] = sy.value() / n;
            lv[2] = sz.value() / n;
        }
        if (q.thermostat) {
            CellSum<R> wx, wy, wz;
            for (int i = a; i < a + n; i++) {
                R nx = (R)(rng::normal(q.seed, q.step, (uint32_t)i, 0) * q.t_factor);
                R ny = (R)(rng::normal(q.seed, q.step, (uint32_t)i, 1) * q.t_factor);
                R nz = (R)(rng::normal(q.seed, q.step, (uint32_t)i, 2) * q.t_factor);
                vx[i] = nx;
                vy[i] = ny;
                vz[i] = nz;
                wx.add(nx);
                wy.add(ny);
                wz.add(nz);
            }
            if (do_cell_v) {
                R dv[3] = {lv[0] - wx.value() / (R)n, lv[1] - wy.value() / (R)n, lv[2] - wz.value() / (R)n};
                for (int i = a; i < a + n; i++) {
                    vx[i] = vx[i] + dv[0];
                    vy[i] = vy[i] + dv[1];
                    vz[i] = vz[i] + dv[2];
                }
            }
        } else {
            double n0, n1, n2;
            rng::sphere(q.seed, q.step, (uint32_t)s, n0, n1, n2);
            Rot o = srd_matrix(n0, n1, n2, q.sin_a, q.cos_a);
            for (int i = a; i < a + n; i++) {
                R x = vx[i], y = vy[i], z = vz[i];
                srd_rotate(x, y, z, lv, o);
                vx[i] = x;
                vy[i] = y;
                vz[i] = z;
            }
        }
    }
}

constexpr int kRedBlocks = 1024;

// compute_temperature, src/mpcd.f90:342-407: per-block partial (te, count),
// then a fixed-order final sum
template <typename R>
__global__ void k_temperature(const int *__restrict__ count, const int *__restrict__ start, int S,
                              const R *vx, const R *vy, const R *vz, const int *__restrict__ species,
                              double *part)
{
    double te = 0, cnt = 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        int n = count[s];
        if (n <= 1) continue;
        int a = start[s];
        cnt += 1;
        int n_eff = 0;
        CellSum<R> sx, sy, sz;
        for (int i = a; i < a + n; i++) {
            if (species[i] > 0) {
                sx.add(vx[i]);
                sy.add(vy[i]);
                sz.add(vz[i]);
                n_eff++;
            }
        }
        if (n_eff <= 1) continue;
        // local_v = local_v / n  (divides by n, not n_effective, as written)
        double l0 = (double)(sx.value() / (R)n), l1 = (double)(sy.value() / (R)n),
               l2 = (double)(sz.value() / (R)n);
        double kin = 0;
        for (int i = a; i < a + n; i++) {
            if (species[i] > 0) {
                double d0 = (double)vx[i] - l0, d1 = (double)vy[i] - l1, d2 = (double)vz[i] - l2;
                kin = kin + (d0 * d0 + d1 * d1 + d2 * d2);
            }
        }
        kin = kin / (double)(3 * (n_eff - 1));
        te = te + kin;
    }
    __shared__ double ste[256], sc[256];
    ste[threadIdx.x] = te;
    sc[threadIdx.x] = cnt;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            ste[threadIdx.x] += ste[threadIdx.x + o];
            sc[threadIdx.x] += sc[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = ste[0];
        part[2 * blockIdx.x + 1] = sc[0];
    }
}

__global__ void k_temperature_final(const double *part, int nb, double *out)
{
    if (threadIdx.x == 0) {
        double te = 0, cnt = 0;
        for (int b = 0; b < nb; b++) {
            te = te + part[2 * b];
            cnt = cnt + part[2 * b + 1];
        }
        out[0] = te / cnt;
    }
}

// rescale_cells, src/mpcd.f90:748-801
template <typename R>
__global__ void k_rescale(const int *__restrict__ count, const int *__restrict__ start, int S, R *vx,
                          R *vy, R *vz, const int *__restrict__ species, double T)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        int n = count[s];
        if (n <= 1) continue;
        int a = start[s];
        int n_eff = 0;
        CellSum<R> sx, sy, sz;
        for (int i = a; i < a + n; i++) {
            if (species[i] > 0) {
                sx.add(vx[i]);
                sy.add(vy[i]);
                sz.add(vz[i]);
                n_eff++;
            }
        }
        if (n_eff <= 1) continue;
        R lv[3] = {sx.value() / n_eff, sy.value() / n_eff, sz.value() / n_eff};
        double kin = 0;
        for (int i = a; i < a + n; i++) {
            if (species[i] > 0) {
                double d0 = (double)(vx[i] - lv[0]), d1 = (double)(vy[i] - lv[1]),
                       d2 = (double)(vz[i] - lv[2]);
                kin = kin + (d0 * d0 + d1 * d1 + d2 * d2);
            }
        }
        R tf = (R)sqrt((3 * (n_eff - 1)) * T / kin);
        for (int i = a; i < a + n; i++) {
            if (species[i] > 0) {
                vx[i] = lv[0] + tf * (vx[i] - lv[0]);
                vy[i] = lv[1] + tf * (vy[i] - lv[1]);
                vz[i] = lv[2] + tf * (vz[i] - lv[2]);
            }
        }
    }
}

// mpcd_stream_periodic, src/mpcd.f90:440-457
template <typename R>
__global__ void k_stream_periodic(PView<R> v, double e0, double e1, double e2, R dt)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x) {
        R x = v.pos.x[i] + v.vel.x[i] * dt;
        R y = v.pos.y[i] + v.vel.y[i] * dt;
        R z = v.pos.z[i] + v.vel.z[i] * dt;
        int jx = floor_div_edge((double)x, e0), jy = floor_div_edge((double)y, e1), jz = floor_div_edge((double)z, e2);
        if (jx) v.ix[i] += jx;
        if (jy) v.iy[i] += jy;
        if (jz) v.iz[i] += jz;
        v.pos.x[i] = x - (R)(jx * e0);
        v.pos.y[i] = y - (R)(jy * e1);
        v.pos.z[i] = z - (R)(jz * e2);
    }
}

// yzwall_collision, src/mpcd.f90:511-589 (0-based dims y=1, z=2); the wall
// loop stops after 64 crossings and reports it instead of spinning
__device__ inline void yzwall_collision(const double x0[3], const double v0[3], double x[3],
                                        double v[3], const double L[3], double t, const int bc[3],
                                        double gx, unsigned *err)
{
    double gvec[3] = {gx, 0, 0};
    int im[3] = {0, 0, 0};
    int cd = -1;
    double tc = 1.7976931348623157e308;
    for (int i = 1; i <= 2; i++) {
        double tt = v0[i] > 0 ? (L[i] - x0[i]) / v0[i] : -x0[i] / v0[i];
        if ((tt > 0) && (tt < tc)) {
            tc = tt;
            cd = i;
        }
    }
    if (cd < 0) return;
    double tr = t - tc;
    for (int k = 0; k < 3; k++) {
        x[k] = x0[k] + v0[k] * tc + gvec[k] * (tc * tc) / 2;
        v[k] = v0[k] + gvec[k] * tc;
    }
    for (int iter = 0;; iter++) {
        if (bc[cd] == BOUNCE_BACK_BC) {
            for (int k = 0; k < 3; k++) v[k] = -v[k];
        } else if (bc[cd] == SPECULAR_BC) {
            v[cd] = -v[cd];
        } else if (bc[cd] == PERIODIC_BC) {
            int jump = ifloor(x[cd] / L[cd]);
            x[cd] = x[cd] - jump * L[cd];
            im[cd] = im[cd] + jump;
        }
        if (iter >= 64) {
            atomicOr(err, DEV_ERR_WALL_LOOP);
            break;
        }
        cd = cd == 1 ? 2 : 1;
        tc = v[cd] > 0 ? (L[cd] - x[cd]) / v[cd] : -x[cd] / v[cd];
        if ((tc < 0) || (tc > tr)) break;
        for (int k = 0; k < 3; k++) {
            x[k] = x[k] + v[k] * tc + gvec[k] * (tc * tc) / 2;
            v[k] = v[k] + gvec[k] * tc;
        }
        tr = tr - tc;
    }
    tc = tr;
    for (int k = 0; k < 3; k++) {
        x[k] = x[k] + v[k] * tc + gvec[k] * (tc * tc) / 2 + im[k] * L[k];
        v[k] = v[k] + gvec[k] * tc;
    }
}

// mpcd_stream_xforce_yzwall, src/mpcd.f90:464-506
template <typename R>
__global__ void k_stream_yzwall(PView<R> v, double L0, double L1, double L2, int bc0, int bc1, int bc2,
                                double dt, double g, unsigned *err)
{
    double L[3] = {L0, L1, L2};
    int bc[3] = {bc0, bc1, bc2};
    double gvec[3] = {g, 0, 0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x) {
        double op[3] = {(double)v.pos.x[i], (double)v.pos.y[i], (double)v.pos.z[i]};
        double ov[3] = {(double)v.vel.x[i], (double)v.vel.y[i], (double)v.vel.z[i]};
        double np[3], nv[3];
        for (int k = 0; k < 3; k++) {
            np[k] = op[k] + ov[k] * dt + gvec[k] * (dt * dt) / 2;
            nv[k] = ov[k];
        }
        bool y_out = (np[1] < 0) || (np[1] > L[1]);
        bool z_out = (np[2] < 0) || (np[2] > L[2]);
        if (((bc[1] == PERIODIC_BC) && z_out) || ((bc[1] != PERIODIC_BC) && (y_out || z_out))) {
            yzwall_collision(op, ov, np, nv, L, dt, bc, g, err);
            v.flags[i] |= (1 << WALL_BIT);
            v.vel.x[i] = (R)nv[0];
            v.vel.y[i] = (R)nv[1];
            v.vel.z[i] = (R)nv[2];
        }
        v.pos.x[i] = (R)np[0];
        v.pos.y[i] = (R)np[1];
        v.pos.z[i] = (R)np[2];
    }
}

// mpcd_stream_nogravity_zwall, src/mpcd.f90:702-745
template <typename R>
__global__ void k_stream_zwall(PView<R> v, double Lz, double dt)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.N;
         i += (long long)gridDim.x * blockDim.x) {
        double op[3] = {(double)v.pos.x[i], (double)v.pos.y[i], (double)v.pos.z[i]};
        double ov[3] = {(double)v.vel.x[i], (double)v.vel.y[i], (double)v.vel.z[i]};
        double f[3] = {(double)v.force.x[i], (double)v.force.y[i], (double)v.force.z[i]};
        double np[3], nv[3];
        for (int k = 0; k < 3; k++) np[k] = op[k] + ov[k] * dt + f[k] * (dt * dt) / 2;
        bool bounce = false;
        double t_c = 0;
        if (np[2] < 0) {
            t_c = -op[2] / ov[2];
            bounce = true;
        } else if (np[2] > Lz) {
            t_c = (Lz - op[2]) / ov[2];
            bounce = true;
        } else {
            for (int k = 0; k < 3; k++) nv[k] = ov[k];
        }
        if (bounce) {
            for (int k = 0; k < 3; k++) {
                np[k] = np[k] - ov[k] * 2 * (dt - t_c);
                nv[k] = -ov[k];
            }
            v.flags[i] |= (1 << WALL_BIT);
        }
        v.pos.x[i] = (R)np[0];
        v.pos.y[i] = (R)np[1];
        v.pos.z[i] = (R)np[2];
        v.vel.x[i] = (R)nv[0];
        v.vel.y[i] = (R)nv[1];
        v.vel.z[i] = (R)nv[2];
    }
}

// bulk_reaction, src/mpcd.f90:605-643
__global__ void k_bulk_reaction(const int *__restrict__ count, const int *__restrict__ start,
                                const unsigned char *__restrict__ is_reac, int S, int *species,
                                int from, int to, double rate, double tau, uint64_t seed, uint64_t step)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        if ((count[s] <= 1) || !is_reac[s]) continue;
        int a = start[s], n = count[s];
        double local_rate = 0;
        int pick = -1;
        for (int i = a; i < a + n; i++)
            if (species[i] == from) {
                local_rate = local_rate + 1;
                pick = i;
            }
        local_rate = local_rate * rate;
        double u0, u1;
        rng::uniform2(seed, step, (uint32_t)s, rng::BULK, 0, u0, u1);
        if (u0 < (1 - exp(-local_rate * tau)) && pick >= 0) species[pick] = to;
    }
}

// bulk_reaction_endothermic, src/mpcd.f90:645-700: the reaction needs
// kin = sum |v - com_v|^2 / 2 > delta_u in the cell and, when it fires, takes
// delta_u from the cell's relative kinetic energy by scaling v - com_v.  Sums
// run in the cell's particle order, as the reference's per-cell loop does.
template <typename R>
__global__ void k_bulk_reaction_endo(const int *__restrict__ count, const int *__restrict__ start,
                                     const unsigned char *__restrict__ is_reac, int S, PView<R> v, int from,
                                     int to, double rate, double tau, double delta_u, uint64_t seed,
                                     uint64_t step)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        if ((count[s] <= 1) || !is_reac[s]) continue;
        int a = start[s], n = count[s];
        double local_rate = 0;
        int pick = -1;
        double cx = 0, cy = 0, cz = 0;
        for (int i = a; i < a + n; i++) {
            if (v.species[i] == from) {
                local_rate = local_rate + 1;
                pick = i;
            }
            cx = cx + (double)v.vel.x[i];
            cy = cy + (double)v.vel.y[i];
            cz = cz + (double)v.vel.z[i];
        }
        cx = cx / n;
        cy = cy / n;
        cz = cz / n;
        double kin = 0;
        for (int i = a; i < a + n; i++) {
            double dx = (double)v.vel.x[i] - cx, dy = (double)v.vel.y[i] - cy, dz = (double)v.vel.z[i] - cz;
            kin = kin + ((dx * dx + dy * dy) + dz * dz);
        }
        kin = kin / 2;
        if ((local_rate > 0) && (kin > delta_u)) {
            local_rate = local_rate * rate;
            double u0, u1;
            rng::uniform2(seed, step, (uint32_t)s, rng::BULK, 0, u0, u1);
            if (u0 < (1 - exp(-local_rate * tau))) {
                v.species[pick] = to;
                double factor = sqrt((kin - delta_u) / kin);
                for (int i = a; i < a + n; i++) {
                    v.vel.x[i] = (R)(cx + factor * ((double)v.vel.x[i] - cx));
                    v.vel.y[i] = (R)(cy + factor * ((double)v.vel.y[i] - cy));
                    v.vel.z[i] = (R)(cz + factor * ((double)v.vel.z[i] - cz));
                }
            }
        }
    }
}

static SrdParams srd_params(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r, int has_alpha,
                            double alpha, int thermostat, double T, int hydro)
{
    SrdParams q;
    q.sin_a = 1;
    q.cos_a = 0;
    if (has_alpha) {
        q.sin_a = sin(alpha);
        q.cos_a = cos(alpha);
    }
    q.t_factor = thermostat ? sqrt(T) : 0.0;
    q.thermostat = thermostat ? 1 : 0;
    q.hydro = hydro ? 1 : 0;
    q.seed = r ? r->seed : 0;
    q.step = r ? r->step : 0;
    q.axes = c->axes;
    q.gauss = p->gauss;
    return q;
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

int rmpcd_simple_mpcd_step(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r, int has_alpha,
                           double alpha, int thermostat, double T, int hydro)
{
    RMPCD_ARG(p && c && r, "null argument");
    if (!hydro && !thermostat)
        return fail(RMPCD_ERR_STOP, "requiring .not.do_hydro without thermostat in simple_mpcd_step");
    PhaseTimer t("step");
    SrdParams q = srd_params(p, c, r, has_alpha, alpha, thermostat, T, hydro);
    cudaStream_t s = stream();
    int g = grid_full(c->S, 128);
    if (thermostat && !q.gauss && p->N > 0) {
        // the normals first, into the sort target's velocity arrays (free
        // between sorts), then the cells
        const int gn = grid_full(((long long)p->N + 32 * kAtChunks - 1) / (32 * kAtChunks) * 32, kAtThreads);
        DISPATCH_R(p,
                   ({ PView<float> v = cur<float>(p), t = alt<float>(p);
                      k_at_normals<float><<<gn, kAtThreads, 0, s>>>(v.species, p->N, q, t.vel.x, t.vel.y, t.vel.z);
                      k_at_cells<float><<<g, 128, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z,
                                                          v.species, q.hydro, t.vel.x, t.vel.y, t.vel.z); }),
                   ({ PView<double> v = cur<double>(p), t = alt<double>(p);
                      k_at_normals<double><<<gn, kAtThreads, 0, s>>>(v.species, p->N, q, t.vel.x, t.vel.y, t.vel.z);
                      k_at_cells<double><<<g, 128, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z,
                                                           v.species, q.hydro, t.vel.x, t.vel.y, t.vel.z); }));
    } else {
        DISPATCH_R(p,
                   ({ PView<float> v = cur<float>(p);
                      k_simple_mpcd<float><<<g, 128, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z, v.species, q); }),
                   ({ PView<double> v = cur<double>(p);
                      k_simple_mpcd<double><<<g, 128, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z, v.species, q); }));
    }
    RMPCD_CHECK_LAUNCH();
    r->step++;
    return RMPCD_OK;
}

int rmpcd_wall_mpcd_step(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *r,
                         const double wall_temperature[2], const double wall_v[6], const int wall_n[2],
                         int thermostat, double bulk_temperature, int has_alpha, double alpha,
                         int keep_cell_v)
{
    RMPCD_ARG(p && c && r, "null argument");
    bool all_present = wall_temperature && wall_v && wall_n;
    bool all_absent = !wall_temperature && !wall_v && !wall_n;
    if (!(all_present || all_absent))
        return fail(RMPCD_ERR_STOP, "wall parameters must be all present or all absent in wall_mpcd_step");
    if (!keep_cell_v && !thermostat)
        return fail(RMPCD_ERR_STOP, "requiring .not. keep_cell_v and .not. thermostat in wall_mpcd_step");
    SrdParams q = srd_params(p, c, r, has_alpha, alpha, thermostat, bulk_temperature, 1);
    double wt0 = all_present ? wall_temperature[0] : 0, wt1 = all_present ? wall_temperature[1] : 0;
    int wn0 = all_present ? wall_n[0] : 0, wn1 = all_present ? wall_n[1] : 0;
    cudaStream_t s = stream();
    int g = grid_full(c->S, 128);
    PhaseTimer t("step");
    DISPATCH_R(p,
               ({ PView<float> v = cur<float>(p);
                  k_wall_mpcd<float><<<g, 128, 0, s>>>(c->count, c->start, c->S, c->M[0], c->M[1], c->M[2], c->L[2],
                                                       v.vel.x, v.vel.y, v.vel.z, q, all_present, wt0, wt1, wn0, wn1, keep_cell_v ? 1 : 0); }),
               ({ PView<double> v = cur<double>(p);
                  k_wall_mpcd<double><<<g, 128, 0, s>>>(c->count, c->start, c->S, c->M[0], c->M[1], c->M[2], c->L[2],
                                                        v.vel.x, v.vel.y, v.vel.z, q, all_present, wt0, wt1, wn0, wn1, keep_cell_v ? 1 : 0); }));
    RMPCD_CHECK_LAUNCH();
    r->step++;
    return RMPCD_OK;
}

int rmpcd_compute_temperature(rmpcd_particles *p, rmpcd_cells *c, double *te)
{
    RMPCD_ARG(p && c && te, "null argument");
    PhaseTimer t("compute_temperature");
    cudaStream_t s = stream();
    double *part = c->d_red;
    DISPATCH_R(p,
               ({ PView<float> v = cur<float>(p);
                  k_temperature<float><<<kRedBlocks, 256, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z, v.species, part); }),
               ({ PView<double> v = cur<double>(p);
                  k_temperature<double><<<kRedBlocks, 256, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z, v.species, part); }));
    k_temperature_final<<<1, 32, 0, s>>>(part, kRedBlocks, part + 2 * kRedBlocks);
    RMPCD_CHECK_LAUNCH();
    RMPCD_CUDA_TRY(cudaMemcpyAsync(te, part + 2 * kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
    return sync();
}

int rmpcd_rescale_cells(rmpcd_particles *p, rmpcd_cells *c, rmpcd_rng *, double T)
{
    RMPCD_ARG(p && c, "null argument");
    PhaseTimer t("step");
    cudaStream_t s = stream();
    int g = grid_full(c->S, 128);
    DISPATCH_R(p,
               ({ PView<float> v = cur<float>(p);
                  k_rescale<float><<<g, 128, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z, v.species, T); }),
               ({ PView<double> v = cur<double>(p);
                  k_rescale<double><<<g, 128, 0, s>>>(c->count, c->start, c->S, v.vel.x, v.vel.y, v.vel.z, v.species, T); }));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_mpcd_stream_periodic(rmpcd_particles *p, rmpcd_cells *c, double dt)
{
    RMPCD_ARG(p && c, "null argument");
    if (p->N == 0) return RMPCD_OK;
    PhaseTimer t("stream");
    cudaStream_t s = stream();
    int g = grid_for(p->N, 256);
    DISPATCH_R(p,
               (k_stream_periodic<float><<<g, 256, 0, s>>>(cur<float>(p), c->edges[0], c->edges[1], c->edges[2], (float)dt)),
               (k_stream_periodic<double><<<g, 256, 0, s>>>(cur<double>(p), c->edges[0], c->edges[1], c->edges[2], dt)));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_mpcd_stream_xforce_yzwall(rmpcd_particles *p, rmpcd_cells *c, double dt, double g)
{
    RMPCD_ARG(p && c, "null argument");
    if (p->N == 0) return RMPCD_OK;
    PhaseTimer t("stream");
    cudaStream_t s = stream();
    int gr = grid_for(p->N, 256);
    unsigned *err = dev_error_word();
    DISPATCH_R(p,
               (k_stream_yzwall<float><<<gr, 256, 0, s>>>(cur<float>(p), c->edges[0], c->edges[1], c->edges[2],
                                                          c->bc[0], c->bc[1], c->bc[2], dt, g, err)),
               (k_stream_yzwall<double><<<gr, 256, 0, s>>>(cur<double>(p), c->edges[0], c->edges[1], c->edges[2],
                                                           c->bc[0], c->bc[1], c->bc[2], dt, g, err)));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_mpcd_stream_nogravity_zwall(rmpcd_particles *p, rmpcd_cells *c, double dt)
{
    RMPCD_ARG(p && c, "null argument");
    if (p->N == 0) return RMPCD_OK;
    PhaseTimer t("stream");
    cudaStream_t s = stream();
    int gr = grid_for(p->N, 256);
    DISPATCH_R(p, (k_stream_zwall<float><<<gr, 256, 0, s>>>(cur<float>(p), c->edges[2], dt)),
               (k_stream_zwall<double><<<gr, 256, 0, s>>>(cur<double>(p), c->edges[2], dt)));
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_bulk_reaction(rmpcd_particles *p, rmpcd_cells *c, int from, int to, double rate, double tau,
                        rmpcd_rng *r)
{
    RMPCD_ARG(p && c && r, "null argument");
    k_bulk_reaction<<<grid_full(c->S, 128), 128, 0, stream()>>>(c->count, c->start, c->is_reac, c->S,
                                                               p->species[p->cur], from, to, rate, tau,
                                                               r->seed, r->step);
    RMPCD_CHECK_LAUNCH();
    r->step++;
    return RMPCD_OK;
}

int rmpcd_bulk_reaction_endothermic(rmpcd_particles *p, rmpcd_cells *c, int from, int to, double rate,
                                    double tau, rmpcd_rng *r, double delta_u)
{
    RMPCD_ARG(p && c && r, "null argument");
    int gr = grid_full(c->S, 128);
    cudaStream_t s = stream();
    DISPATCH_R(p,
               (k_bulk_reaction_endo<float><<<gr, 128, 0, s>>>(c->count, c->start, c->is_reac, c->S, cur<float>(p),
                                                               from, to, rate, tau, delta_u, r->seed, r->step)),
               (k_bulk_reaction_endo<double><<<gr, 128, 0, s>>>(c->count, c->start, c->is_reac, c->S,
                                                                cur<double>(p), from, to, rate, tau, delta_u,
                                                                r->seed, r->step)));
    RMPCD_CHECK_LAUNCH();
    r->step++;
    return RMPCD_OK;
}

}  // extern "C"
