// Colloid-side integrators of the rigid-body programs (programs/single_body.f90):
// multi-link RATTLE (rattle_body_pos / rattle_body_vel, src/md.f90:321-480),
// the harmonic elastic network (src/md.f90:516-544) and the quaternion
// rigid body rigid_body_t (src/md.f90:40-58, :547-700).
//
// These act on the few beads of one body.  The RATTLE sweep is Gauss-Seidel
// (every link sees the positions left by the previous one) and the network's
// forces accumulate link by link, so those run in one thread in the
// reference's order; the rigid body's per-bead updates run one bead per
// thread after a single thread has advanced the body.  FP64 only, like the
// colloids of every program.
//
// Quaternions are (s, x, y, z), the layout of the reference's q(4) (qnew(s=1)
// is the identity).  The fortran_quaternion module the reference uses is not
// part of its tree; its operations are the standard ones, written here as
//   qmul(a, b) = (a.s b.s - a.v.b.v, a.s b.v + b.s a.v + a.v x b.v)
//   qconj(q)   = (q.s, -q.v)
//   qrot(q, v) = vector part of qmul(qmul(q, (0, v)), qconj(q))
//   qnorm(q)   = sqrt(q.s^2 + q.x^2 + q.y^2 + q.z^2), qnormalize(q) = q / qnorm(q)
// with sums taken left to right.
#include <cmath>
#include <cstring>
#include <vector>

#include "rmpcd_common.cuh"
#include "state.cuh"
#include "stepops.cuh"
#include "timers.cuh"

struct rmpcd_rigid_body {
    int i_start = 0, i_stop = 0;  // 1-based bead range
    int nb = 0;
    double *dev = nullptr;        // RigidState on the device
    double *pos_body = nullptr;   // 3 * nb, bead positions in the body frame
};

namespace rmpcd {

// rigid_body_t's scalar state, as one device block of doubles
struct RigidState {
    double mass;
    double pos[3], vel[3], force[3];
    double q[4];
    double L[3], torque[3];
    double I_body[3], omega_body[3];
};
static_assert(sizeof(RigidState) == sizeof(rmpcd_rigid_body_state), "state layouts agree");

constexpr int kRattleMax = 1000;          // rattle_max, src/md.f90:338
constexpr int kQuatIterMax = 100000;      // cap of rigid_body_vv1's iterative_q loop (unbounded in the reference)

// ---------------------------------------------------------------------------
// quaternion algebra
// ---------------------------------------------------------------------------
__device__ inline void qmul(const double a[4], const double b[4], double r[4])
{
    r[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    r[1] = a[0] * b[1] + b[0] * a[1] + (a[2] * b[3] - a[3] * b[2]);
    r[2] = a[0] * b[2] + b[0] * a[2] + (a[3] * b[1] - a[1] * b[3]);
    r[3] = a[0] * b[3] + b[0] * a[3] + (a[1] * b[2] - a[2] * b[1]);
}

__device__ inline void qconj(const double q[4], double r[4])
{
    r[0] = q[0];
    r[1] = -q[1];
    r[2] = -q[2];
    r[3] = -q[3];
}

__device__ inline void qrot(const double q[4], const double v[3], double r[3])
{
    const double pv[4] = {0.0, v[0], v[1], v[2]};
    double t[4], c[4], u[4];
    qmul(q, pv, t);
    qconj(q, c);
    qmul(t, c, u);
    r[0] = u[1];
    r[1] = u[2];
    r[2] = u[3];
}

__device__ inline double qnorm(const double q[4])
{
    return sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
}

__device__ inline void qnormalize(double q[4])
{
    const double n = qnorm(q);
    for (int k = 0; k < 4; k++) q[k] = q[k] / n;
}

// cross, src/common.f90:404-412
__device__ inline void cross3(const double a[3], const double b[3], double r[3])
{
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

// NORM2 of a 3-vector as the scaled sum of squares of the reference BLAS
// dnrm2 (the algorithm gfortran's NORM2 follows)
__device__ inline double norm2_scaled(const double x[3])
{
    double scale = 0, ssq = 1;
    for (int k = 0; k < 3; k++) {
        if (x[k] != 0) {
            const double a = fabs(x[k]);
            if (scale < a) {
                const double r = scale / a;
                ssq = 1 + ssq * r * r;
                scale = a;
            } else {
                const double r = a / scale;
                ssq = ssq + r * r;
            }
        }
    }
    return scale * sqrt(ssq);
}

__device__ inline double inv_mass_of(const Masses &ms, int species, unsigned *err)
{
    if (species < 1 || species > ms.n) {
        atomicOr(err, DEV_ERR_RATTLE);
        return 1.0;
    }
    return 1 / ms.m[species - 1];
}

// ---------------------------------------------------------------------------
// rattle_body_pos / rattle_body_vel
// ---------------------------------------------------------------------------
// image of bead i relative to bead 1: floor((x_i - x_1)/edges + 0.5)
// (src/md.f90:345-355), applied to x and returned
__device__ inline void unwrap_to_first(double *x, double *y, double *z, int N, const E3 &L, int *im)
{
    const double s[3] = {x[0], y[0], z[0]};
    double *c[3] = {x, y, z};
    for (int i = 1; i < N; i++)
        for (int k = 0; k < 3; k++) {
            const int m = (int)floor(((c[k][i] - s[k]) / L.e[k]) + 0.5);
            im[3 * i + k] = m;
            c[k][i] = c[k][i] - m * L.e[k];
        }
}

__global__ void k_rattle_body_pos(PView<double> v, double *rx, double *ry, double *rz, const int *links,
                                  const double *dist, int n_link, Masses ms, double dt, E3 L, double precision,
                                  int *im, int *iters, unsigned *err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int N = v.N;
    unwrap_to_first(v.pos.x, v.pos.y, v.pos.z, N, L, im);
    unwrap_to_first(rx, ry, rz, N, L, im + 3 * N);  // pos_rattle stays unwrapped, as in the reference
    double *px[3] = {v.pos.x, v.pos.y, v.pos.z}, *vx[3] = {v.vel.x, v.vel.y, v.vel.z};
    const double *pr[3] = {rx, ry, rz};
    int it = 1;
    for (; it <= kRattleMax; it++) {
        for (int l = 0; l < n_link; l++) {
            const int i1 = links[2 * l] - 1, i2 = links[2 * l + 1] - 1;
            const double d = dist[l];
            double r[3], s[3];
            for (int k = 0; k < 3; k++) {
                r[k] = pr[k][i1] - pr[k][i2];
                s[k] = px[k][i1] - px[k][i2];
            }
            const double im1 = inv_mass_of(ms, v.species[i1], err), im2 = inv_mass_of(ms, v.species[i2], err);
            const double inv_mass = im1 + im2;
            const double rsq = dot3(r, r), ssq = dot3(s, s), rs = dot3(r, s);
            const double disc = rs * rs - rsq * (ssq - d * d);
            if (disc < 0) atomicOr(err, DEV_ERR_RATTLE);
            double g = rs - sqrt(disc);
            g = g / (dt * inv_mass * rsq);
            for (int k = 0; k < 3; k++) {
                px[k][i1] = px[k][i1] - g * dt * r[k] * im1;
                px[k][i2] = px[k][i2] + g * dt * r[k] * im2;
            }
            for (int k = 0; k < 3; k++) {
                vx[k][i1] = vx[k][i1] - g * r[k] * im1;
                vx[k][i2] = vx[k][i2] + g * r[k] * im2;
            }
        }
        double error = 0;
        for (int l = 0; l < n_link; l++) {
            const int i1 = links[2 * l] - 1, i2 = links[2 * l + 1] - 1;
            double r[3];
            for (int k = 0; k < 3; k++) r[k] = px[k][i1] - px[k][i2];
            const double g = fabs(sqrt(dot3(r, r)) - dist[l]);
            if (g > error) error = g;
        }
        if (error < precision) break;
    }
    *iters = it;
    for (int i = 1; i < N; i++)
        for (int k = 0; k < 3; k++) px[k][i] = px[k][i] + im[3 * i + k] * L.e[k];
}

__global__ void k_rattle_body_vel(PView<double> v, const int *links, const double *dist, int n_link, Masses ms,
                                  E3 L, double precision, int *im, int *iters, unsigned *err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int N = v.N;
    unwrap_to_first(v.pos.x, v.pos.y, v.pos.z, N, L, im);
    double *px[3] = {v.pos.x, v.pos.y, v.pos.z}, *vx[3] = {v.vel.x, v.vel.y, v.vel.z};
    int it = 1;
    for (; it <= kRattleMax; it++) {
        for (int l = 0; l < n_link; l++) {
            const int i1 = links[2 * l] - 1, i2 = links[2 * l + 1] - 1;
            const double d = dist[l];
            const double im1 = inv_mass_of(ms, v.species[i1], err), im2 = inv_mass_of(ms, v.species[i2], err);
            const double inv_mass = im1 + im2;
            double s[3], dv[3];
            for (int k = 0; k < 3; k++) {
                s[k] = px[k][i1] - px[k][i2];
                dv[k] = vx[k][i1] - vx[k][i2];
            }
            const double kk = dot3(dv, s) / (d * d * inv_mass);
            for (int k = 0; k < 3; k++) {
                vx[k][i1] = vx[k][i1] - kk * s[k] * im1;
                vx[k][i2] = vx[k][i2] + kk * s[k] * im2;
            }
        }
        double error = 0;
        for (int l = 0; l < n_link; l++) {
            const int i1 = links[2 * l] - 1, i2 = links[2 * l + 1] - 1;
            const double d = dist[l];
            const double im1 = inv_mass_of(ms, v.species[i1], err), im2 = inv_mass_of(ms, v.species[i2], err);
            const double inv_mass = im1 + im2;
            double s[3], dv[3];
            for (int k = 0; k < 3; k++) {
                s[k] = px[k][i1] - px[k][i2];
                dv[k] = vx[k][i1] - vx[k][i2];
            }
            const double kk = fabs(dot3(dv, s) / (d * d * inv_mass));
            if (kk > error) error = kk;
        }
        if (error < precision) break;
    }
    *iters = it;
    for (int i = 1; i < N; i++)
        for (int k = 0; k < 3; k++) px[k][i] = px[k][i] + im[3 * i + k] * L.e[k];
}

// elastic_network, src/md.f90:516-544
__global__ void k_elastic_network(PView<double> v, const int *links, const double *dist, int n_link, double kel,
                                  E3 L, double *e_out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double *px[3] = {v.pos.x, v.pos.y, v.pos.z}, *fx[3] = {v.force.x, v.force.y, v.force.z};
    double e = 0;
    for (int l = 0; l < n_link; l++) {
        const int i1 = links[2 * l] - 1, i2 = links[2 * l + 1] - 1;
        const double r0 = dist[l];
        double x[3];
        for (int k = 0; k < 3; k++) x[k] = min_image_d(px[k][i1] - px[k][i2], L.e[k]);
        const double r = norm2_scaled(x);
        e = e + kel * ((r - r0) * (r - r0)) / 2;
        for (int k = 0; k < 3; k++) {
            const double f = -(kel * (r - r0) * x[k] / r);
            fx[k][i1] = fx[k][i1] + f;
            fx[k][i2] = fx[k][i2] - f;
        }
    }
    *e_out = e;
}

// ---------------------------------------------------------------------------
// rigid_body_t
// ---------------------------------------------------------------------------
// rigid_body_init, src/md.f90:547-588 (pos_body is indexed from the body's
// first bead; the reference indexes it by the bead number, which is the same
// for the i_start = 1 every program uses)
__global__ void k_rigid_init(PView<double> v, Masses ms, int i0, int nb, E3 L, RigidState *st, double *pos_body,
                             unsigned *err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mass = 0, pos[3] = {0, 0, 0}, vel[3] = {0, 0, 0};
    const double *px[3] = {v.pos.x, v.pos.y, v.pos.z}, *vx[3] = {v.vel.x, v.vel.y, v.vel.z};
    const int *ix[3] = {v.ix, v.iy, v.iz};
    for (int b = 0; b < nb; b++) {
        const int i = i0 + b;
        const double m = bead_mass(ms, v.species, i, err);
        mass = mass + m;
        for (int k = 0; k < 3; k++) {
            pos[k] = pos[k] + m * (px[k][i] + ix[k][i] * L.e[k]);
            vel[k] = vel[k] + m * vx[k][i];
        }
    }
    for (int k = 0; k < 3; k++) {
        pos[k] = pos[k] / mass;
        vel[k] = vel[k] / mass;
    }
    double I[3] = {0, 0, 0};
    for (int b = 0; b < nb; b++) {
        const int i = i0 + b;
        const double m = bead_mass(ms, v.species, i, err);
        double p[3];
        for (int k = 0; k < 3; k++) {
            p[k] = px[k][i] + ix[k][i] * L.e[k] - pos[k];
            pos_body[3 * b + k] = p[k];
        }
        const double sq = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        for (int k = 0; k < 3; k++) I[k] = I[k] + m * (sq - p[k] * p[k]);
    }
    st->mass = mass;
    for (int k = 0; k < 3; k++) {
        st->pos[k] = pos[k];
        st->vel[k] = vel[k];
        st->force[k] = 0;
        st->torque[k] = 0;
        st->L[k] = 0;
        st->I_body[k] = I[k];
        st->omega_body[k] = 0;
    }
    st->q[0] = 1;
    st->q[1] = st->q[2] = st->q[3] = 0;
}

// rigid_body_compute_force_torque, src/md.f90:591-607
__global__ void k_rigid_force_torque(PView<double> v, int i0, int nb, RigidState *st, const double *pos_body)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    for (int b = 0; b < nb; b++) {
        const int i = i0 + b;
        const double f[3] = {v.force.x[i], v.force.y[i], v.force.z[i]};
        double p[3], c[3];
        for (int k = 0; k < 3; k++) F[k] = F[k] + f[k];
        qrot(st->q, pos_body + 3 * b, p);
        cross3(p, f, c);
        for (int k = 0; k < 3; k++) T[k] = T[k] + c[k];
    }
    for (int k = 0; k < 3; k++) {
        st->force[k] = F[k];
        st->torque[k] = T[k];
    }
}

// rigid_body_vv1, src/md.f90:613-673 (Rozmanov & Kusalik's rotational
// velocity Verlet): thread 0 advances the body, then every thread places
// its beads
__global__ void k_rigid_vv1(PView<double> v, int i0, int nb, RigidState *st, const double *pos_body, double dt,
                            double treshold, E3 L, unsigned *err)
{
    __shared__ double s_pos[3], s_q[4];
    if (threadIdx.x == 0) {
        double I_inv[3], Lv[3], q[4], qc[4], Lb[3], tb[3], wb[3], c[3], Lbd[3], qd[4], qo[4];
        for (int k = 0; k < 3; k++) I_inv[k] = 1 / st->I_body[k];
        for (int k = 0; k < 3; k++) Lv[k] = st->L[k];
        for (int k = 0; k < 4; k++) q[k] = st->q[k];
        qconj(q, qc);
        qrot(qc, Lv, Lb);
        qrot(qc, st->torque, tb);
        for (int k = 0; k < 3; k++) wb[k] = Lb[k] * I_inv[k];
        cross3(wb, Lb, c);
        for (int k = 0; k < 3; k++) Lbd[k] = tb[k] - c[k];
        // timestep 1/2
        for (int k = 0; k < 3; k++) Lb[k] = Lb[k] + dt * Lbd[k] / 2;
        for (int k = 0; k < 3; k++) wb[k] = Lb[k] * I_inv[k];
        {
            const double w4[4] = {0.0, wb[0], wb[1], wb[2]};
            qmul(q, w4, qd);
            for (int k = 0; k < 4; k++) qd[k] = qd[k] / 2;
        }
        for (int k = 0; k < 4; k++) q[k] = q[k] + qd[k] * dt / 2;
        qnormalize(q);
        for (int k = 0; k < 3; k++) Lv[k] = st->L[k] + st->torque[k] * dt / 2;
        // iterative procedure
        for (int k = 0; k < 4; k++) qo[k] = q[k];
        int it = 0;
        while (true) {
            qconj(q, qc);
            qrot(qc, Lv, Lb);
            for (int k = 0; k < 3; k++) wb[k] = I_inv[k] * Lb[k];
            const double w4[4] = {0.0, wb[0], wb[1], wb[2]};
            qmul(q, w4, qd);
            for (int k = 0; k < 4; k++) qd[k] = qd[k] / 2;
            for (int k = 0; k < 4; k++) q[k] = st->q[k] + qd[k] * dt / 2;
            qnormalize(q);
            double dq[4];
            for (int k = 0; k < 4; k++) dq[k] = q[k] - qo[k];
            if (qnorm(dq) < treshold) break;
            for (int k = 0; k < 4; k++) qo[k] = q[k];
            if (++it >= kQuatIterMax) {
                atomicOr(err, DEV_ERR_QUAT_LOOP);
                break;
            }
        }
        for (int k = 0; k < 4; k++) st->q[k] = st->q[k] + dt * qd[k];
        qnormalize(st->q);
        for (int k = 0; k < 3; k++)
            st->pos[k] = st->pos[k] + st->vel[k] * dt + st->force[k] * (dt * dt) / (2 * st->mass);
        for (int k = 0; k < 3; k++) s_pos[k] = st->pos[k];
        for (int k = 0; k < 4; k++) s_q[k] = st->q[k];
    }
    __syncthreads();
    double *px[3] = {v.pos.x, v.pos.y, v.pos.z};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int i = i0 + b;
        double r[3];
        qrot(s_q, pos_body + 3 * b, r);
        for (int k = 0; k < 3; k++) {
            const double old = px[k][i];
            const double x = s_pos[k] + r[k];
            const double delta = x - old + L.e[k] / 2;
            px[k][i] = x - floor(delta / L.e[k]) * L.e[k];
        }
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; k++) st->L[k] = st->L[k] + st->torque[k] * dt / 2;
        for (int k = 0; k < 3; k++) st->vel[k] = st->vel[k] + st->force[k] * dt / (2 * st->mass);
    }
}

// rigid_body_vv2, src/md.f90:679-700
__global__ void k_rigid_vv2(PView<double> v, int i0, int nb, RigidState *st, const double *pos_body, double dt)
{
    __shared__ double s_q[4], s_w[3], s_v[3];
    if (threadIdx.x == 0) {
        double qc[4], Lb[3], w[3];
        for (int k = 0; k < 3; k++) st->L[k] = st->L[k] + st->torque[k] * dt / 2;
        qconj(st->q, qc);
        qrot(qc, st->L, Lb);
        for (int k = 0; k < 3; k++) st->omega_body[k] = Lb[k] / st->I_body[k];
        qrot(st->q, st->omega_body, w);
        for (int k = 0; k < 3; k++) st->vel[k] = st->vel[k] + st->force[k] * dt / (2 * st->mass);
        for (int k = 0; k < 4; k++) s_q[k] = st->q[k];
        for (int k = 0; k < 3; k++) {
            s_w[k] = w[k];
            s_v[k] = st->vel[k];
        }
    }
    __syncthreads();
    double *vx[3] = {v.vel.x, v.vel.y, v.vel.z};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int i = i0 + b;
        double p[3], c[3];
        qrot(s_q, pos_body + 3 * b, p);
        cross3(s_w, p, c);
        for (int k = 0; k < 3; k++) vx[k][i] = s_v[k] + c[k];
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static Masses masses_of_body(const rmpcd_particles *p)
{
    Masses ms;
    for (int k = 0; k < RMPCD_MAX_SPECIES; k++) ms.m[k] = p->mass[k];
    ms.n = p->n_species;
    return ms;
}

// links and distances staged on the device (grow-only), plus the image and
// iteration scratch of the RATTLE kernels
struct BodyScratch {
    int *links = nullptr;
    double *dist = nullptr;
    int *im = nullptr;
    int *iters = nullptr;
    double *energy = nullptr;
    int link_cap = 0, im_cap = 0;
};
static BodyScratch g_body;

static int stage_links(const int *links, const double *dist, int n_link, int N)
{
    cudaStream_t s = stream();
    if (!g_body.iters) {
        RMPCD_CUDA_TRY(cudaMalloc(&g_body.iters, sizeof(int)));
        RMPCD_CUDA_TRY(cudaMalloc(&g_body.energy, sizeof(double)));
    }
    if (g_body.link_cap < n_link) {
        cudaStreamSynchronize(s);
        cudaFree(g_body.links);
        cudaFree(g_body.dist);
        g_body.links = nullptr;
        g_body.dist = nullptr;
        g_body.link_cap = 0;
        RMPCD_CUDA_TRY(cudaMalloc(&g_body.links, 2 * (size_t)n_link * sizeof(int)));
        RMPCD_CUDA_TRY(cudaMalloc(&g_body.dist, (size_t)n_link * sizeof(double)));
        g_body.link_cap = n_link;
    }
    if (g_body.im_cap < N) {
        cudaStreamSynchronize(s);
        cudaFree(g_body.im);
        g_body.im = nullptr;
        g_body.im_cap = 0;
        RMPCD_CUDA_TRY(cudaMalloc(&g_body.im, 6 * (size_t)N * sizeof(int)));
        g_body.im_cap = N;
    }
    if (n_link > 0) {
        RMPCD_CUDA_TRY(cudaMemcpyAsync(g_body.links, links, 2 * (size_t)n_link * sizeof(int), cudaMemcpyHostToDevice, s));
        RMPCD_CUDA_TRY(cudaMemcpyAsync(g_body.dist, dist, (size_t)n_link * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    return RMPCD_OK;
}

static int check_links(const rmpcd_particles *p, const int *links, const double *dist, int n_link)
{
    RMPCD_ARG(n_link >= 0 && (n_link == 0 || (links && dist)), "links / distances missing");
    for (int l = 0; l < 2 * n_link; l++)
        if (links[l] < 1 || links[l] > p->N) return fail(RMPCD_ERR_INVALID, "link %d names particle %d of %d", l / 2 + 1, links[l], p->N);
    return RMPCD_OK;
}

static int finish_rattle(int *iterations, const char *name)
{
    int it = 0;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(&it, g_body.iters, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    int rc = sync();
    if (rc) return rc;
    if (iterations) *iterations = it;
    unsigned bits = 0;
    rc = check_dev_error(&bits);
    if (rc) return fail(RMPCD_ERR_DEVICE, "%s: negative discriminant or bad species (bits 0x%x)", name, bits);
    return RMPCD_OK;
}

}  // namespace rmpcd

using namespace rmpcd;

extern "C" {

int rmpcd_rattle_body_pos(rmpcd_particles *p, const int *links, const double *distances, int n_link, double dt,
                          const double edges[3], double precision, int *iterations)
{
    RMPCD_ARG(p && edges, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64 && p->N >= 1, "rattle_body_pos: needs an FP64 system");
    RMPCD_ARG(p->pos_rattle[0] != nullptr, "rattle_body_pos: pos_rattle was never set");
    int rc = check_links(p, links, distances, n_link);
    if (!rc) rc = stage_links(links, distances, n_link, p->N);
    if (rc) return rc;
    PhaseTimer t("rattle_pos");
    E3 L = {{edges[0], edges[1], edges[2]}};
    k_rattle_body_pos<<<1, 32, 0, stream()>>>(cur<double>(p), (double *)p->pos_rattle[0], (double *)p->pos_rattle[1],
                                             (double *)p->pos_rattle[2], g_body.links, g_body.dist, n_link,
                                             masses_of_body(p), dt, L, precision, g_body.im, g_body.iters,
                                             dev_error_word());
    RMPCD_CHECK_LAUNCH();
    return finish_rattle(iterations, "rattle_body_pos");
}

int rmpcd_rattle_body_vel(rmpcd_particles *p, const int *links, const double *distances, int n_link, double dt,
                          const double edges[3], double precision, int *iterations)
{
    (void)dt;
    RMPCD_ARG(p && edges, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64 && p->N >= 1, "rattle_body_vel: needs an FP64 system");
    int rc = check_links(p, links, distances, n_link);
    if (!rc) rc = stage_links(links, distances, n_link, p->N);
    if (rc) return rc;
    PhaseTimer t("rattle_vel");
    E3 L = {{edges[0], edges[1], edges[2]}};
    k_rattle_body_vel<<<1, 32, 0, stream()>>>(cur<double>(p), g_body.links, g_body.dist, n_link, masses_of_body(p), L,
                                             precision, g_body.im, g_body.iters, dev_error_word());
    RMPCD_CHECK_LAUNCH();
    return finish_rattle(iterations, "rattle_body_vel");
}

int rmpcd_elastic_network(rmpcd_particles *p, const int *links, const double *distances, int n_link, double k,
                          const double edges[3], double *energy)
{
    RMPCD_ARG(p && edges, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64, "elastic_network: needs an FP64 system");
    int rc = check_links(p, links, distances, n_link);
    if (!rc) rc = stage_links(links, distances, n_link, p->N);
    if (rc) return rc;
    E3 L = {{edges[0], edges[1], edges[2]}};
    p->force_zero = false;
    k_elastic_network<<<1, 32, 0, stream()>>>(cur<double>(p), g_body.links, g_body.dist, n_link, k, L, g_body.energy);
    RMPCD_CHECK_LAUNCH();
    double e = 0;
    RMPCD_CUDA_TRY(cudaMemcpyAsync(&e, g_body.energy, sizeof(double), cudaMemcpyDeviceToHost, stream()));
    rc = sync();
    if (!rc && energy) *energy = e;
    return rc;
}

int rmpcd_rigid_body_init(rmpcd_rigid_body **out, rmpcd_particles *p, int i_start, int i_stop, const double edges[3])
{
    RMPCD_ARG(out && p && edges, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64, "rigid_body_init: needs an FP64 system");
    RMPCD_ARG(i_start >= 1 && i_stop >= i_start && i_stop <= p->N, "rigid_body_init: 1 <= i_start <= i_stop <= N");
    *out = nullptr;
    rmpcd_rigid_body *rb = new rmpcd_rigid_body;
    rb->i_start = i_start;
    rb->i_stop = i_stop;
    rb->nb = i_stop - i_start + 1;
    if (cudaMalloc(&rb->dev, sizeof(RigidState)) != cudaSuccess ||
        cudaMalloc(&rb->pos_body, 3 * (size_t)rb->nb * sizeof(double)) != cudaSuccess) {
        cudaFree(rb->dev);
        delete rb;
        return fail(RMPCD_ERR_CUDA, "rigid_body_init: allocation failed");
    }
    E3 L = {{edges[0], edges[1], edges[2]}};
    k_rigid_init<<<1, 32, 0, stream()>>>(cur<double>(p), masses_of_body(p), i_start - 1, rb->nb, L,
                                        (RigidState *)rb->dev, rb->pos_body, dev_error_word());
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        rmpcd_rigid_body_destroy(rb);
        return fail(RMPCD_ERR_CUDA, "rigid_body_init: %s", cudaGetErrorString(e));
    }
    int rc = check_dev_error(nullptr);
    if (rc) {
        rmpcd_rigid_body_destroy(rb);
        return rc;
    }
    *out = rb;
    return RMPCD_OK;
}

int rmpcd_rigid_body_destroy(rmpcd_rigid_body *rb)
{
    if (!rb) return RMPCD_OK;
    cudaStreamSynchronize(stream());
    cudaFree(rb->dev);
    cudaFree(rb->pos_body);
    delete rb;
    return RMPCD_OK;
}

static int body_args(const rmpcd_rigid_body *rb, const rmpcd_particles *p)
{
    RMPCD_ARG(rb && p, "null argument");
    RMPCD_ARG(p->precision == RMPCD_FP64 && rb->i_stop <= p->N, "rigid body: its beads are not in this system");
    return RMPCD_OK;
}

int rmpcd_rigid_body_compute_force_torque(rmpcd_rigid_body *rb, rmpcd_particles *p)
{
    int rc = body_args(rb, p);
    if (rc) return rc;
    k_rigid_force_torque<<<1, 32, 0, stream()>>>(cur<double>(p), rb->i_start - 1, rb->nb, (RigidState *)rb->dev,
                                                rb->pos_body);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_rigid_body_vv1(rmpcd_rigid_body *rb, rmpcd_particles *p, double dt, double treshold, const double edges[3])
{
    int rc = body_args(rb, p);
    if (rc) return rc;
    RMPCD_ARG(edges, "null argument");
    E3 L = {{edges[0], edges[1], edges[2]}};
    k_rigid_vv1<<<1, 256, 0, stream()>>>(cur<double>(p), rb->i_start - 1, rb->nb, (RigidState *)rb->dev, rb->pos_body,
                                        dt, treshold, L, dev_error_word());
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_rigid_body_vv2(rmpcd_rigid_body *rb, rmpcd_particles *p, double dt)
{
    int rc = body_args(rb, p);
    if (rc) return rc;
    k_rigid_vv2<<<1, 256, 0, stream()>>>(cur<double>(p), rb->i_start - 1, rb->nb, (RigidState *)rb->dev, rb->pos_body,
                                        dt);
    RMPCD_CHECK_LAUNCH();
    return RMPCD_OK;
}

int rmpcd_rigid_body_get(const rmpcd_rigid_body *rb, rmpcd_rigid_body_state *st, double *pos_body)
{
    RMPCD_ARG(rb && st, "null argument");
    RMPCD_CUDA_TRY(cudaMemcpyAsync(st, rb->dev, sizeof(RigidState), cudaMemcpyDeviceToHost, stream()));
    if (pos_body)
        RMPCD_CUDA_TRY(cudaMemcpyAsync(pos_body, rb->pos_body, 3 * (size_t)rb->nb * sizeof(double),
                                       cudaMemcpyDeviceToHost, stream()));
    return check_dev_error(nullptr);
}

int rmpcd_rigid_body_set(rmpcd_rigid_body *rb, const rmpcd_rigid_body_state *st)
{
    RMPCD_ARG(rb && st, "null argument");
    RMPCD_CUDA_TRY(cudaMemcpyAsync(rb->dev, st, sizeof(RigidState), cudaMemcpyHostToDevice, stream()));
    return sync();
}

}  // extern "C"
