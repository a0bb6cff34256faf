// Per-particle and per-dimer bodies of the MD, MPCD and reaction steps,
// shared by the single-system kernels of the C ABI and the batched replica
// engine so that both perform exactly the same arithmetic.
#pragma once

#include "cellops.cuh"
#include "rmpcd_common.cuh"
#include "rng.cuh"
#include "state.cuh"

namespace rmpcd {

// md_pos, src/md.f90:61-77
template <typename R>
__device__ inline void md_pos_one(const PView<R> &v, long long i, R dt, R dt_sq)
{
    v.pos.x[i] = v.pos.x[i] + dt * v.vel.x[i] + dt_sq * v.force.x[i];
    v.pos.y[i] = v.pos.y[i] + dt * v.vel.y[i] + dt_sq * v.force.y[i];
    v.pos.z[i] = v.pos.z[i] + dt * v.vel.z[i] + dt_sq * v.force.z[i];
}

// md_vel, src/md.f90:219-237
template <typename R>
__device__ inline void md_vel_one(const PView<R> &v, long long i, R dt)
{
    int f = v.flags[i];
    if (!((f >> WALL_BIT) & 1)) {
        v.vel.x[i] = v.vel.x[i] + dt * (v.force.x[i] + v.force_old.x[i]) / 2;
        v.vel.y[i] = v.vel.y[i] + dt * (v.force.y[i] + v.force_old.y[i]) / 2;
        v.vel.z[i] = v.vel.z[i] + dt * (v.force.z[i] + v.force_old.z[i]) / 2;
    } else {
        v.flags[i] = f & ~(1 << WALL_BIT);
    }
}

// apply_pbc, src/md.f90:202-217
template <typename R>
__device__ inline void apply_pbc_one(const PView<R> &v, long long i, double e0, double e1, double e2)
{
    R x = v.pos.x[i], y = v.pos.y[i], z = v.pos.z[i];
    int jx = floor_div_edge((double)x, e0), jy = floor_div_edge((double)y, e1), jz = floor_div_edge((double)z, e2);
    if (jx) {
        v.ix[i] += jx;
        v.pos.x[i] = x - (R)(jx * e0);
    }
    if (jy) {
        v.iy[i] += jy;
        v.pos.y[i] = y - (R)(jy * e1);
    }
    if (jz) {
        v.iz[i] += jz;
        v.pos.z[i] = z - (R)(jz * e2);
    }
}

// PAST_MD <- MD, MD cleared (src/neighbor_list.f90:180-188)
__device__ inline void flag_roll_one(int *flags, long long i)
{
    int f = flags[i];
    if ((f >> MD_BIT) & 1) f |= (1 << PAST_MD_BIT);
    else f &= ~(1 << PAST_MD_BIT);
    flags[i] = f & ~(1 << MD_BIT);
}

// |pos - pos_old|^2 of particle i, or 0 when species(i) < 0
// (src/particle_system.f90:357-378)
template <typename R>
__device__ inline double disp_sq_one(const Vec3<R> &pos, const Vec3<R> &old, const int *species, long long i)
{
    if (species[i] < 0) return 0;
    double d0 = (double)pos.x[i] - (double)old.x[i];
    double d1 = (double)pos.y[i] - (double)old.y[i];
    double d2 = (double)pos.z[i] - (double)old.z[i];
    return d0 * d0 + d1 * d1 + d2 * d2;
}

// colloid velocity-Verlet halves, programs/single_dimer_pbc.f90:312-315, :356-359
__device__ inline void colloid_vv_pos_one(const PView<double> &v, int i, double m, double dt)
{
    double m2 = 2 * m;
    v.pos.x[i] = v.pos.x[i] + dt * v.vel.x[i] + dt * dt * v.force.x[i] / m2;
    v.pos.y[i] = v.pos.y[i] + dt * v.vel.y[i] + dt * dt * v.force.y[i] / m2;
    v.pos.z[i] = v.pos.z[i] + dt * v.vel.z[i] + dt * dt * v.force.z[i] / m2;
}

__device__ inline void colloid_vv_vel_one(const PView<double> &v, int i, double m, double dt)
{
    double m2 = 2 * m;
    v.vel.x[i] = v.vel.x[i] + dt * (v.force.x[i] + v.force_old.x[i]) / m2;
    v.vel.y[i] = v.vel.y[i] + dt * (v.force.y[i] + v.force_old.y[i]) / m2;
    v.vel.z[i] = v.vel.z[i] + dt * (v.force.z[i] + v.force_old.z[i]) / m2;
}

struct E3 {
    double e[3];
};

struct Masses {
    double m[RMPCD_MAX_SPECIES];
    int n;
};

// mass(species(k)) of bead k; out-of-range species flag an error
__device__ inline double bead_mass(const Masses &ms, const int *species, int k, unsigned *err)
{
    int s = species[k];
    if (s < 1 || s > ms.n) {
        atomicOr(err, DEV_ERR_RATTLE);
        return 1.0;
    }
    return ms.m[s - 1];
}

__device__ inline double dot3(const double a[3], const double b[3])
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// rattle_dimer_pos, src/md.f90:265-296: beads 0 and 1 of v; r = pos_rattle
__device__ inline void rattle_pos_dimer(const PView<double> &v, const double *rx, const double *ry,
                                        const double *rz, const Masses &ms, double d, double dt, const E3 &L,
                                        unsigned *err)
{
    double m1 = bead_mass(ms, v.species, 0, err), m2 = bead_mass(ms, v.species, 1, err);
    double r[3], s[3];
    r[0] = min_image_d(rx[0] - rx[1], L.e[0]);
    r[1] = min_image_d(ry[0] - ry[1], L.e[1]);
    r[2] = min_image_d(rz[0] - rz[1], L.e[2]);
    s[0] = min_image_d(v.pos.x[0] - v.pos.x[1], L.e[0]);
    s[1] = min_image_d(v.pos.y[0] - v.pos.y[1], L.e[1]);
    s[2] = min_image_d(v.pos.z[0] - v.pos.z[1], L.e[2]);
    double inv_mass = 1 / m1 + 1 / m2;
    double rsq = dot3(r, r), ssq = dot3(s, s), rs = dot3(r, s);
    double disc = rs * rs - rsq * (ssq - d * d);
    if (disc < 0) atomicOr(err, DEV_ERR_RATTLE);
    double g = rs - sqrt(disc);
    g = g / (dt * inv_mass * rsq);
    double *px[3] = {v.pos.x, v.pos.y, v.pos.z};
    double *vx[3] = {v.vel.x, v.vel.y, v.vel.z};
    for (int k = 0; k < 3; k++) {
        px[k][0] = px[k][0] - g * dt * r[k] / m1;
        px[k][1] = px[k][1] + g * dt * r[k] / m2;
    }
    for (int k = 0; k < 3; k++) {
        vx[k][0] = vx[k][0] - g * r[k] / m1;
        vx[k][1] = vx[k][1] + g * r[k] / m2;
    }
}

// rattle_dimer_vel, src/md.f90:298-319
__device__ inline void rattle_vel_dimer(const PView<double> &v, const Masses &ms, double d, const E3 &L,
                                        unsigned *err)
{
    double m1 = bead_mass(ms, v.species, 0, err), m2 = bead_mass(ms, v.species, 1, err);
    double s[3], dv[3];
    double inv_mass = 1 / m1 + 1 / m2;
    s[0] = min_image_d(v.pos.x[0] - v.pos.x[1], L.e[0]);
    s[1] = min_image_d(v.pos.y[0] - v.pos.y[1], L.e[1]);
    s[2] = min_image_d(v.pos.z[0] - v.pos.z[1], L.e[2]);
    double *vx[3] = {v.vel.x, v.vel.y, v.vel.z};
    for (int k = 0; k < 3; k++) dv[k] = vx[k][0] - vx[k][1];
    double kk = dot3(dv, s) / (d * d * inv_mass);
    for (int k = 0; k < 3; k++) {
        vx[k][0] = vx[k][0] - kk * s[k] / m1;
        vx[k][1] = vx[k][1] + kk * s[k] / m2;
    }
}

// positions of the two beads of a dimer
struct C2 {
    double c1[3], c2[3];
};

// change_species of particle m, programs/single_dimer_pbc.f90:511-542; the
// acceptance uniform is Philox(seed, step, m, REACT) with m the particle's
// index in its own system
template <typename R>
__device__ inline void change_species_one(const PView<R> &v, long long m, long long m_rng, const double a[3],
                                          const double b[3], double L0, double L1, double L2, double cut_c,
                                          double cut_n, double prob, uint64_t seed, uint64_t step)
{
    int f = v.flags[m];
    if (!((f >> REAC_BIT) & 1)) return;
    double px = (double)v.pos.x[m], py = (double)v.pos.y[m], pz = (double)v.pos.z[m];
    double d0 = min_image_d(a[0] - px, L0), d1 = min_image_d(a[1] - py, L1), d2 = min_image_d(a[2] - pz, L2);
    double dC = d0 * d0 + d1 * d1 + d2 * d2;
    d0 = min_image_d(b[0] - px, L0);
    d1 = min_image_d(b[1] - py, L1);
    d2 = min_image_d(b[2] - pz, L2);
    double dN = d0 * d0 + d1 * d1 + d2 * d2;
    if ((dC > cut_c) && (dN > cut_n)) {
        double u0, u1;
        rng::uniform2(seed, step, (uint32_t)m_rng, rng::REACT, 0, u0, u1);
        if (u0 <= prob) v.species[m] = 2;
        v.flags[m] = f & ~(1 << REAC_BIT);
    }
}

// refuel of particle m, programs/single_dimer_pbc.f90:544-565
template <typename R>
__device__ inline void refuel_one(const PView<R> &v, long long m, const double a[3], const double b[3], double L0,
                                  double L1, double L2, double far)
{
    if (v.species[m] != 2) return;
    double px = (double)v.pos.x[m], py = (double)v.pos.y[m], pz = (double)v.pos.z[m];
    double d0 = min_image_d(a[0] - px, L0), d1 = min_image_d(a[1] - py, L1), d2 = min_image_d(a[2] - pz, L2);
    double dC = d0 * d0 + d1 * d1 + d2 * d2;
    d0 = min_image_d(b[0] - px, L0);
    d1 = min_image_d(b[1] - py, L1);
    d2 = min_image_d(b[2] - pz, L2);
    double dN = d0 * d0 + d1 * d1 + d2 * d2;
    if ((dC > far) && (dN > far)) v.species[m] = 1;
}

// flag_particles_nl test of one list entry, programs/single_dimer_pbc.f90:493-509
template <typename R>
__device__ inline void flag_nl_one(int r, const double x[3], const R *sx, const R *sy, const R *sz,
                                   const int *species, int *flags, double L0, double L1, double L2, double cut_sq)
{
    if (species[r] == 1) {
        double d0 = min_image_d(x[0] - (double)sx[r], L0);
        double d1 = min_image_d(x[1] - (double)sy[r], L1);
        double d2 = min_image_d(x[2] - (double)sz[r], L2);
        double d = d0 * d0 + d1 * d1 + d2 * d2;
        if (d < cut_sq) atomicOr(flags + r, 1 << REAC_BIT);
    }
}

struct SrdParams {
    double sin_a, cos_a, t_factor;
    int thermostat, hydro;
    uint64_t seed, step;
    const double *axes;   // injected per-slot axes or null
    const double *gauss;  // injected per-particle normals or null
};

__device__ inline double at_normal(const SrdParams &q, long long j, int k)
{
    return q.gauss ? q.gauss[3 * (size_t)j + k] : rng::normal(q.seed, q.step, (uint32_t)j, (uint32_t)k);
}

// simple_mpcd_step of one slot, src/mpcd.f90:71-183.  Particles a..a+n-1;
// s_rng keys the slot's axis, and particle i's normals are keyed by
// i - i_rng0 (indices of the particle's own system).
template <typename R>
__device__ inline void srd_slot(int n, long long a, long long s_rng, long long i_rng0, R *vx, R *vy, R *vz,
                                const int *species, const SrdParams &q)
{
    if (n <= 1) return;
    int n_eff = 0;
    CellSum<R> sx, sy, sz;
    for (long long i = a; i < a + n; i++) {
        if (species[i] > 0) {
            sx.add(vx[i]);
            sy.add(vy[i]);
            sz.add(vz[i]);
            n_eff++;
        }
    }
    if (n_eff <= 1) return;
    R lv[3] = {sx.value() / n_eff, sy.value() / n_eff, sz.value() / n_eff};
    if (q.thermostat) {
        CellSum<R> wx, wy, wz;
        for (long long i = a; i < a + n; i++) {
            if (species[i] <= 0) continue;
            R nx = (R)(at_normal(q, i - i_rng0, 0) * q.t_factor);
            R ny = (R)(at_normal(q, i - i_rng0, 1) * q.t_factor);
            R nz = (R)(at_normal(q, i - i_rng0, 2) * q.t_factor);
            vx[i] = nx;
            vy[i] = ny;
            vz[i] = nz;
            wx.add(nx);
            wy.add(ny);
            wz.add(nz);
        }
        R dv[3] = {lv[0] - wx.value() / n_eff, lv[1] - wy.value() / n_eff, lv[2] - wz.value() / n_eff};
        if (q.hydro) {
            for (long long i = a; i < a + n; i++) {
                if (species[i] <= 0) continue;
                vx[i] = vx[i] + dv[0];
                vy[i] = vy[i] + dv[1];
                vz[i] = vz[i] + dv[2];
            }
        }
    } else {
        double n0, n1, n2;
        if (q.axes) {
            n0 = q.axes[3 * (size_t)s_rng];
            n1 = q.axes[3 * (size_t)s_rng + 1];
            n2 = q.axes[3 * (size_t)s_rng + 2];
        } else {
            rng::sphere(q.seed, q.step, (uint32_t)s_rng, n0, n1, n2);
        }
        Rot o = srd_matrix(n0, n1, n2, q.sin_a, q.cos_a);
        for (long long i = a; i < a + n; i++) {
            R x = vx[i], y = vy[i], z = vz[i];
            srd_rotate(x, y, z, lv, o);
            vx[i] = x;
            vy[i] = y;
            vz[i] = z;
        }
    }
}

}  // namespace rmpcd
