/* Oracle (test infrastructure): rigid-body colloid routines of src/md.f90 in
 * FP64, in the reference's (3,N) layout with 1-based link lists.
 *
 *   orc_rattle_body_pos        src/md.f90:321-408
 *   orc_rattle_body_vel        src/md.f90:410-480
 *   orc_elastic_network        src/md.f90:516-544
 *   orc_rigid_body_*           src/md.f90:40-58 (type), :547-700
 *
 * The quaternion operations come from the fortran_quaternion submodule,
 * which the reference tree does not contain; they are restated from the
 * standard algebra (q = (s, x, y, z)):
 *   product  (a.s b.s - a.v.b.v, a.s b.v + b.s a.v + a.v x b.v)
 *   rotation vector part of q (0, v) q*, norm sqrt of the sum of squares.
 * NORM2 (elastic_network) is the scaled sum of squares of the reference
 * BLAS dnrm2, the method gfortran's NORM2 uses.  Parity with the Fortran
 * build is unpinned here: neither gfortran nor the quaternion module is
 * available. */
#include <math.h>
#include <string.h>

#include "rmpcd_oracle.h"

static void qprod(const double a[4], const double b[4], double r[4])
{
    double s = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    double x = a[0] * b[1] + b[0] * a[1] + (a[2] * b[3] - a[3] * b[2]);
    double y = a[0] * b[2] + b[0] * a[2] + (a[3] * b[1] - a[1] * b[3]);
    double z = a[0] * b[3] + b[0] * a[3] + (a[1] * b[2] - a[2] * b[1]);
    r[0] = s;
    r[1] = x;
    r[2] = y;
    r[3] = z;
}

static void qstar(const double q[4], double r[4])
{
    r[0] = q[0];
    r[1] = -q[1];
    r[2] = -q[2];
    r[3] = -q[3];
}

static void qrotate(const double q[4], const double v[3], double r[3])
{
    double p[4] = {0.0, v[0], v[1], v[2]}, t[4], c[4], u[4];
    qprod(q, p, t);
    qstar(q, c);
    qprod(t, c, u);
    r[0] = u[1];
    r[1] = u[2];
    r[2] = u[3];
}

static double qlen(const double q[4]) { return sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]); }

static void qunit(double q[4])
{
    double n = qlen(q);
    for (int k = 0; k < 4; k++) q[k] = q[k] / n;
}

/* cross, src/common.f90:404-412 */
static void vcross(const double a[3], const double b[3], double r[3])
{
    double x = a[1] * b[2] - a[2] * b[1];
    double y = a[2] * b[0] - a[0] * b[2];
    double z = a[0] * b[1] - a[1] * b[0];
    r[0] = x;
    r[1] = y;
    r[2] = z;
}

static double vdot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static double dnrm2_3(const double x[3])
{
    double scale = 0, ssq = 1;
    for (int k = 0; k < 3; k++) {
        if (x[k] == 0) continue;
        double a = fabs(x[k]);
        if (scale < a) {
            double r = scale / a;
            ssq = 1 + ssq * r * r;
            scale = a;
        } else {
            double r = a / scale;
            ssq = ssq + r * r;
        }
    }
    return scale * sqrt(ssq);
}

/* positions of particles 2..N moved to the image nearest particle 1
 * (src/md.f90:345-355); the shift is stored in im */
static void to_first_image(double *x, int N, const double *edges, int *im)
{
    for (int i = 1; i < N; i++)
        for (int k = 0; k < 3; k++) {
            int m = (int)floor(((x[3 * i + k] - x[k]) / edges[k]) + 0.5);
            im[3 * i + k] = m;
            x[3 * i + k] = x[3 * i + k] - m * edges[k];
        }
}

int orc_rattle_body_pos(int N, double *pos, double *vel, double *pos_rattle, const int *species,
                        const double *mass, const int *links, const double *dist, int n_link, double dt,
                        const double *edges, double precision, int *im)
{
    to_first_image(pos, N, edges, im);
    to_first_image(pos_rattle, N, edges, im + 3 * N);
    int it;
    for (it = 1; it <= 1000; it++) {
        for (int l = 0; l < n_link; l++) {
            int a = links[2 * l] - 1, b = links[2 * l + 1] - 1;
            double d = dist[l], r[3], s[3];
            for (int k = 0; k < 3; k++) {
                r[k] = pos_rattle[3 * a + k] - pos_rattle[3 * b + k];
                s[k] = pos[3 * a + k] - pos[3 * b + k];
            }
            double ia = 1 / mass[species[a] - 1], ib = 1 / mass[species[b] - 1];
            double inv_mass = ia + ib;
            double rsq = vdot(r, r), ssq = vdot(s, s), rs = vdot(r, s);
            double g = rs - sqrt(rs * rs - rsq * (ssq - d * d));
            g = g / (dt * inv_mass * rsq);
            for (int k = 0; k < 3; k++) {
                pos[3 * a + k] = pos[3 * a + k] - g * dt * r[k] * ia;
                pos[3 * b + k] = pos[3 * b + k] + g * dt * r[k] * ib;
            }
            for (int k = 0; k < 3; k++) {
                vel[3 * a + k] = vel[3 * a + k] - g * r[k] * ia;
                vel[3 * b + k] = vel[3 * b + k] + g * r[k] * ib;
            }
        }
        double error = 0;
        for (int l = 0; l < n_link; l++) {
            int a = links[2 * l] - 1, b = links[2 * l + 1] - 1;
            double r[3];
            for (int k = 0; k < 3; k++) r[k] = pos[3 * a + k] - pos[3 * b + k];
            double g = fabs(sqrt(vdot(r, r)) - dist[l]);
            if (g > error) error = g;
        }
        if (error < precision) break;
    }
    for (int i = 1; i < N; i++)
        for (int k = 0; k < 3; k++) pos[3 * i + k] = pos[3 * i + k] + im[3 * i + k] * edges[k];
    return it;
}

int orc_rattle_body_vel(int N, double *pos, double *vel, const int *species, const double *mass,
                        const int *links, const double *dist, int n_link, const double *edges,
                        double precision, int *im)
{
    to_first_image(pos, N, edges, im);
    int it;
    for (it = 1; it <= 1000; it++) {
        for (int l = 0; l < n_link; l++) {
            int a = links[2 * l] - 1, b = links[2 * l + 1] - 1;
            double d = dist[l];
            double ia = 1 / mass[species[a] - 1], ib = 1 / mass[species[b] - 1];
            double inv_mass = ia + ib, s[3], w[3];
            for (int k = 0; k < 3; k++) {
                s[k] = pos[3 * a + k] - pos[3 * b + k];
                w[k] = vel[3 * a + k] - vel[3 * b + k];
            }
            double kk = vdot(w, s) / (d * d * inv_mass);
            for (int k = 0; k < 3; k++) {
                vel[3 * a + k] = vel[3 * a + k] - kk * s[k] * ia;
                vel[3 * b + k] = vel[3 * b + k] + kk * s[k] * ib;
            }
        }
        double error = 0;
        for (int l = 0; l < n_link; l++) {
            int a = links[2 * l] - 1, b = links[2 * l + 1] - 1;
            double d = dist[l];
            double ia = 1 / mass[species[a] - 1], ib = 1 / mass[species[b] - 1];
            double inv_mass = ia + ib, s[3], w[3];
            for (int k = 0; k < 3; k++) {
                s[k] = pos[3 * a + k] - pos[3 * b + k];
                w[k] = vel[3 * a + k] - vel[3 * b + k];
            }
            double kk = fabs(vdot(w, s) / (d * d * inv_mass));
            if (kk > error) error = kk;
        }
        if (error < precision) break;
    }
    for (int i = 1; i < N; i++)
        for (int k = 0; k < 3; k++) pos[3 * i + k] = pos[3 * i + k] + im[3 * i + k] * edges[k];
    return it;
}

/* rel_pos, src/common.f90:162-178 */
static double rel(double r, double L)
{
    if (r < -0.5 * L) return r + L;
    if (r > 0.5 * L) return r - L;
    return r;
}

double orc_elastic_network(const double *pos, double *force, const int *links, const double *dist, int n_link,
                           double kel, const double *edges)
{
    double e = 0;
    for (int l = 0; l < n_link; l++) {
        int a = links[2 * l] - 1, b = links[2 * l + 1] - 1;
        double r0 = dist[l], x[3];
        for (int k = 0; k < 3; k++) x[k] = rel(pos[3 * a + k] - pos[3 * b + k], edges[k]);
        double r = dnrm2_3(x);
        e = e + kel * ((r - r0) * (r - r0)) / 2;
        for (int k = 0; k < 3; k++) {
            double f = -(kel * (r - r0) * x[k] / r);
            force[3 * a + k] = force[3 * a + k] + f;
            force[3 * b + k] = force[3 * b + k] - f;
        }
    }
    return e;
}

/* rigid_body_init: st = [mass, pos3, vel3, force3, q4, L3, torque3, I3, omega3] */
void orc_rigid_body_init(const double *pos, const double *vel, const int *image, const int *species,
                         const double *mass_table, int i_start, int i_stop, const double *edges, double *st,
                         double *pos_body)
{
    double M = 0, c[3] = {0, 0, 0}, v[3] = {0, 0, 0}, I[3] = {0, 0, 0};
    for (int i = i_start - 1; i < i_stop; i++) {
        double m = mass_table[species[i] - 1];
        M = M + m;
        for (int k = 0; k < 3; k++) {
            c[k] = c[k] + m * (pos[3 * i + k] + image[3 * i + k] * edges[k]);
            v[k] = v[k] + m * vel[3 * i + k];
        }
    }
    for (int k = 0; k < 3; k++) {
        c[k] = c[k] / M;
        v[k] = v[k] / M;
    }
    for (int i = i_start - 1; i < i_stop; i++) {
        double m = mass_table[species[i] - 1], p[3];
        for (int k = 0; k < 3; k++) {
            p[k] = pos[3 * i + k] + image[3 * i + k] * edges[k] - c[k];
            pos_body[3 * (i - (i_start - 1)) + k] = p[k];
        }
        double sq = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        for (int k = 0; k < 3; k++) I[k] = I[k] + m * (sq - p[k] * p[k]);
    }
    memset(st, 0, 26 * sizeof(double));
    st[0] = M;
    for (int k = 0; k < 3; k++) {
        st[1 + k] = c[k];
        st[4 + k] = v[k];
        st[20 + k] = I[k];
    }
    st[10] = 1; /* q = (1, 0, 0, 0) */
}

#define ST_MASS 0
#define ST_POS 1
#define ST_VEL 4
#define ST_FORCE 7
#define ST_Q 10
#define ST_L 14
#define ST_TORQUE 17
#define ST_I 20
#define ST_OMEGA 23

void orc_rigid_body_force_torque(const double *force, int i_start, int i_stop, double *st, const double *pos_body)
{
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    for (int i = i_start - 1; i < i_stop; i++) {
        const double *f = force + 3 * i;
        double p[3], c[3];
        for (int k = 0; k < 3; k++) F[k] = F[k] + f[k];
        qrotate(st + ST_Q, pos_body + 3 * (i - (i_start - 1)), p);
        vcross(p, f, c);
        for (int k = 0; k < 3; k++) T[k] = T[k] + c[k];
    }
    for (int k = 0; k < 3; k++) {
        st[ST_FORCE + k] = F[k];
        st[ST_TORQUE + k] = T[k];
    }
}

int orc_rigid_body_vv1(double *pos, int i_start, int i_stop, double *st, const double *pos_body, double dt,
                       double treshold, const double *edges)
{
    double I_inv[3], L[3], q[4], qc[4], Lb[3], tb[3], wb[3], c[3], Lbd[3], qd[4], qo[4], w4[4];
    for (int k = 0; k < 3; k++) I_inv[k] = 1 / st[ST_I + k];
    for (int k = 0; k < 3; k++) L[k] = st[ST_L + k];
    for (int k = 0; k < 4; k++) q[k] = st[ST_Q + k];
    qstar(q, qc);
    qrotate(qc, L, Lb);
    qrotate(qc, st + ST_TORQUE, tb);
    for (int k = 0; k < 3; k++) wb[k] = Lb[k] * I_inv[k];
    vcross(wb, Lb, c);
    for (int k = 0; k < 3; k++) Lbd[k] = tb[k] - c[k];
    for (int k = 0; k < 3; k++) Lb[k] = Lb[k] + dt * Lbd[k] / 2;
    for (int k = 0; k < 3; k++) wb[k] = Lb[k] * I_inv[k];
    w4[0] = 0;
    for (int k = 0; k < 3; k++) w4[1 + k] = wb[k];
    qprod(q, w4, qd);
    for (int k = 0; k < 4; k++) qd[k] = qd[k] / 2;
    for (int k = 0; k < 4; k++) q[k] = q[k] + qd[k] * dt / 2;
    qunit(q);
    for (int k = 0; k < 3; k++) L[k] = st[ST_L + k] + st[ST_TORQUE + k] * dt / 2;
    for (int k = 0; k < 4; k++) qo[k] = q[k];
    int it = 0;
    for (;;) {
        qstar(q, qc);
        qrotate(qc, L, Lb);
        for (int k = 0; k < 3; k++) wb[k] = I_inv[k] * Lb[k];
        w4[0] = 0;
        for (int k = 0; k < 3; k++) w4[1 + k] = wb[k];
        qprod(q, w4, qd);
        for (int k = 0; k < 4; k++) qd[k] = qd[k] / 2;
        for (int k = 0; k < 4; k++) q[k] = st[ST_Q + k] + qd[k] * dt / 2;
        qunit(q);
        double dq[4];
        for (int k = 0; k < 4; k++) dq[k] = q[k] - qo[k];
        it++;
        if (qlen(dq) < treshold) break;
        for (int k = 0; k < 4; k++) qo[k] = q[k];
        if (it >= 100000) break;
    }
    for (int k = 0; k < 4; k++) st[ST_Q + k] = st[ST_Q + k] + dt * qd[k];
    qunit(st + ST_Q);
    for (int k = 0; k < 3; k++)
        st[ST_POS + k] = st[ST_POS + k] + st[ST_VEL + k] * dt + st[ST_FORCE + k] * (dt * dt) / (2 * st[ST_MASS]);
    for (int i = i_start - 1; i < i_stop; i++) {
        double r[3];
        qrotate(st + ST_Q, pos_body + 3 * (i - (i_start - 1)), r);
        for (int k = 0; k < 3; k++) {
            double old = pos[3 * i + k];
            double x = st[ST_POS + k] + r[k];
            double delta = x - old + edges[k] / 2;
            pos[3 * i + k] = x - floor(delta / edges[k]) * edges[k];
        }
    }
    for (int k = 0; k < 3; k++) st[ST_L + k] = st[ST_L + k] + st[ST_TORQUE + k] * dt / 2;
    for (int k = 0; k < 3; k++) st[ST_VEL + k] = st[ST_VEL + k] + st[ST_FORCE + k] * dt / (2 * st[ST_MASS]);
    return it;
}

void orc_rigid_body_vv2(double *vel, int i_start, int i_stop, double *st, const double *pos_body, double dt)
{
    double qc[4], Lb[3], w[3];
    for (int k = 0; k < 3; k++) st[ST_L + k] = st[ST_L + k] + st[ST_TORQUE + k] * dt / 2;
    qstar(st + ST_Q, qc);
    qrotate(qc, st + ST_L, Lb);
    for (int k = 0; k < 3; k++) st[ST_OMEGA + k] = Lb[k] / st[ST_I + k];
    qrotate(st + ST_Q, st + ST_OMEGA, w);
    for (int k = 0; k < 3; k++) st[ST_VEL + k] = st[ST_VEL + k] + st[ST_FORCE + k] * dt / (2 * st[ST_MASS]);
    for (int i = i_start - 1; i < i_stop; i++) {
        double p[3], c[3];
        qrotate(st + ST_Q, pos_body + 3 * (i - (i_start - 1)), p);
        vcross(w, p, c);
        for (int k = 0; k < 3; k++) vel[3 * i + k] = st[ST_VEL + k] + c[k];
    }
}
