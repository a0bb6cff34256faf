"""ctypes wrapper of the CPU oracle (oracle/_build/librmpcd_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py as the checker.  The oracle is an FP64 C
restatement of the reference routines (each function cites its
src/*.f90 lines in the C sources).  Parity status: pinned against the
reference's own property tests; element values are unpinned against the
Fortran binary, which cannot be built here.

Arrays use the reference layout: 3-vectors as numpy (N, 3) C-order arrays
(= Fortran (3, N)), cell_start 1-based, list entries 1-based.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "librmpcd_oracle.so"

REAC_BIT, MD_BIT, WALL_BIT, PAST_MD_BIT, CATALYZED_BIT = 1, 2, 3, 4, 6
PERIODIC_BC, BOUNCE_BACK_BC, SPECULAR_BC = 1, 2, 3


class Grid(C.Structure):
    _fields_ = [
        ("L", C.c_int * 3), ("edges", C.c_double * 3), ("a", C.c_double), ("origin", C.c_double * 3),
        ("M", C.c_int * 3), ("S", C.c_int), ("has_walls", C.c_int), ("bc", C.c_int * 3), ("max_v", C.c_double),
    ]


class OLJ(C.Structure):
    _fields_ = [("n1", C.c_int), ("n2", C.c_int)] + [
        (n, C.c_double * 16) for n in ("epsilon", "sigma", "sigma_sq", "cut", "cut_sq", "cut_energy")]


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        _lib.orc_compute_temperature.restype = C.c_double
        _lib.orc_maximum_displacement.restype = C.c_double
        _lib.orc_cell_maximum_displacement.restype = C.c_double
        _lib.orc_compute_force.restype = C.c_double
        _lib.orc_compute_force_n2.restype = C.c_double
        _lib.orc_normal.restype = C.c_double
        _lib.orc_lj_energy.restype = C.c_double
        _lib.orc_elastic_network.restype = C.c_double
        _lib.orc_rng_u2.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.POINTER(C.c_double)]
        _lib.orc_rand_sphere.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]
        _lib.orc_normal.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32]
        _lib.orc_random_shift_values.argtypes = [C.c_uint64, C.c_uint64, C.POINTER(C.c_double)]
    return _lib


def dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


def up(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_ubyte))


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---------------------------------------------------------------- hilbert / rng
def compact_p_to_h(p, M) -> int:
    pp = np.ascontiguousarray(p, np.int32)
    mm = np.ascontiguousarray(M, np.int32)
    return int(lib().orc_compact_p_to_h(ip(pp), ip(mm)))


def compact_h_to_p(h, M) -> np.ndarray:
    out = np.zeros(3, np.int32)
    mm = np.ascontiguousarray(M, np.int32)
    lib().orc_compact_h_to_p(int(h), ip(mm), ip(out))
    return out


def p_to_h(p, m) -> int:
    pp = np.ascontiguousarray(p, np.int32)
    return int(lib().orc_p_to_h(ip(pp), int(m)))


def rng_u2(seed, step, index, stream, attempt=0):
    out = np.zeros(2)
    lib().orc_rng_u2(seed, step, index, stream, attempt, dp(out))
    return out


def rand_sphere(seed, step, index):
    out = np.zeros(3)
    lib().orc_rand_sphere(seed, step, index, dp(out))
    return out


def normal(seed, step, index, sub):
    return float(lib().orc_normal(seed, step, index, sub))


def random_shift_values(seed, step):
    out = np.zeros(3)
    lib().orc_random_shift_values(seed, step, dp(out))
    return out


# ---------------------------------------------------------------- LJ
class LJParams:
    def __init__(self, epsilon, sigma, cut):
        eps = np.atleast_2d(np.asarray(epsilon, np.float64))
        sig = np.atleast_2d(np.asarray(sigma, np.float64))
        cu = np.atleast_2d(np.asarray(cut, np.float64))
        self.n1, self.n2 = eps.shape
        self.s = OLJ()
        fe = np.ascontiguousarray(eps.T.reshape(-1))
        fs = np.ascontiguousarray(sig.T.reshape(-1))
        fc = np.ascontiguousarray(cu.T.reshape(-1))
        lib().orc_lj_init(C.byref(self.s), self.n1, self.n2, dp(fe), dp(fs), dp(fc))

    def table(self, name):
        return np.array(getattr(self.s, name)[: self.n1 * self.n2]).reshape(self.n2, self.n1).T

    @property
    def cut_sq(self):
        return self.table("cut_sq")


# ---------------------------------------------------------------- systems
class Cells:
    def __init__(self, L, a=1.0, has_walls=False):
        self.g = Grid()
        lib().orc_grid_init(C.byref(self.g), ip(np.ascontiguousarray(L, np.int32)), C.c_double(a),
                            int(bool(has_walls)))
        self.S = self.g.S
        self.cell_count = np.zeros(self.S, np.int32)
        self.cell_start = np.ones(self.S, np.int32)
        self.is_md = np.zeros(self.S, np.uint8)
        self.is_reac = np.zeros(self.S, np.uint8)

    @property
    def L(self):
        return np.array(self.g.L[:])

    @property
    def M(self):
        return np.array(self.g.M[:])

    @property
    def edges(self):
        return np.array(self.g.edges[:])

    @property
    def origin(self):
        return np.array(self.g.origin[:])

    @origin.setter
    def origin(self, v):
        for k in range(3):
            self.g.origin[k] = float(v[k])

    def set_bc(self, bc):
        for k in range(3):
            self.g.bc[k] = int(bc[k])

    def random_shift(self, seed, step):
        self.origin = random_shift_values(seed, step)


class Particles:
    def __init__(self, N, n_species=1, mass=None):
        self.N = int(N)
        self.n_species = n_species
        self.mass = None if mass is None else np.asarray(mass, np.float64)
        self.pos = np.zeros((N, 3))
        self.pos_old = np.zeros((N, 3))
        self.vel = np.zeros((N, 3))
        self.force = np.zeros((N, 3))
        self.force_old = np.zeros((N, 3))
        self.image = np.zeros((N, 3), np.int32)
        self.id = np.arange(1, N + 1, dtype=np.int32)
        self.species = np.zeros(N, np.int32)
        self.flags = np.zeros(N, np.int32)
        self.id_to_idx = np.zeros(N, np.int32)
        self.pos_rattle = np.zeros((N, 3))

    def sort(self, c: Cells):
        lib().orc_sort(C.byref(c.g), self.N, ip(c.cell_count), ip(c.cell_start), dp(self.pos), dp(self.pos_old),
                       ip(self.image), dp(self.vel), dp(self.force), dp(self.force_old), ip(self.id),
                       ip(self.species), ip(self.flags), ip(self.id_to_idx))

    def count(self, c: Cells):
        lib().orc_count_particles(C.byref(c.g), self.N, dp(self.pos), ip(c.cell_count), ip(c.cell_start))

    def sort_particles(self, c: Cells) -> np.ndarray:
        """cell_system_t%sort_particles of this system's positions; returns
        the scattered positions (cell_start of c advances by the counts)."""
        out = np.zeros_like(self.pos)
        lib().orc_sort_particles(C.byref(c.g), self.N, ip(c.cell_start), dp(self.pos), dp(out))
        return out

    def maximum_displacement(self):
        return float(lib().orc_maximum_displacement(self.N, dp(self.pos), dp(self.pos_old), ip(self.species)))

    def switch_force(self):
        self.force, self.force_old = self.force_old, self.force


def simple_mpcd_step(p: Particles, c: Cells, seed, step, alpha=None, thermostat=False, T=0.0, hydro=True,
                     axes=None, gauss=None):
    ax = None if axes is None else np.ascontiguousarray(axes, np.float64)
    ga = None if gauss is None else np.ascontiguousarray(gauss, np.float64)
    rc = lib().orc_simple_mpcd_step(C.byref(c.g), p.N, ip(c.cell_count), ip(c.cell_start), dp(p.vel),
                                    ip(p.species), int(alpha is not None), C.c_double(alpha or 0.0),
                                    int(bool(thermostat)), C.c_double(T), int(bool(hydro)), C.c_uint64(seed),
                                    C.c_uint64(step), dp(ax), dp(ga))
    if rc != 0:
        raise RuntimeError("requiring .not.do_hydro without thermostat in simple_mpcd_step")


def wall_mpcd_step(p: Particles, c: Cells, seed, step, wall_temperature=None, wall_n=None, thermostat=False,
                   bulk_temperature=0.0, alpha=None, keep_cell_v=True):
    wt = np.zeros(2) if wall_temperature is None else np.ascontiguousarray(wall_temperature, np.float64)
    wn = np.zeros(2, np.int32) if wall_n is None else np.ascontiguousarray(wall_n, np.int32)
    wv = np.zeros(6)
    lib().orc_wall_mpcd_step(C.byref(c.g), p.N, ip(c.cell_count), ip(c.cell_start), dp(p.vel),
                             int(wall_temperature is not None), dp(wt), dp(wv), ip(wn), int(bool(thermostat)),
                             C.c_double(bulk_temperature), int(alpha is not None), C.c_double(alpha or 0.0),
                             int(bool(keep_cell_v)), C.c_uint64(seed), C.c_uint64(step))


def compute_temperature(p: Particles, c: Cells) -> float:
    return float(lib().orc_compute_temperature(C.byref(c.g), p.N, ip(c.cell_count), ip(c.cell_start),
                                               dp(p.vel), ip(p.species)))


def rescale_cells(p: Particles, c: Cells, T):
    lib().orc_rescale_cells(C.byref(c.g), p.N, ip(c.cell_count), ip(c.cell_start), dp(p.vel), ip(p.species),
                            C.c_double(T))


def mpcd_stream_periodic(p: Particles, c: Cells, dt):
    lib().orc_mpcd_stream_periodic(C.byref(c.g), p.N, dp(p.pos), dp(p.vel), ip(p.image), C.c_double(dt))


def mpcd_stream_xforce_yzwall(p: Particles, c: Cells, dt, g):
    lib().orc_mpcd_stream_xforce_yzwall(C.byref(c.g), p.N, dp(p.pos), dp(p.vel), ip(p.flags), C.c_double(dt),
                                        C.c_double(g))


def mpcd_stream_nogravity_zwall(p: Particles, c: Cells, dt):
    lib().orc_mpcd_stream_nogravity_zwall(C.byref(c.g), p.N, dp(p.pos), dp(p.vel), dp(p.force), ip(p.flags),
                                          C.c_double(dt))


def bulk_reaction(p: Particles, c: Cells, frm, to, rate, tau, seed, step):
    lib().orc_bulk_reaction(C.byref(c.g), p.N, ip(c.cell_count), ip(c.cell_start), up(c.is_reac), ip(p.species),
                            int(frm), int(to), C.c_double(rate), C.c_double(tau), C.c_uint64(seed),
                            C.c_uint64(step))


def bulk_reaction_endothermic(p: Particles, c: Cells, frm, to, rate, tau, delta_u, seed, step):
    lib().orc_bulk_reaction_endothermic(C.byref(c.g), p.N, ip(c.cell_count), ip(c.cell_start), up(c.is_reac),
                                        ip(p.species), dp(p.vel), int(frm), int(to), C.c_double(rate),
                                        C.c_double(tau), C.c_double(delta_u), C.c_uint64(seed), C.c_uint64(step))


def md_pos(p: Particles, dt):
    lib().orc_md_pos(p.N, dp(p.pos), dp(p.vel), dp(p.force), C.c_double(dt))


def md_vel(p: Particles, dt):
    lib().orc_md_vel(p.N, dp(p.vel), dp(p.force), dp(p.force_old), ip(p.flags), C.c_double(dt))


def cell_md_pos(c: Cells, p: Particles, dt, md_flag):
    lib().orc_cell_md_pos(C.byref(c.g), ip(c.cell_count), ip(c.cell_start), up(c.is_md), dp(p.pos), dp(p.vel),
                          dp(p.force), C.c_double(dt), int(bool(md_flag)))


def cell_md_vel(c: Cells, p: Particles, dt, md_flag):
    lib().orc_cell_md_vel(C.byref(c.g), ip(c.cell_count), ip(c.cell_start), up(c.is_md), dp(p.vel), dp(p.force),
                          dp(p.force_old), ip(p.flags), C.c_double(dt), int(bool(md_flag)))


def cell_md_pos_wall(c: Cells, p: Particles, dim, dt, md_flag):
    lib().orc_cell_md_pos_wall(C.byref(c.g), int(dim), ip(c.cell_count), ip(c.cell_start), up(c.is_md),
                               dp(p.pos), dp(p.vel), dp(p.force), C.c_double(dt), int(bool(md_flag)))


def apply_pbc(p: Particles, edges):
    e = np.ascontiguousarray(edges, np.float64)
    lib().orc_apply_pbc(p.N, dp(p.pos), ip(p.image), dp(e))


def cell_maximum_displacement(c: Cells, p: Particles, delta_t):
    return float(lib().orc_cell_maximum_displacement(C.byref(c.g), ip(c.cell_count), ip(c.cell_start),
                                                     up(c.is_md), dp(p.pos), dp(p.pos_old), ip(p.species),
                                                     C.c_double(delta_t)))


def rattle_dimer_pos(p: Particles, d, dt, edges):
    e = np.ascontiguousarray(edges, np.float64)
    m1 = p.mass[p.species[0] - 1]
    m2 = p.mass[p.species[1] - 1]
    lib().orc_rattle_dimer_pos(dp(p.pos), dp(p.vel), dp(p.pos_rattle), C.c_double(m1), C.c_double(m2),
                               C.c_double(d), C.c_double(dt), dp(e))


def rattle_dimer_vel(p: Particles, d, dt, edges):
    e = np.ascontiguousarray(edges, np.float64)
    m1 = p.mass[p.species[0] - 1]
    m2 = p.mass[p.species[1] - 1]
    lib().orc_rattle_dimer_vel(dp(p.pos), dp(p.vel), C.c_double(m1), C.c_double(m2), C.c_double(d),
                               C.c_double(dt), dp(e))


def colloid_vv_pos(p: Particles, dt, mass):
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float64), (p.N,)))
    lib().orc_colloid_vv_pos(p.N, dp(p.pos), dp(p.vel), dp(p.force), dp(m), C.c_double(dt))


def colloid_vv_vel(p: Particles, dt, mass):
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float64), (p.N,)))
    lib().orc_colloid_vv_vel(p.N, dp(p.vel), dp(p.force), dp(p.force_old), dp(m), C.c_double(dt))


class NeighborList:
    def __init__(self, Npoints, Nmax):
        self.Npoints, self.Nmax = Npoints, Nmax
        self.list = np.zeros((Npoints, Nmax), np.int32)
        self.n = np.zeros(Npoints, np.int32)
        self.stencil = np.zeros((0, 3), np.int32)

    def make_stencil(self, c: Cells, cut):
        cap = 200000
        buf = np.zeros((cap, 3), np.int32)
        n = lib().orc_make_stencil(C.c_double(c.g.a), C.c_double(cut), ip(buf), cap)
        self.stencil = buf[:n].copy()

    def update_list(self, colloids: Particles, solvent: Particles, radius, c: Cells, lj: LJParams | None = None):
        st = np.ascontiguousarray(self.stencil)
        rc = lib().orc_update_list(C.byref(c.g), colloids.N, dp(colloids.pos), ip(colloids.species), solvent.N,
                                   dp(solvent.pos), ip(solvent.species), ip(c.cell_count), ip(c.cell_start),
                                   ip(st), len(st), C.c_double(radius), C.byref(lj.s) if lj else None, self.Nmax,
                                   ip(self.list), ip(self.n), up(c.is_md), up(c.is_reac))
        if rc != 0:
            raise RuntimeError("maximum of neighbor list reached")


def compute_force(colloids: Particles, solvent: Particles, nl: NeighborList, L, lj: LJParams) -> float:
    e = np.ascontiguousarray(L, np.float64)
    return float(lib().orc_compute_force(colloids.N, dp(colloids.pos), ip(colloids.species), dp(colloids.force),
                                         solvent.N, dp(solvent.pos), ip(solvent.species), dp(solvent.force),
                                         ip(solvent.flags), ip(nl.list), ip(nl.n), nl.Nmax, dp(e), C.byref(lj.s)))


def compute_force_n2(ps: Particles, L, lj: LJParams) -> float:
    e = np.ascontiguousarray(L, np.float64)
    return float(lib().orc_compute_force_n2(ps.N, dp(ps.pos), ip(ps.species), dp(ps.force), dp(e),
                                            C.byref(lj.s)))


def flag_particles_nl(nl: NeighborList, colloids: Particles, solvent: Particles, edges, cut_sq, point=0):
    e = np.ascontiguousarray(edges, np.float64)
    l1 = np.ascontiguousarray(nl.list[point])
    c1 = np.ascontiguousarray(colloids.pos[point])
    lib().orc_flag_particles_nl(int(nl.n[point]), ip(l1), dp(c1), dp(solvent.pos), ip(solvent.species),
                                ip(solvent.flags), dp(e), C.c_double(cut_sq))


def change_species(solvent: Particles, colloids: Particles, edges, cut_c, cut_n, prob, seed, step):
    e = np.ascontiguousarray(edges, np.float64)
    c1 = np.ascontiguousarray(colloids.pos[0])
    c2 = np.ascontiguousarray(colloids.pos[1])
    lib().orc_change_species(solvent.N, dp(c1), dp(c2), dp(solvent.pos), ip(solvent.species), ip(solvent.flags),
                             dp(e), C.c_double(cut_c), C.c_double(cut_n), C.c_double(prob), C.c_uint64(seed),
                             C.c_uint64(step))


def refuel(solvent: Particles, colloids: Particles, edges, L1):
    e = np.ascontiguousarray(edges, np.float64)
    c1 = np.ascontiguousarray(colloids.pos[0])
    c2 = np.ascontiguousarray(colloids.pos[1])
    lib().orc_refuel(solvent.N, dp(c1), dp(c2), dp(solvent.pos), ip(solvent.species), dp(e), int(L1))


def n_solvent(solvent: Particles, n_species):
    out = np.zeros(n_species, np.int32)
    lib().orc_n_solvent(solvent.N, ip(solvent.species), int(n_species), ip(out))
    return out


def cylindrical_shell_histogram(solvent: Particles, x1, x2, L, bin_species, r_min, r_max, xmin, dx, nbins):
    h = np.zeros(nbins)
    a = np.ascontiguousarray(x1, np.float64)
    b = np.ascontiguousarray(x2, np.float64)
    e = np.ascontiguousarray(L, np.float64)
    lib().orc_cylindrical_shell_histogram(dp(a), dp(b), dp(e), int(bin_species), C.c_double(r_min),
                                          C.c_double(r_max), solvent.N, dp(solvent.pos), ip(solvent.species),
                                          C.c_double(xmin), C.c_double(dx), int(nbins), dp(h))
    return h


def velocity_sums(p: Particles):
    out = np.zeros(4)
    lib().orc_velocity_sums(p.N, dp(p.vel), dp(out))
    return out


def random_placement(p: Particles, L, seed, colloids: Particles | None = None, lj: LJParams | None = None):
    e = np.ascontiguousarray(L, np.float64)
    C_ = 0 if colloids is None else colloids.N
    lib().orc_random_placement(p.N, dp(p.pos), ip(p.species) if colloids is not None else None, dp(e), C_,
                               dp(colloids.pos) if colloids is not None else None,
                               ip(colloids.species) if colloids is not None else None,
                               C.byref(lj.s) if lj is not None else None, C.c_uint64(seed))


def maxwell_velocities(p: Particles, T, seed):
    lib().orc_maxwell_velocities(p.N, dp(p.vel), C.c_double(T), C.c_uint64(seed))


def bulk_run(p: Particles, c: Cells, n_intervals, tau, seed, step_base, alpha=None):
    out = np.zeros(3)
    lib().orc_bulk_run(C.byref(c.g), p.N, int(n_intervals), C.c_double(tau), C.c_double(alpha or 0.0),
                       int(alpha is not None), C.c_uint64(seed), C.c_uint64(step_base), dp(p.pos), ip(p.image),
                       dp(p.vel), ip(p.id), ip(p.species), ip(p.flags), ip(c.cell_count), ip(c.cell_start),
                       dp(out))
    c.origin = out


# ---------------------------------------------------------------------------
# rigid-body colloids (src/md.f90:321-700)
# ---------------------------------------------------------------------------
def _links(links, distances):
    lk = np.ascontiguousarray(links, np.int32).reshape(-1, 2)
    d = np.ascontiguousarray(distances, np.float64).reshape(-1)
    assert len(lk) == len(d)
    return lk, d


def rattle_body_pos(p: Particles, links, distances, dt, edges, precision):
    """rattle_body_pos; returns the reference's rattle_i at exit."""
    lk, d = _links(links, distances)
    e = np.ascontiguousarray(edges, np.float64)
    im = np.zeros(6 * p.N, np.int32)
    return int(lib().orc_rattle_body_pos(p.N, dp(p.pos), dp(p.vel), dp(p.pos_rattle), ip(p.species), dp(p.mass),
                                         ip(lk), dp(d), len(d), C.c_double(dt), dp(e), C.c_double(precision),
                                         ip(im)))


def rattle_body_vel(p: Particles, links, distances, dt, edges, precision):
    lk, d = _links(links, distances)
    e = np.ascontiguousarray(edges, np.float64)
    im = np.zeros(6 * p.N, np.int32)
    return int(lib().orc_rattle_body_vel(p.N, dp(p.pos), dp(p.vel), ip(p.species), dp(p.mass), ip(lk), dp(d),
                                         len(d), dp(e), C.c_double(precision), ip(im)))


def elastic_network(p: Particles, links, distances, k, edges):
    lk, d = _links(links, distances)
    e = np.ascontiguousarray(edges, np.float64)
    return float(lib().orc_elastic_network(dp(p.pos), dp(p.force), ip(lk), dp(d), len(d), C.c_double(k), dp(e)))


class RigidBody:
    """rigid_body_t; state st[26] = mass, pos, vel, force, q (s,x,y,z), L,
    torque, I_body, omega_body."""

    FIELDS = (("mass", 0, 1), ("pos", 1, 3), ("vel", 4, 3), ("force", 7, 3), ("q", 10, 4), ("L", 14, 3),
              ("torque", 17, 3), ("I_body", 20, 3), ("omega_body", 23, 3))

    def __init__(self, p: Particles, i_start, i_stop, edges):
        self.i_start, self.i_stop = int(i_start), int(i_stop)
        self.st = np.zeros(26)
        self.pos_body = np.zeros((self.i_stop - self.i_start + 1, 3))
        e = np.ascontiguousarray(edges, np.float64)
        lib().orc_rigid_body_init(dp(p.pos), dp(p.vel), ip(p.image), ip(p.species), dp(p.mass), self.i_start,
                                  self.i_stop, dp(e), dp(self.st), dp(self.pos_body))

    def state(self):
        return {n: (self.st[a] if k == 1 else self.st[a:a + k].copy()) for n, a, k in self.FIELDS}

    def compute_force_torque(self, p: Particles):
        lib().orc_rigid_body_force_torque(dp(p.force), self.i_start, self.i_stop, dp(self.st), dp(self.pos_body))

    def vv1(self, p: Particles, dt, treshold, edges):
        e = np.ascontiguousarray(edges, np.float64)
        return int(lib().orc_rigid_body_vv1(dp(p.pos), self.i_start, self.i_stop, dp(self.st), dp(self.pos_body),
                                            C.c_double(dt), C.c_double(treshold), dp(e)))

    def vv2(self, p: Particles, dt):
        lib().orc_rigid_body_vv2(dp(p.vel), self.i_start, self.i_stop, dp(self.st), dp(self.pos_body),
                                 C.c_double(dt))
