"""Oracle twin of the program drivers (test infrastructure): the loops of
programs/single_dimer_pbc.f90 and programs/n_colloids_pbc.f90 over the
oracle's C routines, consuming random steps in the same order as
rmpcdmd_b200.programs.SingleDimerPBC and NColloidsPBC."""
from __future__ import annotations

import numpy as np

from . import oracle as O

PI_SP = float(np.float32(3.14159265))
TWO_SIXTH = 2.0 ** (1.0 / 6.0)


class SingleDimerPBC:
    def __init__(self, L=(32, 32, 32), rho=10, T=1.0 / 3.0, tau=1.0, N_MD=100, sigma_C=2.0, sigma_N=2.0, d=4.5,
                 epsilon_C=(1.0, 1.0), epsilon_N=(1.0, 0.5), epsilon_CC=1.0, epsilon_NC=1.0, epsilon_NN=1.0,
                 probability=1.0, bulk_rmpcd=False, bulk_rate=0.001, do_thermostat=False, do_hydro=True,
                 seed=1, skin=2.0, list_capacity=None):
        self.L = np.asarray(L, dtype=np.int32)
        self.rho, self.T, self.tau, self.N_MD = rho, T, tau, N_MD
        self.dt = tau / N_MD
        self.d, self.prob = d, probability
        self.bulk_rmpcd, self.bulk_rate = bulk_rmpcd, bulk_rate
        self.do_thermostat, self.do_hydro = do_thermostat, do_hydro
        self.skin = skin
        self.seed = seed
        self.step = 0
        self.N = int(rho * self.L.prod())
        eps = np.zeros((2, 2))
        eps[:, 0] = epsilon_C
        eps[:, 1] = epsilon_N
        sig = np.zeros((2, 2))
        sig[:, 0] = sigma_C
        sig[:, 1] = sigma_N
        self.lj = O.LJParams(eps, sig, sig * TWO_SIXTH)
        self.max_cut = float((sig * TWO_SIXTH).max())
        ceps = np.array([[epsilon_CC, epsilon_NC], [epsilon_NC, epsilon_NN]], dtype=np.float64)
        csig = np.array([[2 * sigma_C, sigma_C + sigma_N], [sigma_C + sigma_N, 2 * sigma_N]], dtype=np.float64)
        self.clj = O.LJParams(ceps, csig, csig * TWO_SIXTH)
        self.mass = np.array([rho * sigma_C ** 3 * 4 * PI_SP / 3, rho * sigma_N ** 3 * 4 * PI_SP / 3])
        self.s = O.Particles(self.N, 2)
        self.c = O.Particles(2, 2, self.mass)
        self.c.species[:] = [1, 2]
        O.maxwell_velocities(self.s, T, seed)
        self.s.species[:] = 1
        self.cells = O.Cells(self.L, 1.0)
        self.edges = self.cells.edges
        self.c.pos[0] = self.edges / 2.0
        self.c.pos[1] = self.edges / 2.0
        self.c.pos[1, 0] += d
        O.random_placement(self.s, self.edges, seed, self.c, self.lj)
        self.s.sort(self.cells)
        cap = list_capacity if list_capacity is not None else int(300 * max(sigma_C, sigma_N) ** 3)
        self.nl = O.NeighborList(2, cap)
        self.nl.make_stencil(self.cells, self.max_cut + skin)
        self.nl.update_list(self.c, self.s, self.max_cut + skin, self.cells, self.lj)
        self.cut_sq = self.lj.cut_sq
        self.e1 = O.compute_force(self.c, self.s, self.nl, self.edges, self.lj)
        self.e2 = O.compute_force_n2(self.c, self.edges, self.clj)
        self.s.force_old[:] = self.s.force
        self.c.force_old[:] = self.c.force
        self.n_extra_sorting = 0

    def _next(self):
        st = self.step
        self.step += 1
        return st

    def _resort(self):
        O.apply_pbc(self.s, self.edges)
        O.apply_pbc(self.c, self.edges)
        self.s.sort(self.cells)
        self.nl.update_list(self.c, self.s, self.max_cut + self.skin, self.cells, self.lj)
        self.s.pos_old[:] = self.s.pos
        self.c.pos_old[:] = self.c.pos

    def md_step(self):
        s, c, dt = self.s, self.c, self.dt
        O.md_pos(s, dt)
        c.pos_rattle[:] = c.pos
        O.colloid_vv_pos(c, dt, self.mass)
        O.rattle_dimer_pos(c, self.d, dt, self.edges)
        so_max = s.maximum_displacement()
        co_max = c.maximum_displacement()
        if (co_max >= self.skin * 0.1) or (so_max >= self.skin * 0.89):
            self._resort()
            self.n_extra_sorting += 1
        s.switch_force()
        c.switch_force()
        s.force[:] = 0
        c.force[:] = 0
        self.e1 = O.compute_force(c, s, self.nl, self.edges, self.lj)
        self.e2 = O.compute_force_n2(c, self.edges, self.clj)
        O.md_vel(s, dt)
        O.colloid_vv_vel(c, dt, self.mass)
        O.rattle_dimer_vel(c, self.d, dt, self.edges)
        O.flag_particles_nl(self.nl, c, s, self.edges, self.cut_sq[0, 0])
        O.change_species(s, c, self.edges, self.cut_sq[0, 0], self.cut_sq[0, 1], self.prob, self.seed, self._next())

    def interval(self):
        self.md_loop()
        self.mpcd()

    def md_loop(self):
        for _ in range(self.N_MD):
            self.md_step()

    def thermo(self):
        """programs/single_dimer_pbc.f90:388-396: internal energy e1 + e2 +
        kinetic and the centre-of-mass velocity after md_loop."""
        cv = self.c.vel
        kin = (self.mass[0] * (cv[0] ** 2).sum() + self.mass[1] * (cv[1] ** 2).sum()) / 2 + (self.s.vel ** 2).sum() / 2
        vcom = (self.s.vel.sum(0) + self.mass[0] * cv[0] + self.mass[1] * cv[1]) / (self.N + self.mass[0] + self.mass[1])
        return dict(internal=self.e1 + self.e2 + kin, v_com=vcom)

    def mpcd(self):
        self.cells.random_shift(self.seed, self._next())
        self._resort()
        O.simple_mpcd_step(self.s, self.cells, self.seed, self._next(), thermostat=self.do_thermostat, T=self.T,
                           hydro=self.do_hydro)
        if self.bulk_rmpcd:
            O.bulk_reaction(self.s, self.cells, 2, 1, self.bulk_rate, self.tau, self.seed, self._next())
        else:
            O.refuel(self.s, self.c, self.edges, int(self.L[0]))


PI_3141 = float(np.float32(3.141))
PI_3142 = float(np.float32(3.142))
COLLOID_PLACE_STEP = 0xFFFFFFFFFFFFFFFF
PLACE_STREAM = 5


def place_colloids(seed, n, edges, min_dist):
    """programs/n_colloids_pbc.f90:193-210 with the oracle's Philox draws."""
    edges = np.asarray(edges, np.float64)
    pos = np.zeros((n, 3))
    i = k = 0
    while i < n:
        u0, u1 = O.rng_u2(seed, COLLOID_PLACE_STEP, k, PLACE_STREAM, 0)
        u2, _ = O.rng_u2(seed, COLLOID_PLACE_STEP, k, PLACE_STREAM, 1)
        k += 1
        x = np.array([u0 * edges[0], u1 * edges[1], u2 * edges[2]])
        ok = True
        for j in range(i):
            d = x - pos[j]
            d = d - np.where(d < -edges / 2, -edges, 0) - np.where(d > edges / 2, edges, 0)
            if float((d ** 2).sum()) < min_dist ** 2:
                ok = False
                break
        if ok:
            pos[i] = x
            i += 1
    return pos


class NColloidsPBC:
    def __init__(self, L=(32, 32, 32), rho=10, T=1.0 / 3.0, T_final=None, tau=1.0, N_MD=100, N_colloids=10,
                 sigma=3.0, epsilon=1.0, epsilon_colloids=1.0, do_hydro=True, do_thermostat=False, seed=1,
                 skin=0.8, list_capacity=None, volume_correction=True):
        self.L = np.asarray(L, dtype=np.int32)
        self.rho, self.T_init, self.tau, self.N_MD = rho, T, tau, N_MD
        self.T_final = T if T_final is None else T_final
        self.dt = tau / N_MD
        self.do_hydro, self.do_thermostat = do_hydro, do_thermostat
        self.skin, self.seed, self.step = skin, seed, 0
        vol = int(rho * 4 * PI_3142 / 3 * sigma ** 3 * N_colloids) if volume_correction else 0
        self.N = int(rho * int(self.L.prod())) - vol
        self.mass = rho * sigma ** 3 * 4 * PI_3141 / 3
        sigma_cut = sigma * 2.0 ** (1.0 / 6.0)
        self.lj = O.LJParams([[epsilon]], [[sigma]], [[sigma_cut]])
        self.clj = O.LJParams([[epsilon_colloids]], [[2 * sigma]], [[2 * (3 * sigma)]])
        self.c = O.Particles(N_colloids, 1, [self.mass])
        self.c.species[:] = 1
        self.vv_mass = np.full(N_colloids, self.mass)
        self.s = O.Particles(self.N, 1)
        O.maxwell_velocities(self.s, T, seed)
        self.s.species[:] = 1
        self.cells = O.Cells(self.L, 1.0)
        self.edges = self.cells.edges
        self.c.pos[:] = place_colloids(seed, N_colloids, self.edges, 2 * sigma)
        O.random_placement(self.s, self.edges, seed, self.c, self.lj)
        self.s.sort(self.cells)
        self.radius = sigma_cut + skin
        cap = list_capacity if list_capacity is not None else int(250 * (sigma_cut + skin) ** 2)
        self.nl = O.NeighborList(N_colloids, cap)
        self.nl.make_stencil(self.cells, self.radius)
        self.nl.update_list(self.c, self.s, self.radius, self.cells)
        self.e1 = O.compute_force(self.c, self.s, self.nl, self.edges, self.lj)
        self.e2 = O.compute_force_n2(self.c, self.edges, self.clj)
        self.s.force_old[:] = self.s.force
        self.c.force_old[:] = self.c.force
        self.s.pos_old[:] = self.s.pos
        self.c.pos_old[:] = self.c.pos
        self.n_extra_sorting = 0
        self.t = 0
        self.last_sort = 0

    def _next(self):
        st = self.step
        self.step += 1
        return st

    def _catch_up_and_sort(self):
        s, c, dtl = self.s, self.c, (self.t - self.last_sort) * self.dt
        O.cell_md_pos(self.cells, s, dtl, False)
        O.cell_md_vel(self.cells, s, dtl, False)
        O.apply_pbc(s, self.edges)
        O.apply_pbc(c, self.edges)
        s.sort(self.cells)
        self.last_sort = self.t
        self.nl.update_list(c, s, self.radius, self.cells)
        s.pos_old[:] = s.pos
        c.pos_old[:] = c.pos

    def md_step(self):
        s, c, dt = self.s, self.c, self.dt
        self.t += 1
        O.cell_md_pos(self.cells, s, dt, True)
        O.colloid_vv_pos(c, dt, self.vv_mass)
        so_max = O.cell_maximum_displacement(self.cells, s, dt * (self.t - self.last_sort))
        co_max = c.maximum_displacement()
        if (co_max >= self.skin * 0.1) or (so_max >= self.skin * 0.9):
            self._catch_up_and_sort()
            self.n_extra_sorting += 1
        s.switch_force()
        c.switch_force()
        s.force[:] = 0
        c.force[:] = 0
        self.e1 = O.compute_force(c, s, self.nl, self.edges, self.lj)
        self.e2 = O.compute_force_n2(c, self.edges, self.clj)
        O.cell_md_vel(self.cells, s, dt, True)
        O.colloid_vv_vel(c, dt, self.vv_mass)

    def interval(self, thermostat, T, rescale=False):
        for _ in range(self.N_MD):
            self.md_step()
        self.cells.random_shift(self.seed, self._next())
        self._catch_up_and_sort()
        O.simple_mpcd_step(self.s, self.cells, self.seed, self._next(), thermostat=thermostat, T=T,
                           hydro=self.do_hydro)
        if rescale:
            O.rescale_cells(self.s, self.cells, self.T_init)

    def thermalise(self, n_loops):
        for i in range(1, n_loops + 1):
            self.interval(True, self.T_init, rescale=(i % 10 == 0))
        self.t = self.last_sort = 0

    def run(self, n_loops):
        for i in range(1, n_loops + 1):
            T = self.T_init + (i - 1) * (self.T_final - self.T_init) / max(1, n_loops - 1)
            self.interval(self.do_thermostat, T)
