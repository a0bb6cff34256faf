"""Oracle twin of the program drivers (test infrastructure): the loop of
programs/single_dimer_pbc.f90 over the oracle's C routines, consuming random
steps in the same order as rmpcdmd_b200.programs.SingleDimerPBC."""
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
        for _ in range(self.N_MD):
            self.md_step()
        self.cells.random_shift(self.seed, self._next())
        self._resort()
        O.simple_mpcd_step(self.s, self.cells, self.seed, self._next(), thermostat=self.do_thermostat, T=self.T,
                           hydro=self.do_hydro)
        if self.bulk_rmpcd:
            O.bulk_reaction(self.s, self.cells, 2, 1, self.bulk_rate, self.tau, self.seed, self._next())
        else:
            O.refuel(self.s, self.c, self.edges, int(self.L[0]))
