"""Host drivers for the reference programs whose solvent loops this library
accelerates, written against the C ABI exactly as the Fortran programs call
their modules:

  * :class:`SingleDimerPBC` -- programs/single_dimer_pbc.f90:108-445
  * :class:`DimerBatch`     -- that program's main loop for many replicas at
                               once (one launch per phase, graph-replayed)
  * :class:`NColloidsPBC`   -- programs/n_colloids_pbc.f90:147-336
  * :func:`bulk_fluid`      -- the loop of test/setup_bulk_decay.f90:99-121

The randomness differs from the reference only in its source (Philox keyed
by seed and step instead of per-thread Threefry streams); the order of random
consumers is fixed so that any other driver making the same calls draws the
same numbers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api as A
from ._capi import DIMER_PARAMS, NCOLLOIDS_PARAMS, NCOLLOIDS_STATE, RNG, call, lib

PI_SP = float(np.float32(3.14159265))  # the default-real constant of the program
TWO_SIXTH = 2.0 ** (1.0 / 6.0)


def dimer_lj_tables(sigma_C, sigma_N, epsilon_C, epsilon_N, epsilon_CC, epsilon_NC, epsilon_NN):
    """The two lj_params_t tables of programs/single_dimer_pbc.f90:156-178."""
    eps = np.zeros((2, 2))
    eps[:, 0] = epsilon_C
    eps[:, 1] = epsilon_N
    sig = np.zeros((2, 2))
    sig[:, 0] = sigma_C
    sig[:, 1] = sigma_N
    solvent_colloid = (eps.copy(), sig.copy(), sig * TWO_SIXTH)
    ceps = np.array([[epsilon_CC, epsilon_NC], [epsilon_NC, epsilon_NN]], dtype=np.float64)
    csig = np.array([[2 * sigma_C, sigma_C + sigma_N], [sigma_C + sigma_N, 2 * sigma_N]], dtype=np.float64)
    colloid = (ceps, csig, csig * TWO_SIXTH)
    return solvent_colloid, colloid


def dimer_masses(rho, sigma_C, sigma_N):
    """mass = rho * sigma**3 * 4 * 3.14159265/3 (programs/single_dimer_pbc.f90:180-181)."""
    return np.array([rho * sigma_C ** 3 * 4 * PI_SP / 3, rho * sigma_N ** 3 * 4 * PI_SP / 3])


class SingleDimerPBC:
    """programs/single_dimer_pbc.f90 on the GPU.

    The neighbor-list capacity is a parameter: the program's own value,
    int(300*max(sigma)**3), is too small for sigma = 2 with skin 2 and makes the
    reference stop with 'maximum of neighbor list reached'.
    """

    def __init__(self, L=(32, 32, 32), rho=10, T=1.0 / 3.0, tau=1.0, N_MD=100, sigma_C=2.0, sigma_N=2.0, d=4.5,
                 epsilon_C=(1.0, 1.0), epsilon_N=(1.0, 0.5), epsilon_CC=1.0, epsilon_NC=1.0, epsilon_NN=1.0,
                 probability=1.0, bulk_rmpcd=False, bulk_rate=0.001, do_thermostat=False, do_hydro=True,
                 seed=1, skin=2.0, list_capacity=None, precision=A.FP64, initial_velocities=None):
        self._init_kwargs = dict(
            L=[int(x) for x in L], rho=rho, T=T, tau=tau, N_MD=N_MD, sigma_C=sigma_C, sigma_N=sigma_N, d=d,
            epsilon_C=[float(x) for x in epsilon_C], epsilon_N=[float(x) for x in epsilon_N], epsilon_CC=epsilon_CC,
            epsilon_NC=epsilon_NC, epsilon_NN=epsilon_NN, probability=probability, bulk_rmpcd=bulk_rmpcd,
            bulk_rate=bulk_rate, do_thermostat=do_thermostat, do_hydro=do_hydro, seed=int(seed), skin=skin,
            list_capacity=list_capacity, precision=precision)
        self.L = np.asarray(L, dtype=np.int32)
        self.rho, self.T, self.tau, self.N_MD = rho, T, tau, N_MD
        self.dt = tau / N_MD
        self.d = d
        self.prob = probability
        self.bulk_rmpcd, self.bulk_rate = bulk_rmpcd, bulk_rate
        self.do_thermostat, self.do_hydro = do_thermostat, do_hydro
        self.skin = skin
        self.N = int(rho * self.L.prod())
        (e, s, c), (ce, cs, cc) = dimer_lj_tables(sigma_C, sigma_N, epsilon_C, epsilon_N, epsilon_CC, epsilon_NC,
                                                  epsilon_NN)
        self.solvent_colloid_lj = A.LJParams(e, s, c)
        self.colloid_lj = A.LJParams(ce, cs, cc)
        self.max_cut = float(c.max())
        self.mass = dimer_masses(rho, sigma_C, sigma_N)
        self.rng = A.Rng(seed)
        self.solvent = A.ParticleSystem(self.N, 2, None, precision)
        self.colloids = A.ParticleSystem(2, 2, self.mass)
        self.colloids.species = [1, 2]
        if initial_velocities is not None:
            self.solvent.vel = initial_velocities
        else:
            self.solvent.maxwell(T, seed)
        self.solvent.species = 1
        self.cells = A.CellSystem(self.L, 1.0)
        self.edges = self.cells.edges
        cpos = np.array([self.edges / 2.0, self.edges / 2.0])
        cpos[1, 0] += d
        self.colloids.pos = cpos
        self.solvent.random_placement(self.edges, self.colloids, self.solvent_colloid_lj, seed)
        self.solvent.sort(self.cells)
        cap = list_capacity if list_capacity is not None else int(300 * max(sigma_C, sigma_N) ** 3)
        self.neigh = A.NeighborList(2, cap)
        self.neigh.make_stencil(self.cells, self.max_cut + skin)
        self.neigh.update_list(self.colloids, self.solvent, self.max_cut + skin, self.cells, self.solvent_colloid_lj)
        self.cut_sq = self.solvent_colloid_lj.cut_sq
        self.e1 = A.compute_force(self.colloids, self.solvent, self.neigh, self.edges, self.solvent_colloid_lj)
        self.e2 = A.compute_force_n2(self.colloids, self.edges, self.colloid_lj)
        self.solvent.copy_force_old()
        self.colloids.copy_force_old()
        self.n_extra_sorting = 0
        self.md_steps = 0

    def md_step(self, want_energy=False):
        """One pass of md_loop, programs/single_dimer_pbc.f90:306-384."""
        s, c, dt = self.solvent, self.colloids, self.dt
        A.md_pos(s, dt)
        c.copy_pos_rattle()
        A.colloid_vv_pos(c, dt, self.mass)
        A.rattle_dimer_pos(c, self.d, dt, self.edges)
        so_max = s.maximum_displacement()
        co_max = c.maximum_displacement()
        if (co_max >= self.skin * 0.1) or (so_max >= self.skin * 0.89):
            self._resort()
            self.n_extra_sorting += 1
        s.switch_force()
        c.switch_force()
        s.zero_force()
        c.zero_force()
        e1 = A.compute_force(c, s, self.neigh, self.edges, self.solvent_colloid_lj, energy=want_energy)
        e2 = A.compute_force_n2(c, self.edges, self.colloid_lj, energy=want_energy)
        if want_energy:
            self.e1, self.e2 = e1, e2
        A.md_vel(s, dt)
        A.colloid_vv_vel(c, dt, self.mass)
        A.rattle_dimer_vel(c, self.d, dt, self.edges)
        A.flag_particles_nl(self.neigh, c, s, self.edges, self.cut_sq[0, 0])
        A.change_species(s, c, self.edges, self.cut_sq[0, 0], self.cut_sq[0, 1], self.prob, self.rng)
        self.md_steps += 1

    def _resort(self):
        A.apply_pbc(self.solvent, self.edges)
        A.apply_pbc(self.colloids, self.edges)
        self.solvent.sort(self.cells)
        self.neigh.update_list(self.colloids, self.solvent, self.max_cut + self.skin, self.cells,
                               self.solvent_colloid_lj)
        self.solvent.copy_pos_old()
        self.colloids.copy_pos_old()

    def interval(self):
        """md_loop followed by the MPCD part, programs/single_dimer_pbc.f90:303-443."""
        self.md_loop()
        self.mpcd()

    def md_loop(self, want_energy: bool = False):
        """The N_MD steps of md_loop (programs/single_dimer_pbc.f90:306-384);
        with want_energy the last step's e1, e2 are kept (the thermo sample)."""
        for j in range(self.N_MD):
            self.md_step(want_energy=want_energy and j == self.N_MD - 1)

    def thermo(self):
        """The thermo sample taken after md_loop (programs/single_dimer_pbc.f90:388-396):
        temperature, potential e1 + e2, kinetic, internal energy and v_com."""
        o = self.observables()
        pot = self.e1 + self.e2
        return dict(temperature=o["temperature"], potential=pot, kinetic=o["kinetic"],
                    internal=pot + o["kinetic"], v_com=o["v_com"])

    def mpcd(self):
        """The MPCD part of an interval (programs/single_dimer_pbc.f90:399-426)."""
        self.cells.random_shift(self.rng)
        self._resort()
        A.simple_mpcd_step(self.solvent, self.cells, self.rng, thermostat=self.do_thermostat, T=self.T,
                           hydro=self.do_hydro)
        if self.bulk_rmpcd:
            A.bulk_reaction(self.solvent, self.cells, 2, 1, self.bulk_rate, self.tau, self.rng)
        else:
            A.refuel(self.solvent, self.colloids, self.edges, int(self.L[0]))

    def observables(self):
        """temperature, kinetic energy, v_com and n_solvent of the interval."""
        te = A.compute_temperature(self.solvent, self.cells)
        cv = self.colloids.vel
        vs = A.velocity_sums(self.solvent)
        kin = (self.mass[0] * (cv[0] ** 2).sum() + self.mass[1] * (cv[1] ** 2).sum()) / 2 + vs[0] / 2
        vcom = (vs[1:] + self.mass[0] * cv[0] + self.mass[1] * cv[1]) / (self.N + self.mass[0] + self.mass[1])
        return dict(temperature=te, kinetic=kin, v_com=vcom, n_solvent=A.n_solvent(self.solvent, 2))


class DimerBatch:
    """Many independent :class:`SingleDimerPBC` systems advanced together by
    ``rmpcd_dimer_batch_run``: each interval is one captured CUDA graph whose
    kernels cover every replica.  The drivers passed in provide the set-up
    (positions, velocities, sort, list, initial forces); :meth:`scatter` copies
    a replica back into its driver's handles, after which the driver's own
    methods (observables, further intervals) continue from there.

    All drivers must share N_MD, tau, the dimer and the LJ tables, start at the
    same RNG step and use the same solvent precision; boxes and seeds may differ.
    """

    def __init__(self, dimers, use_graph: bool = True):
        self.dimers = list(dimers)
        d0 = self.dimers[0]
        R = len(self.dimers)
        prm = DIMER_PARAMS()
        prm.tau, prm.N_MD, prm.bond, prm.skin = d0.tau, d0.N_MD, d0.d, d0.skin
        prm.list_radius = d0.max_cut + d0.skin
        prm.prob = d0.prob
        prm.cut_sq_C, prm.cut_sq_N = float(d0.cut_sq[0, 0]), float(d0.cut_sq[0, 1])
        prm.vv_mass[0], prm.vv_mass[1] = float(d0.mass[0]), float(d0.mass[1])
        prm.thermostat, prm.hydro, prm.T = int(bool(d0.do_thermostat)), int(bool(d0.do_hydro)), float(d0.T)
        for d in self.dimers:
            if d.N_MD != d0.N_MD or d.tau != d0.tau or d.bulk_rmpcd:
                raise ValueError("DimerBatch: replicas must share N_MD and tau and use refuel")
        def hv(xs):
            return (C.c_void_p * R)(*[x.handle.value for x in xs])

        self._extra0 = [d.n_extra_sorting for d in self.dimers]
        rngs = (RNG * R)(*[RNG(d.rng.seed, d.rng.step) for d in self.dimers])
        self._h = C.c_void_p()
        call("rmpcd_dimer_batch_create", C.byref(self._h), R, hv([d.solvent for d in self.dimers]),
             hv([d.colloids for d in self.dimers]), hv([d.cells for d in self.dimers]),
             hv([d.neigh for d in self.dimers]), rngs, C.byref(d0.solvent_colloid_lj.struct),
             C.byref(d0.colloid_lj.struct), C.byref(prm))
        call("rmpcd_dimer_batch_set_graph", self._h, int(bool(use_graph)))
        self.R = R

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().rmpcd_dimer_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def n_solvent(self) -> int:
        n = C.c_longlong()
        call("rmpcd_dimer_batch_info", self._h, None, C.byref(n), None)
        return int(n.value)

    def run(self, n_intervals: int) -> None:
        call("rmpcd_dimer_batch_run", self._h, int(n_intervals))

    def n_extra_sorting(self) -> np.ndarray:
        out = np.zeros(self.R, np.int32)
        call("rmpcd_dimer_batch_info", self._h, None, None, out.ctypes.data_as(C.POINTER(C.c_int)))
        return out

    @staticmethod
    def shapes(precision: int = A.FP32) -> list[dict]:
        """The engine shapes rmpcd_dimer_batch_autotune chooses from."""
        n = C.c_int()
        call("rmpcd_dimer_batch_shapes", int(precision), C.byref(n))
        out = []
        for k in range(n.value):
            v = [C.c_int() for _ in range(6)]
            call("rmpcd_dimer_batch_shape_info", int(precision), k, *[C.byref(x) for x in v])
            out.append(dict(particles_per_tile=v[0].value, per_thread_begin=v[1].value,
                            per_thread_end=v[2].value, blocks_per_sm=v[3].value,
                            list_entries_per_thread=v[4].value, colloid_block_first=bool(v[5].value)))
        return out

    @property
    def shape(self) -> int:
        s = C.c_int()
        call("rmpcd_dimer_batch_get_shape", self._h, C.byref(s))
        return s.value

    @shape.setter
    def shape(self, k: int) -> None:
        call("rmpcd_dimer_batch_set_shape", self._h, int(k))

    def autotune(self, n_intervals: int = 1) -> dict:
        """rmpcd_dimer_batch_autotune: the engine shapes it tries each run
        1 + n_intervals real intervals of this batch (the results do not
        depend on the shape) and the fastest is kept; a batch of a kind
        already tuned takes the remembered choice without running.  Returns
        the choice, the milliseconds per interval of each shape (-1 when not
        run or remembered) and the intervals every replica advanced by."""
        n = C.c_int()
        call("rmpcd_dimer_batch_shapes", int(self.dimers[0].solvent.precision), C.byref(n))
        ms = (C.c_float * n.value)()
        best, ran = C.c_int(), C.c_int()
        call("rmpcd_dimer_batch_autotune", self._h, int(n_intervals), C.byref(best), ms, C.byref(ran))
        return dict(best=best.value, ms_per_interval=[round(float(x), 4) for x in ms], intervals_run=ran.value)

    def scatter(self, r: int, dimer: SingleDimerPBC | None = None) -> SingleDimerPBC:
        """Copy replica r into the handles of ``dimer`` (its own driver by default)."""
        d = dimer if dimer is not None else self.dimers[r]
        call("rmpcd_dimer_batch_scatter", self._h, int(r), d.solvent.handle, d.colloids.handle, d.cells.handle,
             d.neigh.handle, d.rng.ptr)
        d.n_extra_sorting = self._extra0[r] + int(self.n_extra_sorting()[r])
        return d


PI_3141 = float(np.float32(3.141))  # default-real constants of n_colloids_pbc
PI_3142 = float(np.float32(3.142))
COLLOID_PLACE_STEP = 0xFFFFFFFFFFFFFFFF  # RNG step of the colloid placement draws
PLACE_STREAM = 5


def place_colloids(uniform2, seed, n, edges, min_dist):
    """Uniform colloid positions with the program's rejection of pairs closer
    than min_dist (programs/n_colloids_pbc.f90:193-210).  Attempt k draws
    uniform2(seed, COLLOID_PLACE_STEP, k, PLACE, 0) for x, y and (.., 1) for z."""
    edges = np.asarray(edges, np.float64)
    pos = np.zeros((n, 3))
    i = k = 0
    while i < n:
        u0, u1 = uniform2(seed, COLLOID_PLACE_STEP, k, PLACE_STREAM, 0)
        u2, _ = uniform2(seed, COLLOID_PLACE_STEP, k, PLACE_STREAM, 1)
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
    """programs/n_colloids_pbc.f90 on the GPU: passive LJ colloids in an SRD
    fluid with lazy, cell-wise solvent streaming.  Only the solvent in cells
    flagged by the neighbor list (is_md) is advanced every MD step; the other
    cells are streamed in one step of the accumulated time before each sort.

    ``volume_correction`` subtracts the colloid volume from the solvent count
    as the program does (N = rho L^3 - int(rho 4*3.142/3 sigma^3 N_colloids)).
    """

    def __init__(self, L=(32, 32, 32), rho=10, T=1.0 / 3.0, T_final=None, tau=1.0, N_MD=100, N_colloids=10,
                 sigma=3.0, epsilon=1.0, epsilon_colloids=1.0, do_hydro=True, do_thermostat=False, seed=1,
                 skin=0.8, list_capacity=None, precision=A.FP64, volume_correction=True):
        self._init_kwargs = dict(
            L=[int(x) for x in L], rho=rho, T=T, T_final=T_final, tau=tau, N_MD=N_MD, N_colloids=N_colloids,
            sigma=sigma, epsilon=epsilon, epsilon_colloids=epsilon_colloids, do_hydro=do_hydro,
            do_thermostat=do_thermostat, seed=int(seed), skin=skin, list_capacity=list_capacity,
            precision=precision, volume_correction=volume_correction)
        self.L = np.asarray(L, dtype=np.int32)
        self.rho, self.T_init, self.tau, self.N_MD = rho, T, tau, N_MD
        self.T_final = T if T_final is None else T_final
        self.dt = tau / N_MD
        self.do_hydro, self.do_thermostat = do_hydro, do_thermostat
        self.skin = skin
        vol = int(rho * 4 * PI_3142 / 3 * sigma ** 3 * N_colloids) if volume_correction else 0
        self.N = int(rho * int(self.L.prod())) - vol
        if self.N <= 0:
            raise ValueError("Not enough volume available for solvent")
        self.mass = rho * sigma ** 3 * 4 * PI_3141 / 3
        sigma_cut = sigma * 2.0 ** (1.0 / 6.0)
        self.solvent_colloid_lj = A.LJParams([[epsilon]], [[sigma]], [[sigma_cut]])
        self.colloid_lj = A.LJParams([[epsilon_colloids]], [[2 * sigma]], [[2 * (3 * sigma)]])
        self.rng = A.Rng(seed)
        self.colloids = A.ParticleSystem(N_colloids, 1, [self.mass])
        self.colloids.species = 1
        self.vv_mass = np.full(N_colloids, self.mass)
        self.solvent = A.ParticleSystem(self.N, 1, None, precision)
        self.solvent.maxwell(T, seed)
        self.solvent.species = 1
        self.cells = A.CellSystem(self.L, 1.0)
        self.edges = self.cells.edges
        self.colloids.pos = place_colloids(A.rng_uniform2, seed, N_colloids, self.edges, 2 * sigma)
        self.solvent.random_placement(self.edges, self.colloids, self.solvent_colloid_lj, seed)
        self.solvent.sort(self.cells)
        self.radius = sigma_cut + skin
        cap = list_capacity if list_capacity is not None else int(250 * (sigma_cut + skin) ** 2)
        self.neigh = A.NeighborList(N_colloids, cap)
        self.neigh.make_stencil(self.cells, self.radius)
        self.neigh.update_list(self.colloids, self.solvent, self.radius, self.cells)
        self.e1 = A.compute_force(self.colloids, self.solvent, self.neigh, self.edges, self.solvent_colloid_lj)
        self.e2 = A.compute_force_n2(self.colloids, self.edges, self.colloid_lj)
        self.solvent.copy_force_old()
        self.colloids.copy_force_old()
        self.solvent.copy_pos_old()
        self.colloids.copy_pos_old()
        self.n_extra_sorting = 0
        self.t = 0          # MD steps of the current loop (thermalisation or production)
        self.last_sort = 0  # value of t at the last sort

    def _catch_up_and_sort(self):
        """Stream the non-MD cells over the time since the last sort, wrap,
        sort, rebuild the list (programs/n_colloids_pbc.f90:230-241)."""
        s, c, dtl = self.solvent, self.colloids, (self.t - self.last_sort) * self.dt
        A.cell_md_pos(self.cells, s, dtl, False)
        A.cell_md_vel(self.cells, s, dtl, False)
        A.apply_pbc(s, self.edges)
        A.apply_pbc(c, self.edges)
        s.sort(self.cells)
        self.last_sort = self.t
        self.neigh.update_list(c, s, self.radius, self.cells)
        s.copy_pos_old()
        c.copy_pos_old()

    def md_step(self, want_energy=False):
        """One pass of md_loop, programs/n_colloids_pbc.f90:221-254.  The
        energies e1, e2 are only read after the last MD step of an interval
        (the thermo output), so they are computed there only."""
        s, c, dt = self.solvent, self.colloids, self.dt
        self.t += 1
        A.cell_md_pos(self.cells, s, dt, True)
        A.colloid_vv_pos(c, dt, self.vv_mass)
        so_max = A.cell_maximum_displacement(self.cells, s, dt * (self.t - self.last_sort))
        co_max = c.maximum_displacement()
        if (co_max >= self.skin * 0.1) or (so_max >= self.skin * 0.9):
            self._catch_up_and_sort()
            self.n_extra_sorting += 1
        s.switch_force()
        c.switch_force()
        s.zero_force()
        c.zero_force()
        e1 = A.compute_force(c, s, self.neigh, self.edges, self.solvent_colloid_lj, energy=want_energy)
        e2 = A.compute_force_n2(c, self.edges, self.colloid_lj, energy=want_energy)
        if want_energy:
            self.e1, self.e2 = e1, e2
        A.cell_md_vel(self.cells, s, dt, True)
        A.colloid_vv_vel(c, dt, self.vv_mass)

    def interval(self, thermostat: bool, T: float, rescale: bool = False):
        """md_loop followed by the MPCD part (programs/n_colloids_pbc.f90:256-276, :304-324)."""
        for j in range(self.N_MD):
            self.md_step(want_energy=(j == self.N_MD - 1))
        self.cells.random_shift(self.rng)
        self._catch_up_and_sort()
        A.simple_mpcd_step(self.solvent, self.cells, self.rng, thermostat=thermostat, T=T, hydro=self.do_hydro)
        if rescale:
            A.rescale_cells(self.solvent, self.cells, self.rng, self.T_init)

    def _native(self, n, thermostat, Ts, rescale_every):
        """n intervals through rmpcd_ncolloids_run (the same calls, in C)."""
        prm = NCOLLOIDS_PARAMS(self.tau, self.N_MD, self.skin, self.radius, self.mass, int(bool(self.do_hydro)))
        st = NCOLLOIDS_STATE(self.t, self.last_sort, self.n_extra_sorting, self.e1 or 0.0, self.e2 or 0.0)
        T = np.ascontiguousarray(Ts, dtype=np.float64)
        call("rmpcd_ncolloids_run", self.solvent.handle, self.colloids.handle, self.cells.handle, self.neigh.handle,
             C.byref(self.solvent_colloid_lj.struct), C.byref(self.colloid_lj.struct), self.rng.ptr, C.byref(prm),
             int(n), int(bool(thermostat)), T.ctypes.data_as(C.POINTER(C.c_double)), 1, int(rescale_every),
             float(self.T_init), C.byref(st))
        self.t, self.last_sort, self.n_extra_sorting = st.t, st.last_sort, st.n_extra_sorting
        self.e1, self.e2 = st.e1, st.e2

    def thermalise(self, n_loops, native=True):
        """The thermostatted loop: MPC-AT at T, cell rescaling every 10 intervals."""
        if native:
            self._native(n_loops, True, [self.T_init] * max(1, n_loops), 10)
        else:
            for i in range(1, n_loops + 1):
                self.interval(True, self.T_init, rescale=(i % 10 == 0))
        self.t = self.last_sort = 0

    def run(self, n_loops, native=True):
        """The production loop with the temperature ramp T_init -> T_final."""
        Ts = [self.T_init + (i - 1) * (self.T_final - self.T_init) / max(1, n_loops - 1) for i in range(1, n_loops + 1)]
        if native:
            self._native(n_loops, self.do_thermostat, Ts or [self.T_init], 0)
        else:
            for T in Ts:
                self.interval(self.do_thermostat, T)


def bulk_fluid(L, rho=10, T=1.0 / 3.0, tau=1.0, n_intervals=200, seed=1, precision=A.FP64, alpha=None):
    """Bulk SRD fluid: Maxwell velocities, uniform positions, sorted once,
    then n_intervals of collide -> stream -> shift -> sort (fused)."""
    L = np.asarray(L, dtype=np.int32)
    N = int(rho * L.prod())
    cells = A.CellSystem(L, 1.0)
    p = A.ParticleSystem(N, 1, None, precision)
    p.random_placement(cells.edges, seed=seed)
    p.maxwell(T, seed)
    p.species = 1
    rng = A.Rng(seed)
    cells.random_shift(rng)
    p.sort(cells)
    A.bulk_run(p, cells, rng, tau, n_intervals, alpha=alpha)
    return p, cells, rng
