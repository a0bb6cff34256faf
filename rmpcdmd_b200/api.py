"""Python mirror of the reference's Fortran module surface over the C ABI.

Type and procedure names follow RMPCDMD (src/rmpcdmd_module.f90.in):
``cell_system_t`` -> :class:`CellSystem`, ``particle_system_t`` ->
:class:`ParticleSystem`, ``neighbor_list_t`` -> :class:`NeighborList`,
``lj_params_t`` -> :class:`LJParams`, and the free procedures
(``simple_mpcd_step``, ``md_pos``, ``compute_force``...) as functions.

Arrays cross the boundary in the reference layout: 3-vectors as numpy arrays
of shape (N, 3) in C order, which is the Fortran (3, N) column-major layout;
cell starts, list entries and id_to_idx are 1-based.  Every call goes to the
CUDA library; errors raise :class:`RmpcdError` with the reference's message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import LJ, RIGID_STATE, RNG, RmpcdError, call, lib

FP64 = 64
FP32 = 32
PERIODIC_BC = 1
BOUNCE_BACK_BC = 2
SPECULAR_BC = 3

# bit positions, src/common.f90:49-55
REAC_BIT = 1
MD_BIT = 2
WALL_BIT = 3
PAST_MD_BIT = 4
CATALYZED_BIT = 6

__all__ = [
    "FP64", "FP32", "PERIODIC_BC", "BOUNCE_BACK_BC", "SPECULAR_BC", "REAC_BIT", "MD_BIT", "WALL_BIT",
    "PAST_MD_BIT", "CATALYZED_BIT", "RmpcdError", "Rng", "LJParams", "CellSystem", "ParticleSystem",
    "NeighborList", "compact_p_to_h", "compact_h_to_p", "simple_mpcd_step", "wall_mpcd_step",
    "compute_temperature", "rescale_cells", "mpcd_stream_periodic", "mpcd_stream_xforce_yzwall",
    "mpcd_stream_nogravity_zwall", "bulk_reaction", "bulk_reaction_endothermic", "md_pos", "md_vel", "cell_md_pos", "cell_md_vel",
    "cell_md_pos_ywall", "cell_md_pos_zwall", "apply_pbc", "rattle_dimer_pos", "rattle_dimer_vel",
    "colloid_vv_pos", "colloid_vv_vel", "compute_force", "compute_force_n2", "flag_particles_nl",
    "change_species", "refuel", "n_solvent", "cylindrical_shell_histogram", "velocity_sums",
    "bulk_run", "synchronize", "get_status", "Timers", "rng_uniform2",
]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _d3(x) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(3))
    return a


def _i3(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32).reshape(3))


def synchronize() -> None:
    call("rmpcd_synchronize")


def set_device(device: int) -> None:
    """Select this process's GPU before any other call (one process per GPU)."""
    call("rmpcd_set_device", int(device))


__all__.append("set_device")


def get_status() -> None:
    """Synchronize and raise if a kernel reported an error."""
    call("rmpcd_get_status")


class Rng:
    """Counter-based generator state {seed, step} (replaces threefry_rng_t state(:))."""

    def __init__(self, seed: int, step: int = 0):
        self._s = RNG(seed & 0xFFFFFFFFFFFFFFFF, step)

    @property
    def seed(self) -> int:
        return int(self._s.seed)

    @property
    def step(self) -> int:
        return int(self._s.step)

    @step.setter
    def step(self, v: int) -> None:
        self._s.step = v

    @seed.setter
    def seed(self, v: int) -> None:
        self._s.seed = v & 0xFFFFFFFFFFFFFFFF

    @property
    def ptr(self):
        return C.byref(self._s)


def rng_uniform2(seed: int, step: int, index: int, stream: int, attempt: int = 0) -> tuple[float, float]:
    out = np.zeros(2)
    call("rmpcd_rng_uniform2", C.c_uint64(seed), C.c_uint64(step), index, stream, attempt, _dp(out))
    return float(out[0]), float(out[1])


class LJParams:
    """lj_params_t, src/interaction.f90:23-80 (tables indexed (solvent, colloid))."""

    def __init__(self, epsilon, sigma, cut):
        eps = np.asarray(epsilon, dtype=np.float64)
        sig = np.asarray(sigma, dtype=np.float64)
        cut_ = np.asarray(cut, dtype=np.float64)
        if eps.ndim == 0:
            eps, sig, cut_ = eps.reshape(1, 1), sig.reshape(1, 1), cut_.reshape(1, 1)
        if not (eps.shape == sig.shape == cut_.shape):
            raise RmpcdError(1, "lj_params_init", "unequal sizes for arguments to lj_params_init")
        n1, n2 = eps.shape
        self.struct = LJ()
        fe = np.ascontiguousarray(eps.T.reshape(-1))
        fs = np.ascontiguousarray(sig.T.reshape(-1))
        fc = np.ascontiguousarray(cut_.T.reshape(-1))
        call("rmpcd_lj_init", C.byref(self.struct), n1, n2, _dp(fe), _dp(fs), _dp(fc))
        self.n1, self.n2 = n1, n2

    def _table(self, name):
        a = np.array(getattr(self.struct, name)[: self.n1 * self.n2])
        return a.reshape(self.n2, self.n1).T

    @property
    def epsilon(self):
        return self._table("epsilon")

    @property
    def sigma(self):
        return self._table("sigma")

    @property
    def cut(self):
        return self._table("cut")

    @property
    def cut_sq(self):
        return self._table("cut_sq")

    @property
    def cut_energy(self):
        return self._table("cut_energy")

    @property
    def ptr(self):
        return C.byref(self.struct)


def compact_p_to_h(p, M) -> int:
    """compact_p_to_h, src/hilbert.f90:241-271 (0-based index)."""
    h = C.c_int(0)
    pp, mm = _i3(p), _i3(M)
    call("rmpcd_compact_p_to_h", _ip(pp), _ip(mm), C.byref(h))
    return h.value


def compact_h_to_p(h, M) -> np.ndarray:
    """compact_h_to_p, src/hilbert.f90:273-307."""
    out = np.zeros(3, dtype=np.int32)
    mm = _i3(M)
    call("rmpcd_compact_h_to_p", int(h), _ip(mm), _ip(out))
    return out


class CellSystem:
    """cell_system_t, src/cell_system.f90:20-41."""

    def __init__(self, L, a: float = 1.0, has_walls: bool = False):
        self._h = C.c_void_p()
        call("rmpcd_cells_init", C.byref(self._h), _ip(_i3(L)), float(a), int(bool(has_walls)))
        Lo = np.zeros(3, np.int32)
        Mo = np.zeros(3, np.int32)
        S = C.c_int(0)
        e = np.zeros(3)
        call("rmpcd_cells_info", self._h, _ip(Lo), _ip(Mo), C.byref(S), _dp(e))
        self.L, self.M, self.N, self.edges = Lo, Mo, S.value, e
        self.a = float(a)
        self.has_walls = bool(has_walls)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().rmpcd_cells_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def origin(self) -> np.ndarray:
        o = np.zeros(3)
        call("rmpcd_cells_get_origin", self._h, _dp(o))
        return o

    @origin.setter
    def origin(self, v) -> None:
        call("rmpcd_cells_set_origin", self._h, _dp(_d3(v)))

    def set_bc(self, bc) -> None:
        call("rmpcd_cells_set_bc", self._h, _ip(_i3(bc)))

    def set_max_v(self, v: float) -> None:
        call("rmpcd_cells_set_max_v", self._h, float(v))

    def random_shift(self, rng: Rng) -> None:
        call("rmpcd_cells_random_shift", self._h, rng.ptr)

    def count_particles(self, p: "ParticleSystem") -> None:
        call("rmpcd_cells_count_particles", self._h, p.handle)

    def sort_particles(self, position_old: "ParticleSystem", position_new: "ParticleSystem") -> None:
        """sort_particles, src/cell_system.f90:131-151: the positions of
        position_old, in cell order, become those of position_new; the starts
        advance by the counts (call count_particles before using them)."""
        call("rmpcd_cells_sort_particles", self._h, position_old.handle, position_new.handle)

    @property
    def cell_count(self) -> np.ndarray:
        a = np.zeros(self.N, np.int32)
        call("rmpcd_cells_download_count", self._h, _ip(a))
        return a

    @property
    def cell_start(self) -> np.ndarray:
        a = np.zeros(self.N, np.int32)
        call("rmpcd_cells_download_start", self._h, _ip(a))
        return a

    @property
    def is_md(self) -> np.ndarray:
        a = np.zeros(self.N, np.uint8)
        call("rmpcd_cells_download_is_md", self._h, a.ctypes.data_as(C.POINTER(C.c_ubyte)))
        return a.astype(bool)

    @is_md.setter
    def is_md(self, v) -> None:
        a = np.ascontiguousarray(np.asarray(v, dtype=np.uint8).reshape(self.N))
        call("rmpcd_cells_upload_is_md", self._h, a.ctypes.data_as(C.POINTER(C.c_ubyte)))

    @property
    def is_reac(self) -> np.ndarray:
        a = np.zeros(self.N, np.uint8)
        call("rmpcd_cells_download_is_reac", self._h, a.ctypes.data_as(C.POINTER(C.c_ubyte)))
        return a.astype(bool)

    @is_reac.setter
    def is_reac(self, v) -> None:
        a = np.ascontiguousarray(np.asarray(v, dtype=np.uint8).reshape(self.N))
        call("rmpcd_cells_upload_is_reac", self._h, a.ctypes.data_as(C.POINTER(C.c_ubyte)))

    def set_axes(self, axes) -> None:
        """Inject one SRD rotation axis per slot (shape (S, 3)); None restores Philox axes."""
        if axes is None:
            call("rmpcd_cells_set_axes", self._h, None)
            return
        a = np.ascontiguousarray(np.asarray(axes, dtype=np.float64).reshape(self.N, 3))
        call("rmpcd_cells_set_axes", self._h, _dp(a))


_REAL3 = ("pos", "pos_old", "vel", "force", "force_old", "pos_rattle")
_INT3 = ("image",)
_INT1 = ("id", "species", "flags", "id_to_idx")


class ParticleSystem:
    """particle_system_t, src/particle_system.f90:22-77 (data resident on the GPU)."""

    def __init__(self, Nmax: int, n_species: int = 1, mass=None, precision: int = FP64):
        self._h = C.c_void_p()
        m = None
        if mass is not None:
            m = np.ascontiguousarray(np.asarray(mass, dtype=np.float64).reshape(-1))
        call("rmpcd_particles_init", C.byref(self._h), int(Nmax), int(n_species),
             _dp(m) if m is not None else None, int(precision))
        self.Nmax = int(Nmax)
        self.n_species = int(n_species)
        self.mass = m
        self.precision = int(precision)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().rmpcd_particles_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def count_nonfinite(self) -> int:
        """Particles with a NaN or infinite position or velocity component."""
        n = C.c_longlong(0)
        call("rmpcd_particles_count_nonfinite", self._h, C.byref(n))
        return n.value

    def download(self, field: str) -> np.ndarray:
        if field in _REAL3:
            a = np.zeros((self.Nmax, 3))
        elif field in _INT3:
            a = np.zeros((self.Nmax, 3), np.int32)
        elif field in _INT1:
            a = np.zeros(self.Nmax, np.int32)
        else:
            raise RmpcdError(1, "download", f"unknown particle field '{field}'")
        call("rmpcd_particles_download", self._h, field.encode(), a.ctypes.data_as(C.c_void_p))
        return a

    def upload(self, field: str, value) -> None:
        if field in _REAL3:
            a = np.ascontiguousarray(np.broadcast_to(np.asarray(value, np.float64), (self.Nmax, 3)))
        elif field in _INT3:
            a = np.ascontiguousarray(np.broadcast_to(np.asarray(value, np.int32), (self.Nmax, 3)))
        elif field in ("id", "species", "flags"):
            a = np.ascontiguousarray(np.broadcast_to(np.asarray(value, np.int32), (self.Nmax,)))
        else:
            raise RmpcdError(1, "upload", f"unknown or read-only particle field '{field}'")
        call("rmpcd_particles_upload", self._h, field.encode(), a.ctypes.data_as(C.c_void_p))

    # convenience properties in the reference's names
    pos = property(lambda s: s.download("pos"), lambda s, v: s.upload("pos", v))
    pos_old = property(lambda s: s.download("pos_old"), lambda s, v: s.upload("pos_old", v))
    vel = property(lambda s: s.download("vel"), lambda s, v: s.upload("vel", v))
    force = property(lambda s: s.download("force"), lambda s, v: s.upload("force", v))
    force_old = property(lambda s: s.download("force_old"), lambda s, v: s.upload("force_old", v))
    image = property(lambda s: s.download("image"), lambda s, v: s.upload("image", v))
    id = property(lambda s: s.download("id"), lambda s, v: s.upload("id", v))
    species = property(lambda s: s.download("species"), lambda s, v: s.upload("species", v))
    flags = property(lambda s: s.download("flags"), lambda s, v: s.upload("flags", v))
    id_to_idx = property(lambda s: s.download("id_to_idx"))

    def sort(self, cells: CellSystem) -> None:
        call("rmpcd_particles_sort", self._h, cells.handle)

    def maximum_displacement(self) -> float:
        r = C.c_double(0)
        call("rmpcd_particles_maximum_displacement", self._h, C.byref(r))
        return r.value

    def random_placement(self, L, other: "ParticleSystem | None" = None, lj_params: LJParams | None = None,
                         seed: "int | Rng" = 0) -> None:
        """random_placement, src/particle_system.f90:250-302; ``seed`` is a
        seed or the Rng whose seed keys the draws (the reference's state(1))."""
        state = seed if isinstance(seed, Rng) else Rng(seed)
        call("rmpcd_particles_random_placement", self._h, _dp(_d3(L)), other.handle if other else None,
             lj_params.ptr if lj_params else None, state.ptr)

    def maxwell(self, T: float, seed: int) -> None:
        call("rmpcd_particles_maxwell", self._h, float(T), C.c_uint64(seed))

    def switch_force(self) -> None:
        call("rmpcd_particles_switch_force", self._h)

    def zero_force(self) -> None:
        call("rmpcd_particles_zero_force", self._h)

    def copy_pos_old(self) -> None:
        call("rmpcd_particles_copy_pos_old", self._h)

    def copy_pos_rattle(self) -> None:
        call("rmpcd_particles_copy_pos_rattle", self._h)

    def copy_force_old(self) -> None:
        call("rmpcd_particles_copy_force_old", self._h)

    def set_gauss(self, gauss) -> None:
        if gauss is None:
            call("rmpcd_particles_set_gauss", self._h, None)
            return
        a = np.ascontiguousarray(np.asarray(gauss, dtype=np.float64).reshape(self.Nmax, 3))
        call("rmpcd_particles_set_gauss", self._h, _dp(a))


def cell_maximum_displacement(cells: CellSystem, p: ParticleSystem, delta_t: float) -> float:
    r = C.c_double(0)
    call("rmpcd_cell_maximum_displacement", cells.handle, p.handle, float(delta_t), C.byref(r))
    return r.value


__all__.append("cell_maximum_displacement")


class NeighborList:
    """neighbor_list_t, src/neighbor_list.f90:23-34."""

    def __init__(self, Npoints: int, Nmax: int):
        self._h = C.c_void_p()
        call("rmpcd_nlist_init", C.byref(self._h), int(Npoints), int(Nmax))
        self.Npoints, self.Nmax = int(Npoints), int(Nmax)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().rmpcd_nlist_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def make_stencil(self, cells: CellSystem, cut: float) -> None:
        call("rmpcd_nlist_make_stencil", self._h, cells.handle, float(cut))

    @property
    def stencil_size(self) -> int:
        n = C.c_int(0)
        call("rmpcd_nlist_stencil_size", self._h, C.byref(n))
        return n.value

    def update_list(self, system1: ParticleSystem, system2: ParticleSystem, radius: float, cells: CellSystem,
                    lj: LJParams | None = None) -> None:
        call("rmpcd_nlist_update", self._h, system1.handle, system2.handle, float(radius), cells.handle,
             lj.ptr if lj else None)

    def download(self) -> tuple[np.ndarray, np.ndarray]:
        """(list, n): list has shape (Npoints, Nmax) holding 1-based indices (0 past n)."""
        lst = np.zeros((self.Npoints, self.Nmax), np.int32)
        n = np.zeros(self.Npoints, np.int32)
        call("rmpcd_nlist_download", self._h, _ip(lst), _ip(n))
        return lst, n


def simple_mpcd_step(particles: ParticleSystem, cells: CellSystem, state: Rng, alpha: float | None = None,
                     thermostat: bool = False, T: float | None = None, hydro: bool = True) -> None:
    """simple_mpcd_step, src/mpcd.f90:71-183."""
    if thermostat and T is None:
        raise RmpcdError(4, "simple_mpcd_step", "no temperature given for thermostat in simple_mpcd_step")
    call("rmpcd_simple_mpcd_step", particles.handle, cells.handle, state.ptr, int(alpha is not None),
         float(alpha or 0.0), int(bool(thermostat)), float(T or 0.0), int(bool(hydro)))


def wall_mpcd_step(particles: ParticleSystem, cells: CellSystem, state: Rng, wall_temperature=None, wall_v=None,
                   wall_n=None, thermostat: bool = False, bulk_temperature: float | None = None,
                   alpha: float | None = None, keep_cell_v: bool = True) -> None:
    """wall_mpcd_step, src/mpcd.f90:193-337."""
    wt = None if wall_temperature is None else np.ascontiguousarray(np.asarray(wall_temperature, np.float64))
    wv = None if wall_v is None else np.ascontiguousarray(np.asarray(wall_v, np.float64).reshape(6))
    wn = None if wall_n is None else np.ascontiguousarray(np.asarray(wall_n, np.int32))
    if thermostat and bulk_temperature is None:
        raise RmpcdError(4, "wall_mpcd_step", "thermostat requested but no temperature given in wall_mpcd_step")
    call("rmpcd_wall_mpcd_step", particles.handle, cells.handle, state.ptr,
         _dp(wt) if wt is not None else None, _dp(wv) if wv is not None else None,
         _ip(wn) if wn is not None else None, int(bool(thermostat)), float(bulk_temperature or 0.0),
         int(alpha is not None), float(alpha or 0.0), int(bool(keep_cell_v)))


def compute_temperature(particles: ParticleSystem, cells: CellSystem) -> float:
    te = C.c_double(0)
    call("rmpcd_compute_temperature", particles.handle, cells.handle, C.byref(te))
    return te.value


def rescale_cells(particles: ParticleSystem, cells: CellSystem, state: Rng | None, T: float) -> None:
    call("rmpcd_rescale_cells", particles.handle, cells.handle, state.ptr if state is not None else None, float(T))


def mpcd_stream_periodic(particles: ParticleSystem, cells: CellSystem, dt: float) -> None:
    call("rmpcd_mpcd_stream_periodic", particles.handle, cells.handle, float(dt))


def mpcd_stream_xforce_yzwall(particles: ParticleSystem, cells: CellSystem, dt: float, g: float) -> None:
    call("rmpcd_mpcd_stream_xforce_yzwall", particles.handle, cells.handle, float(dt), float(g))


def mpcd_stream_nogravity_zwall(particles: ParticleSystem, cells: CellSystem, dt: float) -> None:
    call("rmpcd_mpcd_stream_nogravity_zwall", particles.handle, cells.handle, float(dt))


def bulk_reaction(p: ParticleSystem, c: CellSystem, frm: int, to: int, rate: float, tau: float, state: Rng) -> None:
    call("rmpcd_bulk_reaction", p.handle, c.handle, int(frm), int(to), float(rate), float(tau), state.ptr)


def bulk_reaction_endothermic(p: ParticleSystem, c: CellSystem, frm: int, to: int, rate: float, tau: float,
                              state: Rng, delta_u: float) -> None:
    """src/mpcd.f90:645-700 (argument order of the reference: ..., state, delta_u)."""
    call("rmpcd_bulk_reaction_endothermic", p.handle, c.handle, int(frm), int(to), float(rate), float(tau),
         state.ptr, float(delta_u))


def md_pos(particles: ParticleSystem, dt: float) -> None:
    call("rmpcd_md_pos", particles.handle, float(dt))


def md_vel(particles: ParticleSystem, dt: float) -> None:
    call("rmpcd_md_vel", particles.handle, float(dt))


def cell_md_pos(cells: CellSystem, particles: ParticleSystem, dt: float, md_flag: bool) -> None:
    call("rmpcd_cell_md_pos", cells.handle, particles.handle, float(dt), int(bool(md_flag)))


def cell_md_vel(cells: CellSystem, particles: ParticleSystem, dt: float, md_flag: bool) -> None:
    call("rmpcd_cell_md_vel", cells.handle, particles.handle, float(dt), int(bool(md_flag)))


def cell_md_pos_ywall(cells: CellSystem, particles: ParticleSystem, dt: float, md_flag: bool) -> None:
    call("rmpcd_cell_md_pos_ywall", cells.handle, particles.handle, float(dt), int(bool(md_flag)))


def cell_md_pos_zwall(cells: CellSystem, particles: ParticleSystem, dt: float, md_flag: bool) -> None:
    call("rmpcd_cell_md_pos_zwall", cells.handle, particles.handle, float(dt), int(bool(md_flag)))


def apply_pbc(particles: ParticleSystem, edges) -> None:
    call("rmpcd_apply_pbc", particles.handle, _dp(_d3(edges)))


def rattle_dimer_pos(p: ParticleSystem, d: float, dt: float, edges) -> None:
    call("rmpcd_rattle_dimer_pos", p.handle, float(d), float(dt), _dp(_d3(edges)))


def rattle_dimer_vel(p: ParticleSystem, d: float, dt: float, edges) -> None:
    call("rmpcd_rattle_dimer_vel", p.handle, float(d), float(dt), _dp(_d3(edges)))


def _links(links, distances):
    lk = np.ascontiguousarray(links, np.int32).reshape(-1, 2)
    d = np.ascontiguousarray(distances, np.float64).reshape(-1)
    if len(lk) != len(d):
        raise ValueError("one distance per link")
    return lk, d


def rattle_body_pos(p: ParticleSystem, links, distances, dt: float, edges, precision: float) -> int:
    """src/md.f90:321-408.  links: (n_link, 2) 1-based particle numbers (the
    reference's links(2, n_link)).  Returns the reference's rattle_i at exit
    (1001 when 1000 sweeps did not converge)."""
    lk, d = _links(links, distances)
    it = C.c_int(0)
    call("rmpcd_rattle_body_pos", p.handle, _ip(lk), _dp(d), len(d), float(dt), _dp(_d3(edges)), float(precision),
         C.byref(it))
    return it.value


def rattle_body_vel(p: ParticleSystem, links, distances, dt: float, edges, precision: float) -> int:
    """src/md.f90:410-480."""
    lk, d = _links(links, distances)
    it = C.c_int(0)
    call("rmpcd_rattle_body_vel", p.handle, _ip(lk), _dp(d), len(d), float(dt), _dp(_d3(edges)), float(precision),
         C.byref(it))
    return it.value


def elastic_network(p: ParticleSystem, links, distances, k: float, edges) -> float:
    """src/md.f90:516-544: adds the link forces to force, returns the energy."""
    lk, d = _links(links, distances)
    e = C.c_double(0)
    call("rmpcd_elastic_network", p.handle, _ip(lk), _dp(d), len(d), float(k), _dp(_d3(edges)), C.byref(e))
    return e.value


class RigidBody:
    """rigid_body_t (src/md.f90:40-58): init, compute_force_torque, vv1, vv2
    on the beads i_start..i_stop (1-based) of an FP64 particle system; the
    state lives on the device (``state()`` reads it)."""

    def __init__(self, p: ParticleSystem, i_start: int, i_stop: int, edges):
        h = C.c_void_p()
        call("rmpcd_rigid_body_init", C.byref(h), p.handle, int(i_start), int(i_stop), _dp(_d3(edges)))
        self._h = h
        self.i_start, self.i_stop = int(i_start), int(i_stop)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                call("rmpcd_rigid_body_destroy", h)
            except Exception:
                pass
            self._h = None

    def state(self) -> dict:
        st = RIGID_STATE()
        call("rmpcd_rigid_body_get", self._h, C.byref(st), None)
        return {n: (getattr(st, n) if n == "mass" else np.array(getattr(st, n)[:])) for n, _ in st._fields_}

    def pos_body(self) -> np.ndarray:
        st = RIGID_STATE()
        out = np.zeros((self.i_stop - self.i_start + 1, 3))
        call("rmpcd_rigid_body_get", self._h, C.byref(st), _dp(out))
        return out

    def set_state(self, **fields) -> None:
        st = RIGID_STATE()
        call("rmpcd_rigid_body_get", self._h, C.byref(st), None)
        for n, v in fields.items():
            if n == "mass":
                st.mass = float(v)
            else:
                arr = getattr(st, n)
                for k, x in enumerate(np.asarray(v, np.float64).reshape(-1)):
                    arr[k] = x
        call("rmpcd_rigid_body_set", self._h, C.byref(st))

    def compute_force_torque(self, p: ParticleSystem) -> None:
        call("rmpcd_rigid_body_compute_force_torque", self._h, p.handle)

    def vv1(self, p: ParticleSystem, dt: float, treshold: float, edges) -> None:
        call("rmpcd_rigid_body_vv1", self._h, p.handle, float(dt), float(treshold), _dp(_d3(edges)))

    def vv2(self, p: ParticleSystem, dt: float) -> None:
        call("rmpcd_rigid_body_vv2", self._h, p.handle, float(dt))


__all__ += ["rattle_body_pos", "rattle_body_vel", "elastic_network", "RigidBody"]


def colloid_vv_pos(p: ParticleSystem, dt: float, mass) -> None:
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float64), (p.Nmax,)))
    call("rmpcd_colloid_vv_pos", p.handle, float(dt), _dp(m))


def colloid_vv_vel(p: ParticleSystem, dt: float, mass) -> None:
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float64), (p.Nmax,)))
    call("rmpcd_colloid_vv_vel", p.handle, float(dt), _dp(m))


def compute_force(ps1: ParticleSystem, ps2: ParticleSystem, n_list: NeighborList, L, lj_params: LJParams,
                  energy: bool = True) -> float | None:
    """compute_force, src/neighbor_list.f90:159-225; returns the energy when asked."""
    e = C.c_double(0)
    call("rmpcd_compute_force", ps1.handle, ps2.handle, n_list.handle, _dp(_d3(L)), lj_params.ptr,
         C.byref(e) if energy else None)
    return e.value if energy else None


def compute_force_n2(ps: ParticleSystem, L, lj_params: LJParams, energy: bool = True) -> float | None:
    e = C.c_double(0)
    call("rmpcd_compute_force_n2", ps.handle, _dp(_d3(L)), lj_params.ptr, C.byref(e) if energy else None)
    return e.value if energy else None


def flag_particles_nl(n_list: NeighborList, colloids: ParticleSystem, solvent: ParticleSystem, edges,
                      cut_sq: float, point: int = 0) -> None:
    call("rmpcd_flag_particles_nl", n_list.handle, int(point), colloids.handle, solvent.handle, _dp(_d3(edges)),
         float(cut_sq))


def change_species(solvent: ParticleSystem, colloids: ParticleSystem, edges, cut_sq_C: float, cut_sq_N: float,
                   prob: float, state: Rng) -> None:
    call("rmpcd_change_species", solvent.handle, colloids.handle, _dp(_d3(edges)), float(cut_sq_C),
         float(cut_sq_N), float(prob), state.ptr)


def refuel(solvent: ParticleSystem, colloids: ParticleSystem, edges, L1: int) -> None:
    call("rmpcd_refuel", solvent.handle, colloids.handle, _dp(_d3(edges)), int(L1))


def n_solvent(solvent: ParticleSystem, n_species: int) -> np.ndarray:
    a = np.zeros(n_species, np.int32)
    call("rmpcd_n_solvent", solvent.handle, int(n_species), _ip(a))
    return a


def cylindrical_shell_histogram(solvent: ParticleSystem, x1, x2, L, bin_species: int, r_min: float,
                                r_max: float, xmin: float, dx: float, nbins: int) -> np.ndarray:
    h = np.zeros(nbins)
    call("rmpcd_cylindrical_shell_histogram", solvent.handle, _dp(_d3(x1)), _dp(_d3(x2)), _dp(_d3(L)),
         int(bin_species), float(r_min), float(r_max), float(xmin), float(dx), int(nbins), _dp(h))
    return h


def velocity_sums(p: ParticleSystem) -> np.ndarray:
    """[sum(vel**2), sum(vel, dim=2)] as used by the thermo observables."""
    out = np.zeros(4)
    call("rmpcd_velocity_sums", p.handle, _dp(out))
    return out


def bulk_run(particles: ParticleSystem, cells: CellSystem, state: Rng, tau: float, n_intervals: int,
             alpha: float | None = None) -> None:
    """n_intervals of simple_mpcd_step -> mpcd_stream_periodic -> random_shift -> sort."""
    call("rmpcd_bulk_run", particles.handle, cells.handle, state.ptr, float(tau), int(alpha is not None),
         float(alpha or 0.0), int(n_intervals))


def bulk_shapes(precision: int = FP32) -> list[tuple[int, int]]:
    """(slots per block, blocks per SM) of every tile shape of the fused interval kernel."""
    n = C.c_int()
    sl = np.zeros(16, np.int32)
    mb = np.zeros(16, np.int32)
    call("rmpcd_bulk_shapes", int(precision), C.byref(n), _ip(sl), _ip(mb))
    return [(int(sl[k]), int(mb[k])) for k in range(n.value)]


def bulk_shape(precision: int = FP32) -> int:
    s = C.c_int()
    call("rmpcd_bulk_get_shape", int(precision), C.byref(s))
    return s.value


def set_bulk_shape(precision: int, shape: int) -> None:
    call("rmpcd_bulk_set_shape", int(precision), int(shape))


def bulk_autotune(L, precision: int = FP32, tau: float = 1.0, n_intervals: int = 5) -> tuple[int, list[float]]:
    """Time every tile shape on a synthetic bulk fluid of box L; the fastest is put in use."""
    n = len(bulk_shapes(precision))
    ms = (C.c_float * n)()
    best = C.c_int()
    call("rmpcd_bulk_autotune", _ip(_i3(L)), int(precision), float(tau), int(n_intervals), C.byref(best), ms)
    return best.value, [float(x) for x in ms]


__all__ += ["bulk_shapes", "bulk_shape", "set_bulk_shape", "bulk_autotune"]


class Timers:
    """Per-phase device timers (the reference's timer_t list)."""

    @staticmethod
    def enable(on: bool = True) -> None:
        call("rmpcd_timers_enable", int(bool(on)))

    @staticmethod
    def reset() -> None:
        call("rmpcd_timers_reset")

    @staticmethod
    def read() -> dict:
        out = {}
        i = 0
        while True:
            name = C.create_string_buffer(64)
            sec = C.c_double(0)
            calls = C.c_longlong(0)
            rc = lib().rmpcd_timers_read(i, name, 64, C.byref(sec), C.byref(calls))
            if rc != 0:
                break
            out[name.value.decode()] = (sec.value, calls.value)
            i += 1
        return out
