"""ctypes binding of the C ABI declared in include/rmpcd.h.

The shared library is built in-tree (``python -m rmpcdmd_b200.build``) and
loaded from ``rmpcdmd_b200/_lib/librmpcd_b200.so``.  There is no fallback:
if the library is missing, importing the package raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "librmpcd_b200.so"

c_int_p = C.POINTER(C.c_int)
c_double_p = C.POINTER(C.c_double)
c_uchar_p = C.POINTER(C.c_ubyte)
c_void_p = C.c_void_p

MAX_SPECIES = 4


class LJ(C.Structure):
    """lj_params_t (src/interaction.f90:23-34), column-major (n1, n2) tables."""

    _fields_ = [
        ("n1", C.c_int),
        ("n2", C.c_int),
        ("epsilon", C.c_double * 16),
        ("sigma", C.c_double * 16),
        ("sigma_sq", C.c_double * 16),
        ("cut", C.c_double * 16),
        ("cut_sq", C.c_double * 16),
        ("cut_energy", C.c_double * 16),
    ]


class RNG(C.Structure):
    """{seed, step}: replaces the reference's threefry_rng_t state(:)."""

    _fields_ = [("seed", C.c_uint64), ("step", C.c_uint64)]


class DIMER_PARAMS(C.Structure):
    """rmpcd_dimer_params: the constants of the single_dimer_pbc main loop."""

    _fields_ = [
        ("tau", C.c_double),
        ("N_MD", C.c_int),
        ("bond", C.c_double),
        ("skin", C.c_double),
        ("list_radius", C.c_double),
        ("prob", C.c_double),
        ("cut_sq_C", C.c_double),
        ("cut_sq_N", C.c_double),
        ("vv_mass", C.c_double * 2),
        ("thermostat", C.c_int),
        ("hydro", C.c_int),
        ("T", C.c_double),
    ]


class NCOLLOIDS_PARAMS(C.Structure):
    """rmpcd_ncolloids_params: the constants of the n_colloids_pbc loops."""

    _fields_ = [("tau", C.c_double), ("N_MD", C.c_int), ("skin", C.c_double), ("list_radius", C.c_double),
                ("mass", C.c_double), ("do_hydro", C.c_int)]


class NCOLLOIDS_STATE(C.Structure):
    """rmpcd_ncolloids_state: the loop counters carried between calls."""

    _fields_ = [("t", C.c_int), ("last_sort", C.c_int), ("n_extra_sorting", C.c_int), ("e1", C.c_double),
                ("e2", C.c_double)]


CELLS_P = c_void_p
class RIGID_STATE(C.Structure):
    """rmpcd_rigid_body_state: rigid_body_t's scalar state (src/md.f90:40-58)."""

    _fields_ = [
        ("mass", C.c_double),
        ("pos", C.c_double * 3),
        ("vel", C.c_double * 3),
        ("force", C.c_double * 3),
        ("q", C.c_double * 4),
        ("L", C.c_double * 3),
        ("torque", C.c_double * 3),
        ("I_body", C.c_double * 3),
        ("omega_body", C.c_double * 3),
    ]


PART_P = c_void_p
NL_P = c_void_p
LJ_P = C.POINTER(LJ)
RNG_P = C.POINTER(RNG)

# name -> argtypes (every function returns int status unless noted)
PROTOTYPES = {
    "rmpcd_version": [c_int_p, c_int_p],
    "rmpcd_set_device": [C.c_int],
    "rmpcd_get_status": [],
    "rmpcd_synchronize": [],
    "rmpcd_timers_enable": [C.c_int],
    "rmpcd_timers_reset": [],
    "rmpcd_timers_read": [C.c_int, C.c_char_p, C.c_int, c_double_p, C.POINTER(C.c_longlong)],
    "rmpcd_mark": [c_int_p],
    "rmpcd_elapsed_ms": [C.c_int, C.c_int, C.POINTER(C.c_float)],
    "rmpcd_host_alloc": [C.c_size_t, C.POINTER(C.c_void_p)],
    "rmpcd_host_free": [C.c_void_p],
    "rmpcd_rng_uniform2": [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, c_double_p],
    "rmpcd_rng_sphere": [C.c_uint64, C.c_uint64, C.c_uint32, c_double_p],
    "rmpcd_rng_normal": [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, c_double_p],
    "rmpcd_compact_p_to_h": [c_int_p, c_int_p, c_int_p],
    "rmpcd_compact_h_to_p": [C.c_int, c_int_p, c_int_p],
    "rmpcd_cells_init": [C.POINTER(CELLS_P), c_int_p, C.c_double, C.c_int],
    "rmpcd_cells_destroy": [CELLS_P],
    "rmpcd_cells_info": [CELLS_P, c_int_p, c_int_p, c_int_p, c_double_p],
    "rmpcd_cells_set_origin": [CELLS_P, c_double_p],
    "rmpcd_cells_get_origin": [CELLS_P, c_double_p],
    "rmpcd_cells_set_bc": [CELLS_P, c_int_p],
    "rmpcd_cells_set_max_v": [CELLS_P, C.c_double],
    "rmpcd_cells_random_shift": [CELLS_P, RNG_P],
    "rmpcd_cells_count_particles": [CELLS_P, PART_P],
    "rmpcd_cells_sort_particles": [CELLS_P, PART_P, PART_P],
    "rmpcd_cells_download_count": [CELLS_P, c_int_p],
    "rmpcd_cells_download_start": [CELLS_P, c_int_p],
    "rmpcd_cells_download_is_md": [CELLS_P, c_uchar_p],
    "rmpcd_cells_download_is_reac": [CELLS_P, c_uchar_p],
    "rmpcd_cells_upload_is_md": [CELLS_P, c_uchar_p],
    "rmpcd_cells_upload_is_reac": [CELLS_P, c_uchar_p],
    "rmpcd_cells_set_axes": [CELLS_P, c_double_p],
    "rmpcd_particles_init": [C.POINTER(PART_P), C.c_int, C.c_int, c_double_p, C.c_int],
    "rmpcd_particles_destroy": [PART_P],
    "rmpcd_particles_info": [PART_P, c_int_p, c_int_p, c_int_p],
    "rmpcd_particles_upload": [PART_P, C.c_char_p, c_void_p],
    "rmpcd_particles_download": [PART_P, C.c_char_p, c_void_p],
    "rmpcd_particles_sort": [PART_P, CELLS_P],
    "rmpcd_particles_maximum_displacement": [PART_P, c_double_p],
    "rmpcd_cell_maximum_displacement": [CELLS_P, PART_P, C.c_double, c_double_p],
    "rmpcd_particles_random_placement": [PART_P, c_double_p, PART_P, LJ_P, RNG_P],
    "rmpcd_particles_count_nonfinite": [PART_P, C.POINTER(C.c_longlong)],
    "rmpcd_particles_maxwell": [PART_P, C.c_double, C.c_uint64],
    "rmpcd_particles_switch_force": [PART_P],
    "rmpcd_particles_zero_force": [PART_P],
    "rmpcd_particles_copy_pos_old": [PART_P],
    "rmpcd_particles_copy_pos_rattle": [PART_P],
    "rmpcd_particles_copy_force_old": [PART_P],
    "rmpcd_particles_set_gauss": [PART_P, c_double_p],
    "rmpcd_simple_mpcd_step": [PART_P, CELLS_P, RNG_P, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int],
    "rmpcd_wall_mpcd_step": [PART_P, CELLS_P, RNG_P, c_double_p, c_double_p, c_int_p, C.c_int, C.c_double,
                             C.c_int, C.c_double, C.c_int],
    "rmpcd_compute_temperature": [PART_P, CELLS_P, c_double_p],
    "rmpcd_rescale_cells": [PART_P, CELLS_P, RNG_P, C.c_double],
    "rmpcd_mpcd_stream_periodic": [PART_P, CELLS_P, C.c_double],
    "rmpcd_mpcd_stream_xforce_yzwall": [PART_P, CELLS_P, C.c_double, C.c_double],
    "rmpcd_mpcd_stream_nogravity_zwall": [PART_P, CELLS_P, C.c_double],
    "rmpcd_bulk_reaction": [PART_P, CELLS_P, C.c_int, C.c_int, C.c_double, C.c_double, RNG_P],
    "rmpcd_bulk_reaction_endothermic": [PART_P, CELLS_P, C.c_int, C.c_int, C.c_double, C.c_double, RNG_P,
                                        C.c_double],
    "rmpcd_md_pos": [PART_P, C.c_double],
    "rmpcd_md_vel": [PART_P, C.c_double],
    "rmpcd_cell_md_pos": [CELLS_P, PART_P, C.c_double, C.c_int],
    "rmpcd_cell_md_vel": [CELLS_P, PART_P, C.c_double, C.c_int],
    "rmpcd_cell_md_pos_ywall": [CELLS_P, PART_P, C.c_double, C.c_int],
    "rmpcd_cell_md_pos_zwall": [CELLS_P, PART_P, C.c_double, C.c_int],
    "rmpcd_apply_pbc": [PART_P, c_double_p],
    "rmpcd_rattle_dimer_pos": [PART_P, C.c_double, C.c_double, c_double_p],
    "rmpcd_rattle_body_pos": [PART_P, c_int_p, c_double_p, C.c_int, C.c_double, c_double_p, C.c_double, c_int_p],
    "rmpcd_rattle_body_vel": [PART_P, c_int_p, c_double_p, C.c_int, C.c_double, c_double_p, C.c_double, c_int_p],
    "rmpcd_elastic_network": [PART_P, c_int_p, c_double_p, C.c_int, C.c_double, c_double_p, c_double_p],
    "rmpcd_rigid_body_init": [C.POINTER(c_void_p), PART_P, C.c_int, C.c_int, c_double_p],
    "rmpcd_rigid_body_destroy": [c_void_p],
    "rmpcd_rigid_body_compute_force_torque": [c_void_p, PART_P],
    "rmpcd_rigid_body_vv1": [c_void_p, PART_P, C.c_double, C.c_double, c_double_p],
    "rmpcd_rigid_body_vv2": [c_void_p, PART_P, C.c_double],
    "rmpcd_rigid_body_get": [c_void_p, C.POINTER(RIGID_STATE), c_double_p],
    "rmpcd_rigid_body_set": [c_void_p, C.POINTER(RIGID_STATE)],
    "rmpcd_rattle_dimer_vel": [PART_P, C.c_double, C.c_double, c_double_p],
    "rmpcd_colloid_vv_pos": [PART_P, C.c_double, c_double_p],
    "rmpcd_colloid_vv_vel": [PART_P, C.c_double, c_double_p],
    "rmpcd_colloid_vv_pos_noalloc": [PART_P, C.c_double, c_double_p],
    "rmpcd_lj_init": [LJ_P, C.c_int, C.c_int, c_double_p, c_double_p, c_double_p],
    "rmpcd_nlist_init": [C.POINTER(NL_P), C.c_int, C.c_int],
    "rmpcd_nlist_destroy": [NL_P],
    "rmpcd_nlist_make_stencil": [NL_P, CELLS_P, C.c_double],
    "rmpcd_nlist_stencil_size": [NL_P, c_int_p],
    "rmpcd_nlist_update": [NL_P, PART_P, PART_P, C.c_double, CELLS_P, LJ_P],
    "rmpcd_nlist_download": [NL_P, c_int_p, c_int_p],
    "rmpcd_compute_force": [PART_P, PART_P, NL_P, c_double_p, LJ_P, c_double_p],
    "rmpcd_compute_force_n2": [PART_P, c_double_p, LJ_P, c_double_p],
    "rmpcd_flag_particles_nl": [NL_P, C.c_int, PART_P, PART_P, c_double_p, C.c_double],
    "rmpcd_change_species": [PART_P, PART_P, c_double_p, C.c_double, C.c_double, C.c_double, RNG_P],
    "rmpcd_refuel": [PART_P, PART_P, c_double_p, C.c_int],
    "rmpcd_n_solvent": [PART_P, C.c_int, c_int_p],
    "rmpcd_cylindrical_shell_histogram": [PART_P, c_double_p, c_double_p, c_double_p, C.c_int, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_int, c_double_p],
    "rmpcd_velocity_sums": [PART_P, c_double_p],
    "rmpcd_bulk_run": [PART_P, CELLS_P, RNG_P, C.c_double, C.c_int, C.c_double, C.c_int],
    "rmpcd_bulk_shapes": [C.c_int, c_int_p, c_int_p, c_int_p],
    "rmpcd_bulk_set_shape": [C.c_int, C.c_int],
    "rmpcd_bulk_get_shape": [C.c_int, c_int_p],
    "rmpcd_bulk_autotune": [c_int_p, C.c_int, C.c_double, C.c_int, c_int_p, C.POINTER(C.c_float)],
    "rmpcd_ncolloids_set_graphs": [C.c_int],
    "rmpcd_ncolloids_run": [PART_P, PART_P, CELLS_P, NL_P, LJ_P, LJ_P, RNG_P, C.POINTER(NCOLLOIDS_PARAMS),
                            C.c_int, C.c_int, c_double_p, C.c_int, C.c_int, C.c_double,
                            C.POINTER(NCOLLOIDS_STATE)],
    "rmpcd_dimer_batch_create": [C.POINTER(c_void_p), C.c_int, C.POINTER(c_void_p), C.POINTER(c_void_p),
                                 C.POINTER(c_void_p), C.POINTER(c_void_p), RNG_P, LJ_P, LJ_P,
                                 C.POINTER(DIMER_PARAMS)],
    "rmpcd_dimer_batch_destroy": [c_void_p],
    "rmpcd_dimer_batch_run": [c_void_p, C.c_int],
    "rmpcd_dimer_batch_set_graph": [c_void_p, C.c_int],
    "rmpcd_dimer_batch_scatter": [c_void_p, C.c_int, PART_P, PART_P, CELLS_P, NL_P, RNG_P],
    "rmpcd_dimer_batch_info": [c_void_p, c_int_p, C.POINTER(C.c_longlong), c_int_p],
    "rmpcd_dimer_batch_shapes": [C.c_int, c_int_p],
    "rmpcd_dimer_batch_shape_info": [C.c_int, C.c_int, c_int_p, c_int_p, c_int_p, c_int_p, c_int_p, c_int_p],
    "rmpcd_dimer_batch_set_shape": [c_void_p, C.c_int],
    "rmpcd_dimer_batch_get_shape": [c_void_p, c_int_p],
    "rmpcd_dimer_batch_autotune": [c_void_p, C.c_int, c_int_p, C.POINTER(C.c_float), c_int_p],
}


class RmpcdError(RuntimeError):
    """A non-zero rmpcd_status, with the library's message."""

    def __init__(self, code: int, fn: str, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code
        self.fn = fn
        self.msg = msg


def load(path: Path | str | None = None) -> C.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"rmpcdmd_b200: CUDA library {p} not built (run `python -m rmpcdmd_b200.build`); "
            "there is no CPU fallback")
    lib = C.CDLL(str(p))
    for name, argtypes in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = C.c_int
    lib.rmpcd_last_error_string.argtypes = []
    lib.rmpcd_last_error_string.restype = C.c_char_p
    return lib


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def call(name: str, *args) -> None:
    """Call a C-ABI function and raise RmpcdError on a non-zero status."""
    L = lib()
    rc = getattr(L, name)(*args)
    if rc != 0:
        msg = L.rmpcd_last_error_string().decode(errors="replace")
        raise RmpcdError(rc, name, msg)
