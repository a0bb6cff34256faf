"""The C-ABI library loads without a GPU, exports every entry point that
include/rmpcd.h declares, and fails loudly (no CPU fallback) when no device
is present."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    txt = (ROOT / "include" / "rmpcd.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rmpcd_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert len(names) > 70
    for n in ("rmpcd_particles_sort", "rmpcd_simple_mpcd_step", "rmpcd_nlist_update", "rmpcd_compute_force",
              "rmpcd_bulk_run", "rmpcd_rattle_dimer_pos", "rmpcd_change_species"):
        assert n in names


def test_library_exports_every_declared_symbol(rm):
    lib = ctypes.CDLL(str(rm._capi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_prototypes_cover_header(rm):
    names = set(declared_functions()) - {"rmpcd_last_error_string"}
    assert names <= set(rm._capi.PROTOTYPES), sorted(names - set(rm._capi.PROTOTYPES))


def test_no_device_is_an_error_not_a_fallback(rm):
    from conftest import HAVE_GPU

    if HAVE_GPU:
        pytest.skip("a device is present")
    with pytest.raises(rm.RmpcdError) as e:
        rm.CellSystem([4, 4, 4])
    assert e.value.code == 6
    with pytest.raises(rm.RmpcdError):
        rm.ParticleSystem(10)


def test_lj_params_host(rm, oracle):
    eps = [[1.0, 0.5], [1.0, 1.0]]
    sig = [[2.0, 2.0], [2.0, 2.0]]
    cut = [[2 ** (1 / 6) * 2] * 2] * 2
    a = rm.LJParams(eps, sig, cut)
    b = oracle.LJParams(eps, sig, cut)
    for name in ("epsilon", "sigma", "cut", "cut_sq", "cut_energy"):
        assert (getattr(a, name) == b.table(name)).all(), name
