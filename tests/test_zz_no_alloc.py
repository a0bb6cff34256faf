"""rmpcd_colloid_vv_pos_noalloc (masses in fixed library scratch, no device
allocation) against rmpcd_colloid_vv_pos, both called through the C ABI.
The file name sorts last so the test also runs after every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 8192


def system(rm, N, seed):
    r = np.random.default_rng(seed)
    mass = np.array([335.1, 97.3, 12.5])
    p = rm.ParticleSystem(N, 3, mass)
    p.upload("pos", r.uniform(0, 30, size=(N, 3)))
    p.upload("vel", r.normal(size=(N, 3)) * 0.05)
    p.upload("force", r.normal(size=(N, 3)) * 10)
    p.upload("force_old", r.normal(size=(N, 3)) * 10)
    p.upload("species", r.integers(1, 4, size=N).astype(np.int32))
    per_particle = r.uniform(1.0, 400.0, size=N)
    return p, per_particle


def vv_pos(rm, name, p, dt, m):
    rm._capi.call(name, p.handle, C.c_double(dt), m.ctypes.data_as(C.POINTER(C.c_double)))


@pytest.mark.parametrize("N", [1, 300, MAX_PARTICLES])
def test_noalloc_matches_allocating_entry_point(rm, N):
    a, m = system(rm, N, 7)
    b, _ = system(rm, N, 7)
    for dt in (0.01, 0.02):  # two calls in a row on the same systems
        vv_pos(rm, "rmpcd_colloid_vv_pos", a, dt, m)
        vv_pos(rm, "rmpcd_colloid_vv_pos_noalloc", b, dt, m)
        np.testing.assert_allclose(b.download("pos"), a.download("pos"), rtol=1e-15, atol=0)
    rm.get_status()


def _free_device_bytes():
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            cudart = C.CDLL(name)
            break
        except OSError:
            continue
    else:
        pytest.skip("no CUDA runtime library to query free device memory")
    free, total = C.c_size_t(0), C.c_size_t(0)
    assert cudart.cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
    return free.value


def test_noalloc_leaves_free_device_memory_unchanged(rm):
    # the property the entry point exists for: after its one-time set-up it
    # takes no device memory, even for a system larger than any seen before
    warm, m0 = system(rm, 16, 9)
    vv_pos(rm, "rmpcd_colloid_vv_pos_noalloc", warm, 0.01, m0)
    p, m = system(rm, MAX_PARTICLES, 10)
    rm._capi.call("rmpcd_synchronize")
    before = _free_device_bytes()
    for dt in (0.01, 0.02, 0.005, 0.01):
        vv_pos(rm, "rmpcd_colloid_vv_pos_noalloc", p, dt, m)
    rm._capi.call("rmpcd_synchronize")
    assert _free_device_bytes() == before
    rm.get_status()


def test_noalloc_rejects_more_particles_than_its_scratch(rm):
    p, m = system(rm, MAX_PARTICLES + 1, 8)
    before = p.download("pos")
    with pytest.raises(rm.RmpcdError) as e:
        vv_pos(rm, "rmpcd_colloid_vv_pos_noalloc", p, 0.01, m)
    assert e.value.code == 5
    assert "8192" in str(e.value)
    assert np.array_equal(p.download("pos"), before)
    rm.get_status()
