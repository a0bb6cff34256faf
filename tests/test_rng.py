"""Counter-based random numbers: the product's generator (host evaluation of
the same inline code the kernels run) equals the oracle's independent C
implementation draw for draw, and the derived distributions are correct.

The reference draws from Threefry streams (an absent submodule), so there is
no reference value to pin; distribution tests stand in for that.
"""
import numpy as np
import pytest
from scipy import stats


def _keys(n, seed=1):
    r = np.random.default_rng(seed)
    return [(int(r.integers(0, 2**63)), int(r.integers(0, 2**40)), int(r.integers(0, 2**31)))
            for _ in range(n)]


def test_uniform_bit_exact(oracle, rm):
    for s, st, i in _keys(500):
        for stream in (1, 2, 3, 4, 5, 7):
            a = rm.rng_uniform2(s, st, i, stream, 3)
            b = oracle.rng_u2(s, st, i, stream, 3)
            assert a[0] == b[0] and a[1] == b[1]


def test_sphere_and_normal_bit_exact(oracle, rm):
    import ctypes as C

    L = rm._capi.lib()
    for s, st, i in _keys(500, 2):
        out = np.zeros(3)
        assert L.rmpcd_rng_sphere(s, st, i, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        assert np.array_equal(out, oracle.rand_sphere(s, st, i))
        for sub in range(3):
            z = C.c_double(0)
            assert L.rmpcd_rng_normal(s, st, i, sub, C.byref(z)) == 0
            assert z.value == oracle.normal(s, st, i, sub)


def test_uniform_distribution(oracle):
    u = np.array([oracle.rng_u2(7, 3, i, 1)[k] for i in range(20000) for k in range(2)])
    assert u.min() >= 0.0 and u.max() < 1.0
    assert stats.kstest(u, "uniform").pvalue > 1e-3
    # consecutive draws are uncorrelated
    assert abs(np.corrcoef(u[:-1], u[1:])[0, 1]) < 0.02


def test_sphere_distribution(oracle):
    n = np.array([oracle.rand_sphere(11, 5, i) for i in range(20000)])
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-14)
    # Archimedes: each coordinate of a uniform unit vector is uniform on [-1, 1]
    for k in range(3):
        assert stats.kstest((n[:, k] + 1) / 2, "uniform").pvalue > 1e-3
    assert np.abs(n.mean(axis=0)).max() < 0.02


def test_normal_distribution(oracle):
    z = np.array([oracle.normal(13, 2, i, k) for i in range(10000) for k in range(3)])
    assert stats.kstest(z, "norm").pvalue > 1e-3
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1) < 0.02
    assert abs(stats.skew(z)) < 0.05 and abs(stats.kurtosis(z)) < 0.1


def test_leva_quadratic_bounds_are_valid():
    """Q < r1 must imply acceptance and Q > r2 rejection (Leva 1992)."""
    u = np.linspace(1e-6, 1.0, 1500)
    v = np.linspace(-0.8578, 0.8578, 1500)
    U, V = np.meshgrid(u, v)
    x = U - 0.449871
    y = np.abs(V) + 0.386595
    Q = x * x + y * (0.19600 * y - 0.25472 * x)
    accept = V * V <= -4.0 * np.log(U) * U * U
    assert accept[Q < 0.27597].all()
    assert not accept[Q > 0.27846].any()


def test_random_shift_values_in_range(oracle):
    o = np.array([oracle.random_shift_values(3, s) for s in range(5000)])
    assert (o >= -1).all() and (o < 0).all()
