"""Checkpoint / resume at interval boundaries (bit-exact continuation), and
the non-finite-value check with NaN velocities injected on the host."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "image", "id", "species", "flags", "force", "force_old")


def bulk_system(rm, L, precision, seed=3):
    N = 10 * int(np.prod(L))
    r = np.random.default_rng(seed)
    c = rm.CellSystem(L, 1.0)
    p = rm.ParticleSystem(N, 1, None, precision)
    p.upload("pos", r.random((N, 3)) * c.edges)
    p.upload("vel", r.normal(size=(N, 3)) * np.sqrt(1 / 3))
    p.upload("species", np.ones(N, np.int32))
    c.origin = [-0.3, -0.6, -0.2]
    p.sort(c)
    return p, c


@pytest.mark.parametrize("precision", [64, 32])
def test_bulk_resume_is_bit_exact(rm, tmp_path, precision):
    from rmpcdmd_b200 import checkpoint as ck

    p, c = bulk_system(rm, [12, 10, 8], precision)
    rng = rm.Rng(17, 4)
    rm.bulk_run(p, c, rng, 1.0, 2)
    ck.save_bulk(tmp_path / "b.npz", p, c, rng)
    rm.bulk_run(p, c, rng, 1.0, 3)
    q, d, rng2 = ck.load_bulk(tmp_path / "b.npz")
    rm.bulk_run(q, d, rng2, 1.0, 3)
    for f in ("pos", "vel", "image", "id", "species", "flags"):
        assert np.array_equal(p.download(f), q.download(f)), f
    assert rng.step == rng2.step
    assert np.array_equal(c.origin, d.origin)
    assert np.array_equal(c.cell_count, d.cell_count)


def test_dimer_resume_is_bit_exact(rm, tmp_path):
    from rmpcdmd_b200 import checkpoint as ck
    from rmpcdmd_b200.programs import SingleDimerPBC

    g = SingleDimerPBC(L=(14, 14, 14), rho=10, N_MD=20, seed=9, list_capacity=4000)
    g.interval()
    g.interval()
    ck.save_dimer(tmp_path / "d.npz", g)
    g.interval()
    g.interval()
    h = ck.load_dimer(tmp_path / "d.npz")
    h.interval()
    h.interval()
    for f in FIELDS:
        assert np.array_equal(g.solvent.download(f), h.solvent.download(f)), f
        assert np.array_equal(g.colloids.download(f), h.colloids.download(f)), f
    assert (g.rng.step, g.n_extra_sorting, g.md_steps) == (h.rng.step, h.n_extra_sorting, h.md_steps)


def test_n_colloids_resume_is_bit_exact(rm, tmp_path):
    from rmpcdmd_b200 import checkpoint as ck
    from rmpcdmd_b200.programs import NColloidsPBC

    kw = dict(L=(20, 20, 20), rho=10, N_MD=20, N_colloids=5, seed=31, T_final=0.4)
    g = NColloidsPBC(**kw)
    g.thermalise(2)
    g.run(1)
    ck.save_ncolloids(tmp_path / "n.npz", g)
    g.run(2)
    h = ck.load_ncolloids(tmp_path / "n.npz")
    h.run(2)
    for f in FIELDS:
        assert np.array_equal(g.solvent.download(f), h.solvent.download(f)), f
    for f in ("pos", "vel", "force", "image"):
        assert np.array_equal(g.colloids.download(f), h.colloids.download(f)), f
    assert (g.rng.step, g.t, g.last_sort, g.n_extra_sorting) == (h.rng.step, h.t, h.last_sort, h.n_extra_sorting)
    assert g.e1 == h.e1 and g.e2 == h.e2


@pytest.mark.parametrize("precision", [64, 32])
def test_nan_velocities_are_counted_and_contained(rm, precision):
    p, c = bulk_system(rm, [8, 8, 8], precision, seed=5)
    assert p.count_nonfinite() == 0
    v = p.download("vel")
    v[[3, 100, 2000]] = np.nan
    p.upload("vel", v)
    assert p.count_nonfinite() == 3
    # a collision spreads a NaN to its cell; the run keeps every slot index in
    # the grid and finishes
    rm.bulk_run(p, c, rm.Rng(1), 1.0, 2)
    n = p.count_nonfinite()
    assert n >= 3
    assert int(c.cell_count.sum()) == p.Nmax
    rm.get_status()
