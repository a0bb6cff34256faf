"""GPU parity: stencil, neighbor list, list-based LJ forces, colloid-colloid
forces, reactions and observables of single_dimer_pbc (bit-exact)."""
import numpy as np
import pytest

from helpers import assert_same, make_pair, upload

pytestmark = pytest.mark.gpu

TWO16 = 2 ** (1 / 6)


def dimer_lj(rm, oracle, sigma=2.0, eps_C=(1.0, 1.0), eps_N=(1.0, 0.5)):
    eps = np.array([[eps_C[0], eps_N[0]], [eps_C[1], eps_N[1]]])
    sig = np.full((2, 2), sigma)
    cut = sig * TWO16
    return rm.LJParams(eps, sig, cut), oracle.LJParams(eps, sig, cut)


def dimer_setup(rm, oracle, L=(16, 16, 16), rho=10, d=4.5, sigma=2.0, nmax=4000, seed=1):
    L = np.array(L)
    N = int(np.prod(L) * rho)
    mass = np.array([rho * sigma ** 3 * 4 * np.float32(3.14159265) / 3] * 2)
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=seed, species=1, sorted_=False, origin=[-0.3, -0.6, -0.2])
    ocol = oracle.Particles(2, 2, mass)
    gcol = rm.ParticleSystem(2, 2, mass)
    ocol.species[:] = [1, 2]
    ocol.pos[:] = [L / 2, L / 2 + [d, 0, 0]]
    upload(gcol, ocol, ("pos", "species"))
    glj, olj = dimer_lj(rm, oracle, sigma)
    oracle.random_placement(op, oc.edges, 77, ocol, olj)
    gp.random_placement(gc.edges, gcol, glj, 77)
    assert_same(gp, op, ("pos",))
    op.sort(oc)
    gp.sort(gc)
    radius = sigma * TWO16 + 2
    onl = oracle.NeighborList(2, nmax)
    gnl = rm.NeighborList(2, nmax)
    onl.make_stencil(oc, radius)
    gnl.make_stencil(gc, radius)
    return dict(L=L, N=N, oc=oc, op=op, gc=gc, gp=gp, ocol=ocol, gcol=gcol, glj=glj, olj=olj, onl=onl, gnl=gnl,
                radius=radius, mass=mass)


def test_stencil_size(rm, oracle):
    for cut in (1.0, 2.5, 4.245, 4.17, 7.3):
        c = oracle.Cells([16, 16, 16])
        nl = oracle.NeighborList(1, 10)
        nl.make_stencil(c, cut)
        g = rm.NeighborList(1, 10)
        g.make_stencil(rm.CellSystem([16, 16, 16]), cut)
        assert g.stencil_size == len(nl.stencil)


def test_update_list_and_forces(rm, oracle):
    s = dimer_setup(rm, oracle)
    s["onl"].update_list(s["ocol"], s["op"], s["radius"], s["oc"], s["olj"])
    s["gnl"].update_list(s["gcol"], s["gp"], s["radius"], s["gc"], s["glj"])
    lst, n = s["gnl"].download()
    assert np.array_equal(n, s["onl"].n)
    assert np.array_equal(lst, np.where(np.arange(s["onl"].Nmax) < n[:, None], s["onl"].list, 0))
    assert np.array_equal(s["gc"].is_md, s["oc"].is_md.astype(bool))
    assert np.array_equal(s["gc"].is_reac, s["oc"].is_reac.astype(bool))
    # forces from zero (the program zeroes them before compute_force)
    e_o = oracle.compute_force(s["ocol"], s["op"], s["onl"], s["oc"].edges, s["olj"])
    e_g = rm.compute_force(s["gcol"], s["gp"], s["gnl"], s["gc"].edges, s["glj"])
    assert e_g == e_o
    assert_same(s["gp"], s["op"], ("force", "flags"))
    assert_same(s["gcol"], s["ocol"], ("force",))
    # a second call accumulates onto existing forces in reference order
    e_o = oracle.compute_force(s["ocol"], s["op"], s["onl"], s["oc"].edges, s["olj"])
    e_g = rm.compute_force(s["gcol"], s["gp"], s["gnl"], s["gc"].edges, s["glj"])
    assert e_g == e_o
    assert_same(s["gp"], s["op"], ("force", "flags"))


def test_update_list_overflow_is_reported(rm, oracle):
    s = dimer_setup(rm, oracle, nmax=100)
    with pytest.raises(rm.RmpcdError) as e:
        s["gnl"].update_list(s["gcol"], s["gp"], s["radius"], s["gc"], s["glj"])
    assert "maximum of neighbor list reached" in str(e.value)
    rm.get_status()


def test_neighbor_list_many_colloids_small_box(rm, oracle):
    # test/test_neighbor_list_0.f90 geometry, plus a box smaller than the
    # stencil so one list can hold a particle twice
    for L, C, cutoff in (([20, 10, 35], 20, 3.6), ([6, 6, 6], 5, 3.0)):
        L = np.array(L)
        N = int(L.prod()) * 20
        (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=3, origin=[-0.5, -0.5, -0.5])
        r = np.random.default_rng(4)
        ocol = oracle.Particles(C, 1, [100.0])
        gcol = rm.ParticleSystem(C, 1, [100.0])
        ocol.species[:] = 1
        ocol.pos[:] = r.random((C, 3)) * L
        upload(gcol, ocol, ("pos", "species"))
        nmax = 20 * 6 * int(cutoff ** 3) * 2
        onl = oracle.NeighborList(C, nmax)
        gnl = rm.NeighborList(C, nmax)
        onl.make_stencil(oc, cutoff)
        gnl.make_stencil(gc, cutoff)
        onl.update_list(ocol, op, cutoff, oc)
        gnl.update_list(gcol, gp, cutoff, gc)
        lst, n = gnl.download()
        assert np.array_equal(n, onl.n)
        for i in range(C):
            assert np.array_equal(lst[i, :n[i]], onl.list[i, :n[i]])
        lj_o = oracle.LJParams([[1.0]], [[1.5]], [[1.5 * TWO16]])
        lj_g = rm.LJParams([[1.0]], [[1.5]], [[1.5 * TWO16]])
        e_o = oracle.compute_force(ocol, op, onl, oc.edges, lj_o)
        e_g = rm.compute_force(gcol, gp, gnl, gc.edges, lj_g)
        assert e_g == e_o
        assert_same(gp, op, ("force", "flags"))
        assert_same(gcol, ocol, ("force",))


@pytest.mark.parametrize("rho", [10, 40])
def test_update_list_fp32_solvent(rm, oracle, rho):
    # the FP32 solvent form of update_list: the oracle gets the same float
    # positions; at density 40 every full stencil chunk holds more candidates
    # than the shared-memory stage and reads them directly, at 10 they are
    # staged by bulk copies
    L = np.array([24, 20, 22])
    N = int(L.prod()) * rho
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=7, precision=32, origin=[-0.5, -0.25, -0.75],
                                   sorted_=False)
    op.pos[:] = gp.download("pos")
    op.vel[:] = gp.download("vel")
    op.sort(oc)
    gp.sort(gc)
    C, cutoff = 12, 4.0
    r = np.random.default_rng(8)
    ocol = oracle.Particles(C, 1, [100.0])
    gcol = rm.ParticleSystem(C, 1, [100.0])
    ocol.species[:] = 1
    ocol.pos[:] = r.random((C, 3)) * L
    upload(gcol, ocol, ("pos", "species"))
    nmax = rho * 6 * int(cutoff ** 3) * 2
    onl = oracle.NeighborList(C, nmax)
    gnl = rm.NeighborList(C, nmax)
    onl.make_stencil(oc, cutoff)
    gnl.make_stencil(gc, cutoff)
    onl.update_list(ocol, op, cutoff, oc)
    gnl.update_list(gcol, gp, cutoff, gc)
    lst, n = gnl.download()
    assert np.array_equal(n, onl.n) and n.min() > 0
    for i in range(C):
        assert np.array_equal(lst[i, :n[i]], onl.list[i, :n[i]])
    assert np.array_equal(gc.is_md, oc.is_md.astype(bool))
    rm.get_status()


def fp32_colloid_force_case(rm, oracle, seed):
    """compute_force with an FP32 solvent on both sides: the oracle gets the
    same float positions (its FP64 arithmetic then sees the same inputs)."""
    L = np.array([24, 20, 22])
    N = int(L.prod()) * 10
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=seed, precision=32, origin=[-0.5, -0.25, -0.75],
                                   sorted_=False)
    op.pos[:] = gp.download("pos")
    op.sort(oc)
    gp.sort(gc)
    C, cutoff = 12, 4.0
    r = np.random.default_rng(seed + 1)
    ocol = oracle.Particles(C, 1, [100.0])
    gcol = rm.ParticleSystem(C, 1, [100.0])
    ocol.species[:] = 1
    ocol.pos[:] = r.random((C, 3)) * L
    upload(gcol, ocol, ("pos", "species"))
    onl = oracle.NeighborList(C, 12000)
    gnl = rm.NeighborList(C, 12000)
    onl.make_stencil(oc, cutoff)
    gnl.make_stencil(gc, cutoff)
    onl.update_list(ocol, op, cutoff, oc)
    gnl.update_list(gcol, gp, cutoff, gc)
    lj_o = oracle.LJParams([[1.0]], [[1.5]], [[1.5 * TWO16]])
    lj_g = rm.LJParams([[1.0]], [[1.5]], [[1.5 * TWO16]])
    e_o = oracle.compute_force(ocol, op, onl, oc.edges, lj_o)
    e_g = rm.compute_force(gcol, gp, gnl, gc.edges, lj_g)
    return e_o, e_g, ocol, gcol, op, gp


def test_compute_force_fp32_solvent_tree_sums(rm, oracle):
    """With an FP32 solvent each colloid's force is the FP64 sum of its pair
    forces by a fixed tree instead of list order: equal to the oracle's
    list-order sum to FP64 rounding and the same bits on every run; the
    energy keeps list order (equal bit for bit) and each solvent force is the
    oracle's, rounded to FP32."""
    e_o, e_g, ocol, gcol, op, gp = fp32_colloid_force_case(rm, oracle, 7)
    assert e_g == e_o
    cf_o, cf_g = ocol.force, gcol.download("force")
    assert np.isfinite(cf_o).all() and np.abs(cf_o).max() > 1.0
    assert not np.array_equal(cf_g, np.zeros_like(cf_g))
    np.testing.assert_allclose(cf_g, cf_o, rtol=0, atol=1e-12 * np.abs(cf_o).max())
    # a particle with one contribution gets -pf rounded once, as the oracle's
    # value rounded to FP32; the few with several differ by FP32 rounding
    sf_o, sf_g = op.force.astype(np.float32), gp.download("force")
    assert np.isfinite(sf_g).all() and np.count_nonzero(sf_o) > 1000
    same = np.all(sf_g == sf_o, axis=1)
    assert same.mean() > 0.99
    np.testing.assert_allclose(sf_g[~same], sf_o[~same], rtol=1e-5)
    _, _, _, gcol2, _, _ = fp32_colloid_force_case(rm, oracle, 7)
    assert np.array_equal(gcol2.download("force"), cf_g)
    rm.get_status()


@pytest.mark.parametrize("C,box", [(200, 20.0), (300, 70.0), (20, 30.0)])
def test_compute_force_n2(rm, oracle, C, box):
    # box 20: every pair inside the cut; box 70: most pairs beyond it; C = 20:
    # the single-thread path
    r = np.random.default_rng(5)
    ocol = oracle.Particles(C, 1, [100.0])
    gcol = rm.ParticleSystem(C, 1, [100.0])
    ocol.species[:] = 1
    ocol.pos[:] = r.random((C, 3)) * box
    ocol.force[:] = r.normal(size=(C, 3))
    upload(gcol, ocol, ("pos", "species", "force"))
    lj_o = oracle.LJParams([[1.0]], [[6.0]], [[18.0]])
    lj_g = rm.LJParams([[1.0]], [[6.0]], [[18.0]])
    e_o = oracle.compute_force_n2(ocol, [box] * 3, lj_o)
    e_g = rm.compute_force_n2(gcol, [box] * 3, lj_g)
    assert e_o != 0
    assert e_g == e_o
    assert_same(gcol, ocol, ("force",))


def test_reactions_and_observables(rm, oracle):
    s = dimer_setup(rm, oracle, L=(20, 20, 20), seed=7)
    op, gp, ocol, gcol = s["op"], s["gp"], s["ocol"], s["gcol"]
    s["onl"].update_list(ocol, op, s["radius"], s["oc"], s["olj"])
    s["gnl"].update_list(gcol, gp, s["radius"], s["gc"], s["glj"])
    edges = s["oc"].edges
    cut = s["olj"].cut_sq
    # move solvent a little so some flagged particles leave the cutoffs
    oracle.flag_particles_nl(s["onl"], ocol, op, edges, cut[0, 0])
    rm.flag_particles_nl(s["gnl"], gcol, gp, edges, cut[0, 0])
    assert_same(gp, op, ("flags",))
    op.pos[:] = (op.pos + np.random.default_rng(8).normal(size=op.pos.shape)) % edges
    gp.upload("pos", op.pos)
    for prob in (1.0, 0.5):
        oracle.change_species(op, ocol, edges, cut[0, 0], cut[0, 1], prob, 5, 11)
        rm.change_species(gp, gcol, edges, cut[0, 0], cut[0, 1], prob, rm.Rng(5, 11))
        assert_same(gp, op, ("species", "flags"))
    # refuel with far = (L1*0.45)**2 in single precision
    op.species[::3] = 2
    gp.upload("species", op.species)
    oracle.refuel(op, ocol, edges, int(s["L"][0]))
    rm.refuel(gp, gcol, edges, int(s["L"][0]))
    assert_same(gp, op, ("species",))
    assert np.array_equal(rm.n_solvent(gp, 2), oracle.n_solvent(op, 2))
    h_o = oracle.cylindrical_shell_histogram(op, ocol.pos[0], ocol.pos[1], edges, 2, 2.0, 4.0, -5.0, 0.095, 100)
    h_g = rm.cylindrical_shell_histogram(gp, ocol.pos[0], ocol.pos[1], edges, 2, 2.0, 4.0, -5.0, 0.095, 100)
    assert np.array_equal(h_o, h_g)
    vo = oracle.velocity_sums(op)
    vg = rm.velocity_sums(gp)
    assert abs(vg[0] - vo[0]) <= 1e-12 * vo[0]
    assert np.allclose(vg[1:], vo[1:], rtol=0, atol=1e-9)
