"""GPU parity: collisions, temperature, rescaling, streaming, bulk reactions.

FP64 results must equal the oracle bit for bit (same arithmetic order, no
FMA, same Philox draws); reductions over cells (temperature) agree to 1e-12
relative because their summation order differs.
"""
import numpy as np
import pytest

from helpers import assert_cells_same, assert_same, make_pair, upload

pytestmark = pytest.mark.gpu


def species_mix(N, seed):
    # mostly solvent (1, 2) plus some species <= 0, which the collision
    # excludes from the cell mean but still rotates
    r = np.random.default_rng(seed)
    return r.choice([1, 2, 0, -1], size=N, p=[0.6, 0.3, 0.05, 0.05]).astype(np.int32)


@pytest.mark.parametrize("L,N", [([8, 8, 8], 5120), ([5, 7, 9], 3150), ([32, 32, 32], 327680)])
@pytest.mark.parametrize("alpha", [None, 2.0])
def test_simple_mpcd_step_srd(rm, oracle, L, N, alpha):
    sp = species_mix(N, 1)
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=2, species=sp, origin=[-0.3, -0.8, -0.1])
    st = rm.Rng(1234, 17)
    oracle.simple_mpcd_step(op, oc, 1234, 17, alpha=alpha)
    rm.simple_mpcd_step(gp, gc, st, alpha=alpha)
    assert st.step == 18
    assert_same(gp, op, ("vel",))


def test_simple_mpcd_step_injected_axes(rm, oracle):
    L, N = [10, 6, 7], 4200
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=3, origin=[-0.5, -0.5, -0.5])
    r = np.random.default_rng(4)
    ax = r.normal(size=(oc.S, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    gc.set_axes(ax)
    oracle.simple_mpcd_step(op, oc, 0, 0, axes=ax)
    rm.simple_mpcd_step(gp, gc, rm.Rng(0))
    assert_same(gp, op, ("vel",))
    gc.set_axes(None)


@pytest.mark.parametrize("hydro", [True, False])
def test_simple_mpcd_step_thermostat(rm, oracle, hydro):
    L, N = [8, 8, 8], 5120
    sp = species_mix(N, 5)
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=6, species=sp)
    g = np.random.default_rng(7).normal(size=(N, 3))
    gp.set_gauss(g)
    oracle.simple_mpcd_step(op, oc, 5, 3, thermostat=True, T=0.5, hydro=hydro, gauss=g)
    rm.simple_mpcd_step(gp, gc, rm.Rng(5, 3), thermostat=True, T=0.5, hydro=hydro)
    assert_same(gp, op, ("vel",))
    gp.set_gauss(None)
    # Philox normals (Leva's method) on both sides
    oracle.simple_mpcd_step(op, oc, 5, 4, thermostat=True, T=0.5, hydro=hydro)
    rm.simple_mpcd_step(gp, gc, rm.Rng(5, 4), thermostat=True, T=0.5, hydro=hydro)
    assert_same(gp, op, ("vel",))


@pytest.mark.parametrize("hydro", [True, False])
def test_simple_mpcd_step_thermostat_fp32_draws(rm, oracle, hydro):
    """FP32 MPC-AT: the normals drawn on the device (the attempts of a warp's
    deviates shared by its lanes) give the velocities of the same deviates,
    computed by the oracle's generator, injected into the per-cell path."""
    L, N = [8, 8, 8], 5120
    sp = species_mix(N, 5)
    _, (gc, gp) = make_pair(rm, oracle, L, N, seed=6, species=sp, precision=32)
    _, (gc2, gp2) = make_pair(rm, oracle, L, N, seed=6, species=sp, precision=32)
    seed, step = 5, 4
    g = np.array([[oracle.normal(seed, step, i, k) for k in range(3)] for i in range(N)])
    gp2.set_gauss(g)
    rm.simple_mpcd_step(gp, gc, rm.Rng(seed, step), thermostat=True, T=0.5, hydro=hydro)
    rm.simple_mpcd_step(gp2, gc2, rm.Rng(seed, step), thermostat=True, T=0.5, hydro=hydro)
    v, v2 = gp.download("vel"), gp2.download("vel")
    assert np.array_equal(v, v2)
    assert not np.array_equal(v, make_pair(rm, oracle, L, N, seed=6, species=sp, precision=32)[1][1].download("vel"))


def test_thermostat_stop_conditions(rm, oracle):
    (oc, op), (gc, gp) = make_pair(rm, oracle, [4, 4, 4], 640, seed=1)
    with pytest.raises(rm.RmpcdError):
        rm.simple_mpcd_step(gp, gc, rm.Rng(1), thermostat=False, hydro=False)
    with pytest.raises(rm.RmpcdError):
        rm.simple_mpcd_step(gp, gc, rm.Rng(1), thermostat=True, T=None)


def test_compute_temperature_and_rescale(rm, oracle):
    L, N = [16, 12, 10], 19200
    sp = species_mix(N, 8)
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=9, species=sp, origin=[-0.2, -0.4, -0.6])
    t_o = oracle.compute_temperature(op, oc)
    t_g = rm.compute_temperature(gp, gc)
    assert abs(t_g - t_o) <= 1e-12 * abs(t_o)
    oracle.rescale_cells(op, oc, 0.7)
    rm.rescale_cells(gp, gc, None, 0.7)
    assert_same(gp, op, ("vel",))


def test_stream_periodic(rm, oracle):
    L, N = [9, 11, 13], 12870
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=10, vel_scale=3.0)
    for dt in (1.0, 0.37):
        oracle.mpcd_stream_periodic(op, oc, dt)
        rm.mpcd_stream_periodic(gp, gc, dt)
        assert_same(gp, op, ("pos", "vel", "image"))


@pytest.mark.parametrize("bc", [(1, 2, 2), (1, 3, 3), (1, 1, 2), (1, 2, 3)])
def test_stream_xforce_yzwall(rm, oracle, bc):
    L, N = [10, 8, 6], 4800
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=11, vel_scale=1.5, sorted_=False)
    oc.set_bc(bc)
    gc.set_bc(bc)
    for _ in range(3):
        oracle.mpcd_stream_xforce_yzwall(op, oc, 0.5, 0.1)
        rm.mpcd_stream_xforce_yzwall(gp, gc, 0.5, 0.1)
        assert_same(gp, op, ("pos", "vel", "flags"))
    rm.get_status()


def test_stream_nogravity_zwall(rm, oracle):
    L, N = [6, 6, 8], 2880
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=12, vel_scale=2.0, sorted_=False)
    op.force[:] = np.random.default_rng(13).normal(size=(N, 3)) * 0.1
    gp.upload("force", op.force)
    for _ in range(3):
        oracle.mpcd_stream_nogravity_zwall(op, oc, 0.3)
        rm.mpcd_stream_nogravity_zwall(gp, gc, 0.3)
        assert_same(gp, op, ("pos", "vel", "flags"))


def test_bulk_reaction(rm, oracle):
    L, N = [10, 10, 10], 9000
    sp = np.random.default_rng(14).choice([1, 2], size=N).astype(np.int32)
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=15, species=sp)
    reac = (np.arange(oc.S) % 3 != 0).astype(np.uint8)
    oc.is_reac[:] = reac
    gc.is_reac = reac
    oracle.bulk_reaction(op, oc, 2, 1, 0.3, 1.0, 21, 5)
    rm.bulk_reaction(gp, gc, 2, 1, 0.3, 1.0, rm.Rng(21, 5))
    assert_same(gp, op, ("species",))


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("delta_u", [0.5, 3.0])
def test_bulk_reaction_endothermic(rm, oracle, precision, delta_u):
    # delta_u = 3.0 is above the relative kinetic energy of many cells (10
    # particles at kT = 1/3 hold ~1.5), so both sides of the kin > delta_u
    # test occur
    L, N = [10, 10, 10], 9000
    sp = np.random.default_rng(14).choice([1, 2], size=N).astype(np.int32)
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=15, species=sp, precision=precision)
    reac = (np.arange(oc.S) % 3 != 0).astype(np.uint8)
    oc.is_reac[:] = reac
    gc.is_reac = reac
    if precision == 32:
        op.vel[:] = gp.download("vel")  # the FP32 form starts from the rounded velocities
    sp0, v0 = op.species.copy(), op.vel.copy()
    oracle.bulk_reaction_endothermic(op, oc, 2, 1, 0.3, 1.0, delta_u, 21, 5)
    st = rm.Rng(21, 5)
    rm.bulk_reaction_endothermic(gp, gc, 2, 1, 0.3, 1.0, st, delta_u)
    assert st.step == 6
    fired = np.nonzero(op.species != sp0)[0]
    assert fired.size > 0 and np.all(op.species[fired] == 1)
    assert_same(gp, op, ("species",))
    if precision == 64:
        assert_same(gp, op, ("vel",))
    else:
        # velocities computed in FP64 from the same FP32 inputs and rounded once
        assert_same(gp, op, ("vel",), exact=False, rtol=0, atol=4e-7 * np.abs(op.vel).max())
    # each reacting cell lost exactly delta_u of relative kinetic energy and kept its momentum
    starts, counts = oc.cell_start - 1, oc.cell_count
    cells = np.searchsorted(starts, fired, side="right") - 1
    for c in cells[:20]:
        a, n = starts[c], counts[c]
        vb, va = v0[a:a + n], op.vel[a:a + n]
        kin = lambda v: 0.5 * ((v - v.mean(0)) ** 2).sum()
        assert kin(vb) > delta_u
        assert abs(kin(vb) - kin(va) - delta_u) < 1e-9
        np.testing.assert_allclose(va.sum(0), vb.sum(0), atol=1e-9)


@pytest.mark.parametrize("thermostat", [False, True])
def test_wall_mpcd_step(rm, oracle, thermostat):
    L, N = [6, 6, 6], 2000
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=16, walls=True, origin=[-0.5, -0.5, 0.0])
    wt, wn = [0.8, 1.2], [10, 10]
    oracle.wall_mpcd_step(op, oc, 3, 9, wall_temperature=wt, wall_n=wn, thermostat=thermostat,
                          bulk_temperature=1.0)
    rm.wall_mpcd_step(gp, gc, rm.Rng(3, 9), wall_temperature=wt, wall_v=np.zeros((3, 2)), wall_n=wn,
                      thermostat=thermostat, bulk_temperature=1.0)
    assert_same(gp, op, ("vel",))
