"""GPU parity: velocity-Verlet halves, lazy cell-wise updates with walls,
PBC wrap, displacement bounds, dimer RATTLE and the colloid integrator."""
import numpy as np
import pytest

from helpers import assert_same, make_pair, upload

pytestmark = pytest.mark.gpu


def with_forces(op, gp, seed, flags=True):
    r = np.random.default_rng(seed)
    N = op.N
    op.force[:] = r.normal(size=(N, 3))
    op.force_old[:] = r.normal(size=(N, 3))
    if flags:
        op.flags[:] = r.integers(0, 128, size=N)
    upload(gp, op, ("force", "force_old", "flags"))


def test_md_pos_vel_pbc(rm, oracle):
    L, N = [10, 12, 14], 16800
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=1)
    with_forces(op, gp, 2)
    for _ in range(3):
        oracle.md_pos(op, 0.01)
        rm.md_pos(gp, 0.01)
        oracle.md_vel(op, 0.01)
        rm.md_vel(gp, 0.01)
    assert_same(gp, op, ("pos", "vel", "flags"))
    op.pos[:] += np.random.default_rng(3).normal(size=(N, 3)) * 5
    gp.upload("pos", op.pos)
    oracle.apply_pbc(op, oc.edges)
    rm.apply_pbc(gp, gc.edges)
    assert_same(gp, op, ("pos", "image"))


def test_maximum_displacement(rm, oracle):
    L, N = [8, 8, 8], 5000
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=4, species=np.where(np.arange(5000) % 9 == 0, -1, 1))
    gp.copy_pos_old()
    op.pos_old[:] = op.pos
    r = np.random.default_rng(5)
    op.pos[:] += r.normal(size=(N, 3)) * 0.1
    gp.upload("pos", op.pos)
    assert rm.ParticleSystem.maximum_displacement(gp) == op.maximum_displacement()
    md = (np.arange(oc.S) % 2).astype(np.uint8)
    oc.is_md[:] = md
    gc.is_md = md
    gc.set_max_v(0.3)
    oc.g.max_v = 0.3
    assert rm.cell_maximum_displacement(gc, gp, 0.5) == oracle.cell_maximum_displacement(oc, op, 0.5)


@pytest.mark.parametrize("md_flag", [True, False])
def test_cell_md_pos_vel(rm, oracle, md_flag):
    L, N = [9, 9, 9], 7290
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=6)
    with_forces(op, gp, 7)
    md = (np.random.default_rng(8).random(oc.S) < 0.3).astype(np.uint8)
    oc.is_md[:] = md
    gc.is_md = md
    oracle.cell_md_pos(oc, op, 0.05, md_flag)
    rm.cell_md_pos(gc, gp, 0.05, md_flag)
    oracle.cell_md_vel(oc, op, 0.05, md_flag)
    rm.cell_md_vel(gc, gp, 0.05, md_flag)
    assert_same(gp, op, ("pos", "vel", "flags"))


@pytest.mark.parametrize("dim,bc", [(1, 2), (1, 3), (2, 2), (2, 3)])
def test_cell_md_pos_wall(rm, oracle, dim, bc):
    # test/test_md_0.f90 as a parity case: random velocities of the order of L
    L, N = [1, 20, 5], 679
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=9 + dim)
    bcs = [1, 1, 1]
    bcs[dim] = bc
    oc.set_bc(bcs)
    gc.set_bc(bcs)
    op.vel[:] = (-0.5 + np.random.default_rng(11).random((N, 3))) * 2 * np.array(L)
    gp.upload("vel", op.vel)
    oc.is_md[:] = 0
    gc.is_md = np.zeros(oc.S, np.uint8)
    oracle.cell_md_pos_wall(oc, op, dim, 1.0, False)
    (rm.cell_md_pos_ywall if dim == 1 else rm.cell_md_pos_zwall)(gc, gp, 1.0, False)
    assert_same(gp, op, ("pos", "vel"))


def dimer_pair(rm, oracle):
    mass = np.array([335.1, 335.1])
    oc = oracle.Particles(2, 2, mass)
    gc = rm.ParticleSystem(2, 2, mass)
    oc.species[:] = [1, 2]
    oc.pos[:] = [[16.0, 16.0, 16.0], [20.5, 16.0, 16.0]]
    r = np.random.default_rng(12)
    oc.vel[:] = r.normal(size=(2, 3)) * 0.05
    oc.force[:] = r.normal(size=(2, 3)) * 10
    oc.force_old[:] = r.normal(size=(2, 3)) * 10
    upload(gc, oc, ("pos", "vel", "species", "force", "force_old"))
    return oc, gc, mass


def test_rattle_and_colloid_vv(rm, oracle):
    oc, gc, mass = dimer_pair(rm, oracle)
    edges = [32.0, 32.0, 32.0]
    for _ in range(5):
        oc.pos_rattle[:] = oc.pos
        gc.copy_pos_rattle()
        oracle.colloid_vv_pos(oc, 0.01, mass)
        rm.colloid_vv_pos(gc, 0.01, mass)
        oracle.rattle_dimer_pos(oc, 4.5, 0.01, edges)
        rm.rattle_dimer_pos(gc, 4.5, 0.01, edges)
        oracle.colloid_vv_vel(oc, 0.01, mass)
        rm.colloid_vv_vel(gc, 0.01, mass)
        oracle.rattle_dimer_vel(oc, 4.5, 0.01, edges)
        rm.rattle_dimer_vel(gc, 4.5, 0.01, edges)
        assert_same(gc, oc, ("pos", "vel"))
    assert abs(np.linalg.norm(oc.pos[0] - oc.pos[1]) - 4.5) < 1e-10
    rm.get_status()
