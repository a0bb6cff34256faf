"""GPU parity: count_particles and particle_system_t%sort (bit-exact).

cell_count, cell_start, the sorted order (id) and every permuted array must
equal the oracle's single-thread result, including the padded-slot boxes,
walls, empty systems, oversized cells and positions outside the box.
"""
import numpy as np
import pytest

from helpers import assert_cells_same, assert_same, make_pair, upload

pytestmark = pytest.mark.gpu

BOXES = [([8, 8, 8], 5120), ([5, 7, 9], 3150), ([1, 20, 5], 1000), ([32, 32, 32], 327680), ([96, 96, 96], 400000)]


@pytest.mark.parametrize("L,N", BOXES)
@pytest.mark.parametrize("precision", [64, 32])
def test_sort_bit_exact(rm, oracle, L, N, precision):
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=N % 97, precision=precision,
                                   origin=[-0.25, -0.5, -0.75], sorted_=False)
    if precision == 32:
        # the FP32 form keys its float positions: give the oracle the same values
        op.pos[:] = gp.download("pos")
        op.vel[:] = gp.download("vel")
    op.sort(oc)
    gp.sort(gc)
    assert_cells_same(gc, oc)
    assert_same(gp, op, ("pos", "vel", "image", "id", "species", "flags"))
    assert np.array_equal(gp.id_to_idx, op.id_to_idx)


def test_sort_chain_with_forces_and_pos_old(rm, oracle):
    L, N = [12, 10, 9], 12000
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=3)
    rng = np.random.default_rng(4)
    op.force[:] = rng.normal(size=(N, 3))
    op.force_old[:] = rng.normal(size=(N, 3))
    op.image[:] = rng.integers(-3, 3, size=(N, 3))
    op.flags[:] = rng.integers(0, 64, size=N)
    upload(gp, op, ("force", "force_old", "image", "flags"))
    for k in range(4):
        o = rng.random(3) - 1
        oc.origin = o
        gc.origin = o
        op.pos[:] = (op.pos + rng.normal(size=(N, 3)) * 0.3) % L
        gp.upload("pos", op.pos)
        op.sort(oc)
        gp.sort(gc)
        assert_cells_same(gc, oc)
        assert_same(gp, op, ("pos", "vel", "force", "force_old", "image", "id", "species", "flags", "pos_old"))


def test_sort_walls(rm, oracle):
    (oc, op), (gc, gp) = make_pair(rm, oracle, [6, 6, 6], 3000, seed=5, walls=True, origin=[-0.4, -0.6, 0.0])
    assert gc.N == oc.S
    assert_cells_same(gc, oc)
    assert_same(gp, op)


def test_sort_empty_and_single(rm, oracle):
    for N in (0, 1):
        (oc, op), (gc, gp) = make_pair(rm, oracle, [4, 4, 4], N, seed=1)
        assert_cells_same(gc, oc)
        assert_same(gp, op)


def test_sort_one_dense_cell(rm, oracle):
    # 5000 particles in one cell: the long-segment ordering path
    N = 5000
    (oc, op), (gc, gp) = make_pair(rm, oracle, [4, 4, 4], N, seed=2, sorted_=False)
    rng = np.random.default_rng(9)
    op.pos[:] = 1.0 + 0.5 * rng.random((N, 3))
    op.pos[::7] = rng.random((len(op.pos[::7]), 3)) * 4
    gp.upload("pos", op.pos)
    op.sort(oc)
    gp.sort(gc)
    assert_cells_same(gc, oc)
    assert_same(gp, op)


def test_sort_positions_outside_box(rm, oracle):
    # out-of-box positions are hashed as the reference's compact_p_to_h does
    N = 4000
    (oc, op), (gc, gp) = make_pair(rm, oracle, [8, 6, 10], N, seed=6, sorted_=False)
    rng = np.random.default_rng(10)
    op.pos[:] = rng.random((N, 3)) * 30 - 10
    gp.upload("pos", op.pos)
    op.sort(oc)
    gp.sort(gc)
    assert_cells_same(gc, oc)
    assert_same(gp, op)


def test_count_particles(rm, oracle):
    (oc, op), (gc, gp) = make_pair(rm, oracle, [16, 8, 12], 20000, seed=7, sorted_=False, origin=[-0.9, -0.1, -0.5])
    op.count(oc)
    gc.count_particles(gp)
    assert_cells_same(gc, oc)


@pytest.mark.parametrize("L,N", [([1, 1, 1], 7), ([3, 1, 2], 50), ([256, 128, 128], 30000)])
def test_count_particles_slot_scan_extremes(rm, oracle, L, N):
    # a single slot (one partial scan tile), a few slots, and 2^23 slots
    # (2048 scan tiles: each block adds more than one round of earlier
    # tile totals); counted twice so the second scan starts from the first's
    # state
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=N, sorted_=False, origin=[-0.5, -0.5, -0.5])
    for _ in range(2):
        op.count(oc)
        gc.count_particles(gp)
        assert_cells_same(gc, oc)
    assert int(gc.cell_count.sum()) == N


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("L,N,lo,hi", [([120, 30, 30], 1000000, 0.0, 1.0), ([7, 5, 9], 3000, -0.5, 1.5),
                                       ([4, 4, 4], 0, 0.0, 1.0)])
def test_sort_particles(rm, oracle, precision, L, N, lo, hi):
    """cell_system_t%sort_particles on test/test_cell_system_0.f90's geometry
    (10^6 positions in a 120 x 30 x 30 box), on positions partly outside the
    box, and on an empty system: count_particles, sort_particles, the starts
    the scatter leaves, then the reference test's checks after a recount."""
    rng = np.random.default_rng(N + 1)
    pos = (lo + (hi - lo) * rng.random((N, 3))) * np.asarray(L)
    if precision == 32:
        pos = pos.astype(np.float32).astype(np.float64)
    oc = oracle.Cells(L)
    op = oracle.Particles(N, 1)
    op.pos[:] = pos
    op.count(oc)
    want = op.sort_particles(oc)
    gc = rm.CellSystem(L, 1.0)
    a = rm.ParticleSystem(N, 1, None, precision)
    b = rm.ParticleSystem(N, 1, None, precision)
    a.pos = pos
    gc.count_particles(a)
    gc.sort_particles(a, b)
    assert np.array_equal(b.pos, want)
    assert np.array_equal(a.pos, pos)
    assert np.array_equal(gc.cell_start, oc.cell_start)  # advanced by the counts, as the reference leaves them
    gc.count_particles(b)
    start, count = gc.cell_start, gc.cell_count
    S = len(count)
    assert start[0] == 1 and start[S - 1] + count[S - 1] == N + 1 and count.sum() == N
    # every position lies in the cell of its range (test_cell_system_0.f90:61-70)
    if N:
        b.sort(gc)  # the scattered order is already the cell order: the sort is the identity
        assert np.array_equal(b.pos, want)
    rm.get_status()


def test_sort_particles_rejects_counts_of_other_positions(rm):
    L = [6, 6, 6]
    r = np.random.default_rng(3)
    gc = rm.CellSystem(L, 1.0)
    a = rm.ParticleSystem(2000, 1)
    b = rm.ParticleSystem(2000, 1)
    a.pos = r.random((2000, 3)) * 6
    b.pos = r.random((2000, 3)) * 6
    gc.count_particles(b)
    before = b.pos
    with pytest.raises(rm.RmpcdError) as e:
        gc.sort_particles(a, b)
    assert e.value.code == 1 and "count_particles" in str(e.value)
    assert np.array_equal(b.pos, before)
    with pytest.raises(rm.RmpcdError):
        gc.sort_particles(a, a)
    rm.get_status()
