"""GPU parity of whole schedules: the fused bulk-fluid interval against the
oracle's collide -> stream -> shift -> sort loop, and the single_dimer_pbc
MD + MPCD loop, both bit-exact in FP64; FP32 bulk runs checked against the
conservation laws and the FP64 run."""
import numpy as np
import pytest

from helpers import assert_cells_same, assert_same, make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,rho", [([16, 16, 16], 10), ([12, 10, 9], 10), ([6, 5, 4], 300), ([1, 20, 5], 10),
                                   ([64, 64, 40], 1)])
def test_bulk_run_fp64_bit_exact(rm, oracle, L, rho):
    N = int(np.prod(L)) * rho
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=N % 101, origin=[-0.1, -0.9, -0.45])
    n_int = 4
    rng = rm.Rng(99, 7)
    rm.bulk_run(gp, gc, rng, 1.0, n_int)
    oracle.bulk_run(op, oc, n_int, 1.0, 99, 7)
    assert rng.step == 7 + 2 * n_int
    assert np.array_equal(gc.origin, oc.origin)
    assert_cells_same(gc, oc)
    assert_same(gp, op, ("pos", "vel", "image", "id", "species", "flags"))


def test_bulk_run_alpha_and_injected_axes(rm, oracle):
    L = [8, 8, 8]
    N = 5120
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=3)
    rm.bulk_run(gp, gc, rm.Rng(5, 0), 1.0, 3, alpha=2.3)
    oracle.bulk_run(op, oc, 3, 1.0, 5, 0, alpha=2.3)
    assert_same(gp, op, ("pos", "vel", "image", "id"))


def test_bulk_run_fp32_conservation(rm, oracle):
    L = [16, 16, 16]
    N = 40960
    (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=4, precision=32)
    p0 = gp.download("vel").sum(0)
    e0 = (gp.download("vel") ** 2).sum()
    rm.bulk_run(gp, gc, rm.Rng(8), 1.0, 20)
    v = gp.download("vel")
    # SRD conserves momentum and energy cell by cell; FP32 drift per step is tiny
    assert np.abs(v.sum(0) - p0).max() / np.sqrt(e0) < 1e-4
    assert abs((v ** 2).sum() - e0) / e0 < 1e-4
    # the final state is sorted for the final grid
    ids = gp.download("id")
    assert np.array_equal(np.sort(ids), np.arange(1, N + 1))
    cnt = gc.cell_count
    assert cnt.sum() == N
    # temperature of the FP32 run agrees with the FP64 oracle run statistically
    oracle.bulk_run(op, oc, 20, 1.0, 8, 0)
    t64 = oracle.compute_temperature(op, oc)
    t32 = rm.compute_temperature(gp, gc)
    assert abs(t32 - t64) / t64 < 0.05


def test_bulk_run_fp32_order_and_determinism(rm, oracle):
    """The FP32 fused form sums each cell exactly, so its result does not
    depend on the order of a cell's particles: two runs give the same arrays,
    and each cell ends in ascending order of the particles' positions on
    entry."""
    L, N = [16, 12, 10], 19200
    outs = []
    for _ in range(2):
        (oc, op), (gc, gp) = make_pair(rm, oracle, L, N, seed=12, precision=32)
        entry_id = gp.download("id")
        rm.bulk_run(gp, gc, rm.Rng(6, 0), 1.0, 3)
        outs.append({f: gp.download(f) for f in ("pos", "vel", "image", "id")})
    for f in outs[0]:
        assert np.array_equal(outs[0][f], outs[1][f]), f
    ids = outs[0]["id"]
    where = np.empty(N + 1, np.int64)
    where[entry_id] = np.arange(N)
    cnt = gc.cell_count
    start = gc.cell_start - 1
    for s in np.nonzero(cnt > 1)[0]:
        seg = where[ids[start[s]:start[s] + cnt[s]]]
        assert np.all(np.diff(seg) > 0), f"cell {s}"
    assert np.array_equal(np.sort(ids), np.arange(1, N + 1))


@pytest.mark.parametrize("n_int", [2])
def test_single_dimer_pbc_bit_exact(rm, oracle, n_int):
    from oracle.programs import SingleDimerPBC as OD
    from rmpcdmd_b200.programs import SingleDimerPBC as GD

    kw = dict(L=(12, 12, 12), rho=10, N_MD=25, seed=11, list_capacity=4000)
    o = OD(**kw)
    g = GD(**kw)
    assert_same(g.solvent, o.s, ("pos", "vel", "species", "id"))
    for _ in range(n_int):
        o.interval()
        g.interval()
    assert_same(g.colloids, o.c, ("pos", "vel", "force"))
    assert_same(g.solvent, o.s, ("pos", "vel", "image", "id", "species", "flags", "force"))
    assert g.n_extra_sorting == o.n_extra_sorting
    assert g.rng.step == o.step


def test_reference_dimer_test(rm):
    """test/dimer_test.py:13-22 on test/dimer_test.parameters, full length
    (200 loops after 20 of equilibration): the internal energy e1 + e2 +
    kinetic sampled after each md_loop has std < 0.1 and the centre-of-mass
    velocity is constant to 1e-15."""
    from rmpcdmd_b200.programs import SingleDimerPBC

    g = SingleDimerPBC(L=(24, 24, 24), rho=10, T=1.0, tau=1.0, N_MD=125, sigma_C=3.0, sigma_N=3.0, d=6.5,
                       epsilon_C=(1.0, 1.0), epsilon_N=(1.0, 0.2), epsilon_CC=1.0, epsilon_NC=1.0, epsilon_NN=1.0,
                       probability=1.0, bulk_rmpcd=False, do_thermostat=False, do_hydro=True, seed=5)
    n_loop, equilibration = 200, 20
    E, V = [], []
    for i in range(0, n_loop + equilibration + 1):
        g.md_loop(want_energy=i >= equilibration)
        if i >= equilibration:
            th = g.thermo()
            E.append(th["internal"])
            V.append(th["v_com"])
        g.mpcd()
    E, V = np.array(E), np.array(V)
    assert len(E) == n_loop + 1
    assert (E - E.mean()).std() < 0.1
    assert np.abs(V - V.mean(0)).max() < 1e-15
    # reactions happened and B was refuelled (species 2 present, then converted)
    assert g.n_extra_sorting > 0


def test_n_colloids_pbc_bit_exact(rm, oracle):
    """programs/n_colloids_pbc.f90: thermalisation (MPC-AT + rescaling) and
    production intervals with lazy cell-wise streaming, against the oracle."""
    from oracle.programs import NColloidsPBC as OC
    from rmpcdmd_b200.programs import NColloidsPBC as GC

    kw = dict(L=(20, 20, 20), rho=10, N_MD=20, N_colloids=5, seed=31, T_final=0.4)
    o = OC(**kw)
    g = GC(**kw)
    assert g.N == o.N
    assert_same(g.colloids, o.c, ("pos",))
    assert_same(g.solvent, o.s, ("pos", "vel", "species", "id"))
    o.thermalise(2)
    g.thermalise(2)
    o.run(2)
    g.run(2)
    assert_same(g.colloids, o.c, ("pos", "vel", "force", "image"))
    assert_same(g.solvent, o.s, ("pos", "vel", "image", "id", "species", "flags", "force"))
    assert g.n_extra_sorting == o.n_extra_sorting
    assert g.rng.step == o.step
    assert np.array_equal(g.cells.origin, o.cells.origin)
    assert g.e1 == o.e1 and g.e2 == o.e2


@pytest.mark.parametrize("precision", [64, 32])
def test_bulk_shapes_give_identical_results(rm, oracle, precision):
    """Every tile shape of the fused interval (and the autotuner's choice)
    produces the same arrays bit for bit."""
    shapes = rm.bulk_shapes(precision)
    assert len(shapes) >= 2
    keep = rm.bulk_shape(precision)
    outs = []
    try:
        for k in range(len(shapes)):
            rm.set_bulk_shape(precision, k)
            (_, _), (gc, gp) = make_pair(rm, oracle, [16, 12, 10], 19200, seed=8, precision=precision)
            rm.bulk_run(gp, gc, rm.Rng(3, 0), 1.0, 3)
            outs.append({f: gp.download(f) for f in ("pos", "vel", "image", "id")})
        for o in outs[1:]:
            for f in o:
                assert np.array_equal(o[f], outs[0][f]), f
        best, ms = rm.bulk_autotune([24, 24, 24], precision, 1.0, 2)
        assert 0 <= best < len(shapes) and rm.bulk_shape(precision) == best
        assert len(ms) == len(shapes) and all(m > 0 for m in ms)
    finally:
        rm.set_bulk_shape(precision, keep)


def test_n_colloids_native_loop_kept_between_calls(rm):
    """rmpcd_ncolloids_run keeps its scratch and captured MD-step graphs for
    the next call on the same systems and parameters, and rebuilds them when
    the systems change: calls alternating between two systems (and a change
    of skin) give the states of the same calls made without alternation, and
    of the same calls with graphs off."""
    from rmpcdmd_b200._capi import call
    from rmpcdmd_b200.programs import NColloidsPBC

    def make(seed):
        return NColloidsPBC(L=(20, 20, 20), rho=10, N_MD=10, N_colloids=6, seed=seed, precision=32)

    a, b, a_ref, b_ref, a_off = make(3), make(4), make(3), make(4), make(3)
    for k in range(3):
        a.thermalise(1)
        b.thermalise(1)
        if k == 1:
            a.skin = b.skin = 0.9 * a.skin
    for k in range(3):
        a_ref.thermalise(1)
        if k == 1:
            a_ref.skin = 0.9 * a_ref.skin
    for k in range(3):
        b_ref.thermalise(1)
        if k == 1:
            b_ref.skin = 0.9 * b_ref.skin
    call("rmpcd_ncolloids_set_graphs", 0)
    try:
        for k in range(3):
            a_off.thermalise(1)
            if k == 1:
                a_off.skin = 0.9 * a_off.skin
    finally:
        call("rmpcd_ncolloids_set_graphs", 1)
    for x, y in ((a, a_ref), (b, b_ref), (a, a_off)):
        for f in ("pos", "vel", "image", "id", "flags", "force", "force_old"):
            assert np.array_equal(x.solvent.download(f), y.solvent.download(f)), f
        for f in ("pos", "vel", "force"):
            assert np.array_equal(x.colloids.download(f), y.colloids.download(f)), f
        assert x.n_extra_sorting == y.n_extra_sorting
    assert a.n_extra_sorting > 0


@pytest.mark.parametrize("precision,graphs", [(64, True), (32, True), (64, False)])
def test_n_colloids_native_loop_matches_call_by_call(rm, precision, graphs):
    """rmpcd_ncolloids_run issues the program's calls in C; the state after
    thermalisation (with the 10th-interval rescaling) and a temperature ramp
    equals the Python loop making the same calls one by one (flags, pos_old
    and both force buffers included: the native loop rolls flags over the MD
    cells only from the third MD step after a sort on, reads force entries of
    flagged particles only, and copies pos_old of the MD cells only except
    at its last sort)."""
    from rmpcdmd_b200.programs import NColloidsPBC

    kw = dict(L=(24, 24, 24), rho=10, N_MD=10, N_colloids=8, seed=77, T_final=0.5, precision=precision)
    a = NColloidsPBC(**kw)
    b = NColloidsPBC(**kw)
    from rmpcdmd_b200._capi import call

    call("rmpcd_ncolloids_set_graphs", int(graphs))
    try:
        a.thermalise(10, native=False)
        b.thermalise(10, native=True)
        a.run(3, native=False)
        b.run(3, native=True)
    finally:
        call("rmpcd_ncolloids_set_graphs", 1)
    for f in ("pos", "pos_old", "vel", "image", "id", "flags", "force", "force_old"):
        assert np.array_equal(a.solvent.download(f), b.solvent.download(f)), f
    for f in ("pos", "vel", "force", "image"):
        assert np.array_equal(a.colloids.download(f), b.colloids.download(f)), f
    assert (a.t, a.last_sort, a.n_extra_sorting, a.rng.step) == (b.t, b.last_sort, b.n_extra_sorting, b.rng.step)
    assert b.n_extra_sorting > 0  # sorts inside MD steps occurred
    assert a.e1 == b.e1 and a.e2 == b.e2
