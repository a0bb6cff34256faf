"""The batched single_dimer_pbc engine (rmpcd_dimer_batch_*) against the
same program driven call by call through the C ABI: every replica, with its
own box and seed, must end bit for bit where its own driver ends, in FP64
and in the FP32-solvent form, with the interval graph replayed or the
kernels launched one by one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOLVENT_FIELDS = ("pos", "vel", "image", "id", "species", "flags", "force", "force_old")
COLLOID_FIELDS = ("pos", "vel", "force", "force_old")


def drivers(rm, boxes, seeds, precision, N_MD):
    from rmpcdmd_b200.programs import SingleDimerPBC

    return [SingleDimerPBC(L=L, rho=10, N_MD=N_MD, seed=s, list_capacity=12000, precision=precision)
            for L, s in zip(boxes, seeds)]


def assert_dimers_equal(a, b):
    for f in SOLVENT_FIELDS:
        x, y = a.solvent.download(f), b.solvent.download(f)
        assert np.array_equal(x, y), f"solvent {f}: {np.sum(x != y)} entries differ"
    for f in COLLOID_FIELDS:
        assert np.array_equal(a.colloids.download(f), b.colloids.download(f)), f"colloid {f}"
    assert np.array_equal(a.cells.cell_count, b.cells.cell_count)
    assert np.array_equal(a.cells.cell_start, b.cells.cell_start)
    assert np.array_equal(a.cells.origin, b.cells.origin)
    la, na = a.neigh.download()
    lb, nb = b.neigh.download()
    assert np.array_equal(na, nb) and np.array_equal(la, lb)
    assert a.rng.step == b.rng.step
    assert a.n_extra_sorting == b.n_extra_sorting


@pytest.mark.parametrize("precision,N_MD,use_graph", [(64, 10, True), (64, 21, False), (32, 10, True), (64, 21, True)])
def test_batch_matches_call_by_call_driver(rm, precision, N_MD, use_graph):
    from rmpcdmd_b200.programs import DimerBatch

    boxes = [(10, 10, 10), (12, 11, 14), (16, 12, 12)]
    seeds = [3, 17, 101]
    ref = drivers(rm, boxes, seeds, precision, N_MD)
    mine = drivers(rm, boxes, seeds, precision, N_MD)
    batch = DimerBatch(mine, use_graph=use_graph)
    n_int = 3
    for d in ref:
        for _ in range(n_int):
            d.interval()
    batch.run(1)
    batch.run(n_int - 1)
    for r in range(len(mine)):
        batch.scatter(r)
        assert_dimers_equal(ref[r], mine[r])
    assert sum(d.n_extra_sorting for d in ref) > 0  # the device-decided re-sort was exercised
    rm.get_status()


def test_batch_continues_after_scatter(rm):
    """A scattered replica continues call by call exactly like its twin."""
    from rmpcdmd_b200.programs import DimerBatch

    ref = drivers(rm, [(10, 10, 10)], [5], 64, 10)
    mine = drivers(rm, [(10, 10, 10)], [5], 64, 10)
    batch = DimerBatch(mine)
    batch.run(1)
    batch.scatter(0)
    ref[0].interval()
    ref[0].interval()
    mine[0].interval()
    assert_dimers_equal(ref[0], mine[0])
    ob_r, ob_m = ref[0].observables(), mine[0].observables()
    assert ob_r["temperature"] == ob_m["temperature"]
    assert np.array_equal(ob_r["n_solvent"], ob_m["n_solvent"])


def test_batch_rejects_mixed_inputs(rm):
    from rmpcdmd_b200.programs import DimerBatch

    a = drivers(rm, [(10, 10, 10)], [1], 64, 10)
    b = drivers(rm, [(10, 10, 10)], [2], 32, 10)
    with pytest.raises(rm.RmpcdError):
        DimerBatch(a + b)
    c = drivers(rm, [(10, 10, 10)], [3], 64, 10)
    c[0].rng.step = 5
    with pytest.raises(rm.RmpcdError):
        DimerBatch(a + c)


@pytest.mark.parametrize("precision", [64, 32])
def test_every_engine_shape_gives_the_same_results(rm, precision):
    """The autotuner's choices (particles per tile, per thread, blocks per SM)
    only decide which thread handles which particle: every shape ends bit
    for bit where the default shape ends, the shape switched between
    intervals included."""
    from rmpcdmd_b200.programs import DimerBatch

    boxes, seeds = [(10, 10, 10), (12, 11, 14), (16, 12, 12)], [4, 18, 102]
    shapes = DimerBatch.shapes(precision)
    assert len(shapes) >= 8 and len({s["particles_per_tile"] for s in shapes}) >= 3
    ref = drivers(rm, boxes, seeds, precision, 10)
    batch_ref = DimerBatch(ref)
    batch_ref.run(2)
    for r in range(len(ref)):
        batch_ref.scatter(r)
    for k in range(len(shapes)):
        mine = drivers(rm, boxes, seeds, precision, 10)
        batch = DimerBatch(mine)
        batch.shape = k
        assert batch.shape == k
        batch.run(1)
        batch.shape = (k + 1) % len(shapes)
        batch.run(1)
        for r in range(len(mine)):
            batch.scatter(r)
            assert_dimers_equal(ref[r], mine[r])
    rm.get_status()


def test_engine_autotune_runs_real_intervals_and_remembers(rm):
    """rmpcd_dimer_batch_autotune advances the batch by real intervals (the
    state equals that of the same number of plain intervals), keeps the
    fastest shape, and a second batch of the same kind takes the remembered
    choice without running."""
    from rmpcdmd_b200.programs import DimerBatch

    boxes, seeds = [(12, 12, 12), (10, 10, 10)], [7, 8]
    tuned = drivers(rm, boxes, seeds, 32, 10)
    bt = DimerBatch(tuned)
    res = bt.autotune(1)
    shapes = DimerBatch.shapes(32)
    n = len(shapes)
    timed = [m for m in res["ms_per_interval"] if m > 0]
    # every tile and variant with one list entry per thread, then the best
    # of them with the other list setting
    first = [k for k, s in enumerate(shapes) if s["list_entries_per_thread"] == 1]
    assert all(res["ms_per_interval"][k] > 0 for k in first) and len(timed) == len(first) + 1
    assert all(m == -1 or m > 0 for m in res["ms_per_interval"])
    assert res["intervals_run"] == 2 * len(timed)
    assert 0 <= res["best"] < n and bt.shape == res["best"]
    assert res["ms_per_interval"][res["best"]] == min(timed)
    plain = drivers(rm, boxes, seeds, 32, 10)
    bp = DimerBatch(plain)
    bp.run(res["intervals_run"])
    for r in range(len(boxes)):
        bt.scatter(r)
        bp.scatter(r)
        assert_dimers_equal(tuned[r], plain[r])
    again = DimerBatch(drivers(rm, boxes, seeds, 32, 10))
    res2 = again.autotune(1)
    assert res2["intervals_run"] == 0 and res2["best"] == res["best"] and again.shape == res["best"]
    rm.get_status()
