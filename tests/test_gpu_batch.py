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
