"""Bit-exact parity at the benchmark sizes, against golden fixtures that the
oracle wrote (tests/golden/make_golden.py, one oracle thread).

* bulk fluid 128^3 at density 10 (20,971,520 particles, the headline
  workload) after 5 and 100 collision steps, through rmpcd_bulk_run (fused
  schedule, every FP64 tile shape) and, for the first 5, through the
  procedure entry points called one by one (simple_mpcd_step ->
  mpcd_stream_periodic -> random_shift -> sort, test/setup_bulk_decay.f90:112-121);
* bulk fluid 32^3 after 5 and 100 collision steps;
* single_dimer_pbc at 32^3 (programs/single_dimer_pbc.f90:303-445) for 10
  intervals (1,000 MD steps) and 100 intervals (100 collision steps), through
  the call-by-call driver and through the replica engine: the colloid
  trajectory after every interval and every solvent array, the cell counts
  and starts and the neighbor lists at the checkpoints;
* single_dimer_pbc at 96^3 for 2 intervals in the replica engine;
* n_colloids_pbc at 128^3 with 200 colloids (rmpcd_ncolloids_run): one
  thermostatted interval and one production interval.

Every array is compared by its SHA-256 digest, so a match is equality bit for
bit; on a mismatch the sampled rows say where the arrays part."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = G.SOLVENT


def check_state(rec: dict, arrays: dict, count, start, origin, what: str):
    bad = []
    for f, a in arrays.items():
        r = rec[f]
        c = G.canonical(a)
        assert list(c.shape) == r["shape"], f"{what} {f}: shape {c.shape} vs {r['shape']}"
        if G.digest(c) != r["sha256"]:
            rows = {i: (c[int(i)].tolist(), v) for i, v in r["rows"].items() if c[int(i)].tolist() != v}
            bad.append(f"{f} (sampled rows that differ, gpu vs oracle: {dict(list(rows.items())[:3])})")
    if G.digest(count) != rec["cell_count"]["sha256"]:
        bad.append("cell_count")
    if G.digest(start) != rec["cell_start"]["sha256"]:
        bad.append("cell_start")
    if [float(x) for x in origin] != rec["origin"]:
        bad.append(f"origin {list(origin)} vs {rec['origin']}")
    assert not bad, f"{what}: differs from the oracle in " + "; ".join(bad)


# ------------------------------------------------------------------ bulk fluid
def bulk_setup(rm, case):
    """rmpcdmd_b200.programs.bulk_fluid's set-up, to the first interval."""
    L = np.asarray(case["L"])
    N = int(L.prod()) * case["rho"]
    cells = rm.CellSystem(L, 1.0)
    p = rm.ParticleSystem(N, 1, None, rm.FP64)
    p.random_placement(cells.edges, seed=case["seed"])
    p.maxwell(1.0 / 3.0, case["seed"])
    p.species = 1
    rng = rm.Rng(case["seed"])
    cells.random_shift(rng)
    p.sort(cells)
    return p, cells, rng


def bulk_check(p, cells, rec, what):
    arrays = {f: p.download(f) for f in FIELDS}
    check_state(rec, arrays, cells.cell_count, cells.cell_start, cells.origin, what)


def run_bulk_golden(rm, name, shape=None):
    fx = G.load(name)
    if shape is not None:
        old = rm.bulk_shape(rm.FP64)
        rm.set_bulk_shape(rm.FP64, shape)
    try:
        p, cells, rng = bulk_setup(rm, fx)
        done = 0
        for k in fx["checkpoints"]:
            rm.bulk_run(p, cells, rng, 1.0, k - done)
            done = k
            assert rng.step == 1 + 2 * done
            bulk_check(p, cells, fx["checkpoint_states"][str(k)], f"{name} after {k} collisions")
    finally:
        if shape is not None:
            rm.set_bulk_shape(rm.FP64, old)
    rm.get_status()


def test_bulk_32_fused_100_collisions(rm):
    run_bulk_golden(rm, "bulk_32")


def test_bulk_128_fused_100_collisions(rm):
    run_bulk_golden(rm, "bulk_128")


@pytest.mark.parametrize("shape", [1, 2])
def test_bulk_128_other_tile_shapes(rm, shape):
    if shape >= len(rm.bulk_shapes(rm.FP64)):
        pytest.skip("no such FP64 tile shape")
    run_bulk_golden(rm, "bulk_128", shape)


def test_bulk_128_call_by_call_5_collisions(rm):
    """The interval as separate procedure calls, as test/setup_bulk_decay.f90
    issues them, against the same golden state after 5 collisions."""
    fx = G.load("bulk_128")
    p, cells, rng = bulk_setup(rm, fx)
    for _ in range(5):
        rm.simple_mpcd_step(p, cells, rng)
        rm.mpcd_stream_periodic(p, cells, 1.0)
        cells.random_shift(rng)
        p.sort(cells)
    bulk_check(p, cells, fx["checkpoint_states"]["5"], "bulk_128 call by call after 5 collisions")
    rm.get_status()


# ------------------------------------------------------------- single dimer
def dimer_check(d, rec, what):
    arrays = {f: d.solvent.download(f) for f in FIELDS + ("force",)}
    check_state(rec, arrays, d.cells.cell_count, d.cells.cell_start, d.cells.origin, what)
    lst, n = d.neigh.download()
    assert [int(x) for x in n] == rec["lists"]["n"], f"{what}: list lengths"
    for i in range(len(n)):
        assert G.digest(lst[i, : n[i]]) == rec["lists"]["sha256"][i], f"{what}: neighbor list of colloid {i + 1}"
    assert d.n_extra_sorting == rec["n_extra_sorting"], f"{what}: extra sorts"
    assert d.rng.step == rec["rng_step"], f"{what}: random-number step"


def check_colloids(d, frame, what):
    for f in ("pos", "vel", "force"):
        a = d.colloids.download(f)
        assert a.tolist() == frame[f], f"{what}: colloid {f} {a.tolist()} vs oracle {frame[f]}"


def test_single_dimer_32_call_by_call_100_intervals(rm):
    from rmpcdmd_b200.programs import SingleDimerPBC

    fx = G.load("dimer_32")
    d = SingleDimerPBC(**G.dimer_kwargs(fx))
    for i in range(1, max(fx["checkpoints"]) + 1):
        d.interval()
        check_colloids(d, fx["colloids"][i - 1], f"dimer_32 interval {i}")
        if str(i) in fx["checkpoint_states"]:
            dimer_check(d, fx["checkpoint_states"][str(i)], f"dimer_32 after {i} intervals")
    rm.get_status()


def test_single_dimer_32_engine_100_intervals(rm):
    """The same run in the replica engine (one replica, one captured graph per
    interval), stopped at every checkpoint."""
    from rmpcdmd_b200.programs import DimerBatch, SingleDimerPBC

    fx = G.load("dimer_32")
    d = SingleDimerPBC(**G.dimer_kwargs(fx))
    batch = DimerBatch([d])
    done = 0
    for k in fx["checkpoints"]:
        batch.run(k - done)
        done = k
        g = batch.scatter(0)
        check_colloids(g, fx["colloids"][k - 1], f"dimer_32 engine interval {k}")
        dimer_check(g, fx["checkpoint_states"][str(k)], f"dimer_32 engine after {k} intervals")
    rm.get_status()


def test_single_dimer_96_engine_2_intervals(rm):
    """The large-box dimer (96^3, 8,847,360 solvent particles) in the replica
    engine against the oracle's run of the same program."""
    from rmpcdmd_b200.programs import DimerBatch, SingleDimerPBC

    fx = G.load("dimer_96")
    d = SingleDimerPBC(**G.dimer_kwargs(fx))
    batch = DimerBatch([d])
    done = 0
    for k in fx["checkpoints"]:
        batch.run(k - done)
        done = k
        g = batch.scatter(0)
        check_colloids(g, fx["colloids"][k - 1], f"dimer_96 engine interval {k}")
        dimer_check(g, fx["checkpoint_states"][str(k)], f"dimer_96 engine after {k} intervals")
    rm.get_status()


def test_n_colloids_128_native_loop(rm):
    """n_colloids_pbc at its configuration size (128^3, 200 colloids): one
    thermostatted and one production interval of rmpcd_ncolloids_run against
    the oracle's run of the program."""
    from rmpcdmd_b200.programs import NColloidsPBC

    fx = G.load("ncolloids_128")
    g = NColloidsPBC(**G.ncolloids_kwargs(fx))
    for k, step in ((1, lambda: g.thermalise(1)), (2, lambda: g.run(1))):
        step()
        rec = fx["checkpoint_states"][str(k)]
        what = f"ncolloids_128 checkpoint {k}"
        arrays = {f: g.solvent.download(f) for f in FIELDS + ("force",)}
        check_state(rec, arrays, g.cells.cell_count, g.cells.cell_start, g.cells.origin, what)
        for f in ("pos", "vel", "force", "image"):
            assert g.colloids.download(f).tolist() == rec["colloids"][f], f"{what}: colloid {f}"
        lst, n = g.neigh.download()
        assert [int(x) for x in n] == rec["lists"]["n"], f"{what}: list lengths"
        for i in range(len(n)):
            assert G.digest(lst[i, : n[i]]) == rec["lists"]["sha256"][i], f"{what}: list of colloid {i + 1}"
        assert g.n_extra_sorting == rec["n_extra_sorting"] and g.rng.step == rec["rng_step"], what
    rm.get_status()
