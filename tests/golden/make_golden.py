"""Writes the golden fixtures of the full-size parity tests from the oracle.

The oracle (the FP64 C restatement under oracle/) is run on the workloads of
the benchmark configurations, and what the tests compare is stored compactly:
a SHA-256 digest of every particle array and of the cell counts and starts at
chosen interval counts, a few sampled rows of each array (to show where a
mismatch lies), the grid origin, and -- for the dimer -- the whole colloid
trajectory (position, velocity, force after every interval) and the neighbor
lists.  The GPU tests (tests/test_gpu_golden.py) run the CUDA path from the
same seeds and require every digest to match, i.e. bit-exact results, without
running the oracle themselves; tests/test_golden_fixtures.py re-derives the
smaller fixtures from the oracle on the CPU.

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py bulk_32    # one of them

The oracle runs on one thread.  That is the reference's own deterministic
order: its sort places each cell's particles through an OpenMP atomic capture
(src/particle_system.f90:322-338), so with more than one thread the order
inside a cell -- and everything downstream of it -- varies from run to run.

Cases (all plain FP64, density 10, kT = 1/3, alpha = pi/2, tau = 1):
  bulk_128  128^3 cells, 20,971,520 particles: the bulk loop of
            test/setup_bulk_decay.f90:112-121 (simple_mpcd_step ->
            mpcd_stream_periodic -> random_shift -> sort), checkpoints after 5
            and after 100 collision steps.
  bulk_32   32^3 cells, 327,680 particles, the same loop, checkpoints after 5
            and 100 collision steps.
  dimer_32  programs/single_dimer_pbc.f90 with its parameters (sigma 2, bond
            4.5, N_MD = 100, dt = 0.01, probability 1), 32^3 cells, 327,680
            solvent particles: 10 intervals (1,000 MD steps) and 100 intervals
            (100 collision steps, 10,000 MD steps).
  dimer_96  the same program in a 96^3 box (8,847,360 solvent particles, the
            large-box dimer configuration): 1 and 2 intervals.
  ncolloids_128  programs/n_colloids_pbc.f90: 200 passive colloids (sigma 3)
            in 128^3 cells (20,971,520 solvent particles, no volume
            correction), one thermostatted interval (MPC-AT, lazy cell-wise
            streaming) and one production interval.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

SOLVENT = ("pos", "vel", "image", "id", "species", "flags")
N_SAMPLES = 8

CASES = {
    "bulk_128": dict(kind="bulk", L=[128, 128, 128], rho=10, seed=1, checkpoints=[5, 100]),
    "bulk_32": dict(kind="bulk", L=[32, 32, 32], rho=10, seed=3, checkpoints=[5, 100]),
    "dimer_32": dict(kind="dimer", L=[32, 32, 32], rho=10, N_MD=100, seed=1, list_capacity=6000,
                     checkpoints=[10, 100]),
    "dimer_96": dict(kind="dimer", L=[96, 96, 96], rho=10, N_MD=100, seed=5, list_capacity=6000,
                     checkpoints=[1, 2]),
    "ncolloids_128": dict(kind="ncolloids", L=[128, 128, 128], rho=10, N_MD=100, N_colloids=200, seed=7,
                          checkpoints=[1, 2]),
}


def canonical(a: np.ndarray) -> np.ndarray:
    """Arrays are hashed as little-endian float64 / int32 in row order."""
    a = np.asarray(a)
    dt = "<f8" if a.dtype.kind == "f" else "<i4"
    return np.ascontiguousarray(a, dtype=dt)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(canonical(a).tobytes()).hexdigest()


def sample_rows(n: int, seed: int) -> list[int]:
    r = np.random.default_rng(seed)
    return sorted({0, n - 1, *r.integers(0, n, N_SAMPLES - 2).tolist()})


def array_record(a: np.ndarray, rows: list[int]) -> dict:
    c = canonical(a)
    return {"sha256": digest(c), "shape": list(c.shape), "rows": {str(i): c[i].tolist() for i in rows}}


def state_record(arrays: dict, count, start, origin, rows) -> dict:
    rec = {k: array_record(v, rows) for k, v in arrays.items()}
    rec["cell_count"] = array_record(count, [])
    rec["cell_start"] = array_record(start, [])
    rec["origin"] = [float(x) for x in origin]
    return rec


def lists_record(lst: np.ndarray, n: np.ndarray) -> dict:
    rows = [np.ascontiguousarray(lst[i, : n[i]], np.int32) for i in range(len(n))]
    return {"n": [int(x) for x in n], "sha256": [digest(r) for r in rows]}


# ------------------------------------------------------------------ bulk fluid
def bulk_oracle(case: dict, O):
    """Generator of (intervals done, particles, cells): the set-up of
    rmpcdmd_b200.programs.bulk_fluid (random placement and Maxwell velocities
    from the seed, all species A, one random shift, sort), then the loop."""
    L = np.asarray(case["L"])
    N = int(L.prod()) * case["rho"]
    seed = case["seed"]
    c = O.Cells(L)
    p = O.Particles(N, 1)
    O.random_placement(p, c.edges, seed)
    O.maxwell_velocities(p, 1.0 / 3.0, seed)
    p.species[:] = 1
    c.random_shift(seed, 0)
    step = 1
    p.sort(c)
    done = 0
    for k in case["checkpoints"]:
        O.bulk_run(p, c, k - done, 1.0, seed, step)
        step += 2 * (k - done)
        done = k
        yield done, p, c


def make_bulk(name: str, case: dict) -> dict:
    from oracle import oracle as O

    out = dict(case, name=name, checkpoint_states={})
    L = np.asarray(case["L"])
    N = int(L.prod()) * case["rho"]
    rows = sample_rows(N, case["seed"])
    for done, p, c in bulk_oracle(case, O):
        arrays = {f: getattr(p, f) for f in SOLVENT}
        out["checkpoint_states"][str(done)] = state_record(arrays, c.cell_count, c.cell_start, c.origin, rows)
        print(f"  {name}: {done} intervals", flush=True)
    return out


# ------------------------------------------------------------- single dimer
def dimer_kwargs(case: dict) -> dict:
    return dict(L=tuple(case["L"]), rho=case["rho"], N_MD=case["N_MD"], seed=case["seed"],
                list_capacity=case["list_capacity"])


def dimer_state(d, rows) -> dict:
    arrays = {f: getattr(d.s, f) for f in SOLVENT + ("force",)}
    rec = state_record(arrays, d.cells.cell_count, d.cells.cell_start, d.cells.origin, rows)
    rec["lists"] = lists_record(d.nl.list, d.nl.n)
    rec["n_extra_sorting"] = int(d.n_extra_sorting)
    rec["rng_step"] = int(d.step)
    return rec


def make_dimer(name: str, case: dict) -> dict:
    from oracle.programs import SingleDimerPBC as OD

    d = OD(**dimer_kwargs(case))
    rows = sample_rows(d.N, case["seed"])
    out = dict(case, name=name, checkpoint_states={}, colloids=[])
    for i in range(1, max(case["checkpoints"]) + 1):
        d.interval()
        out["colloids"].append({"pos": d.c.pos.tolist(), "vel": d.c.vel.tolist(), "force": d.c.force.tolist()})
        if i in case["checkpoints"]:
            out["checkpoint_states"][str(i)] = dimer_state(d, rows)
            print(f"  {name}: {i} intervals", flush=True)
    return out


# ------------------------------------------------------------ n colloids
def ncolloids_kwargs(case: dict) -> dict:
    return dict(L=tuple(case["L"]), rho=case["rho"], N_MD=case["N_MD"], N_colloids=case["N_colloids"],
                seed=case["seed"], volume_correction=False)


def ncolloids_state(d, rows) -> dict:
    arrays = {f: getattr(d.s, f) for f in SOLVENT + ("force",)}
    rec = state_record(arrays, d.cells.cell_count, d.cells.cell_start, d.cells.origin, rows)
    rec["lists"] = lists_record(d.nl.list, d.nl.n)
    rec["colloids"] = {f: getattr(d.c, f).tolist() for f in ("pos", "vel", "force", "image")}
    rec["n_extra_sorting"] = int(d.n_extra_sorting)
    rec["rng_step"] = int(d.step)
    return rec


def make_ncolloids(name: str, case: dict) -> dict:
    """Checkpoint 1: one thermostatted interval (thermalise(1)); checkpoint 2:
    one production interval after it (run(1))."""
    from oracle.programs import NColloidsPBC as ON

    d = ON(**ncolloids_kwargs(case))
    rows = sample_rows(d.N, case["seed"])
    out = dict(case, name=name, checkpoint_states={})
    d.thermalise(1)
    out["checkpoint_states"]["1"] = ncolloids_state(d, rows)
    print(f"  {name}: thermalised", flush=True)
    d.run(1)
    out["checkpoint_states"]["2"] = ncolloids_state(d, rows)
    print(f"  {name}: 1 production interval", flush=True)
    return out


def make(name: str) -> dict:
    case = CASES[name]
    if case["kind"] == "bulk":
        return make_bulk(name, case)
    if case["kind"] == "ncolloids":
        return make_ncolloids(name, case)
    return make_dimer(name, case)


def path_of(name: str) -> Path:
    return HERE / f"{name}.json"


def load(name: str) -> dict:
    return json.loads(path_of(name).read_text())


def main(argv) -> int:
    from oracle import oracle as O

    O.set_threads(1)
    names = argv or list(CASES)
    for name in names:
        t = time.time()
        rec = make(name)
        rec["generated_by"] = "tests/golden/make_golden.py"
        path_of(name).write_text(json.dumps(rec, indent=1) + "\n")
        print(f"{name}: {time.time() - t:.1f} s -> {path_of(name).name}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
