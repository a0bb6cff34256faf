"""The committed golden fixtures (tests/golden/*.json) against the oracle that
wrote them: the 32^3 bulk fluid to its last checkpoint and the 32^3
single_dimer_pbc to its first (1,000 MD steps) are re-derived on the CPU and
must match digest for digest.  The 128^3 fixture takes the single-threaded
oracle about half an hour, so only its form is checked here; the GPU tests
compare the CUDA path with all of them."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_golden as G  # noqa: E402


def test_fixture_files_are_complete():
    for name, case in G.CASES.items():
        fx = G.load(name)
        assert fx["L"] == case["L"] and fx["seed"] == case["seed"]
        assert sorted(map(int, fx["checkpoint_states"])) == case["checkpoints"]
        N = int(np.prod(case["L"])) * case["rho"]
        for rec in fx["checkpoint_states"].values():
            assert rec["pos"]["shape"] == [N, 3] and rec["id"]["shape"] == [N]
            assert rec["cell_count"]["shape"] == rec["cell_start"]["shape"]
        if case["kind"] == "dimer":
            assert len(fx["colloids"]) == max(case["checkpoints"])


def test_bulk_32_fixture_from_the_oracle(oracle):
    fx = G.load("bulk_32")
    rec = G.make_bulk("bulk_32", G.CASES["bulk_32"])
    assert rec["checkpoint_states"] == fx["checkpoint_states"]


def test_dimer_32_fixture_from_the_oracle(oracle):
    fx = G.load("dimer_32")
    first = min(G.CASES["dimer_32"]["checkpoints"])
    rec = G.make_dimer("dimer_32", dict(G.CASES["dimer_32"], checkpoints=[first]))
    assert rec["colloids"] == fx["colloids"][:first]
    assert rec["checkpoint_states"][str(first)] == fx["checkpoint_states"][str(first)]


def test_oracle_is_thread_order_dependent_only_through_the_sort(oracle):
    """With one thread the oracle's sort places a cell's particles in
    ascending source order; that order is what the fixtures record (the
    reference's OpenMP sort, src/particle_system.f90:322-338, takes places by
    atomic capture and so varies with more threads)."""
    L = [6, 5, 4]
    r = np.random.default_rng(0)
    c = oracle.Cells(L)
    p = oracle.Particles(1200, 1)
    p.pos[:] = r.random((1200, 3)) * L
    p.species[:] = 1
    p.sort(c)
    for s in np.nonzero(c.cell_count > 1)[0]:
        a = c.cell_start[s] - 1
        ids = p.id[a : a + c.cell_count[s]]
        assert np.all(np.diff(ids) > 0)
