"""Checkpoint / resume at an interval boundary.

The reference has no restart files (it writes a final snapshot only); a run
here can be stopped after any MPCD interval and resumed bit for bit from one
``.npz`` archive holding the particle arrays in their current (sorted) order,
the grid origin, the random-number counter and the program's counters.

At an interval boundary the solvent is sorted for the current origin (the
interval ends with its sort; the collision and refuelling do not move
particles), so on loading a sort is the identity permutation and rebuilds the
cell counts and starts, and the neighbor list and ``is_md`` / ``is_reac``
flags are rebuilt from the same positions as the run built them.
"""
from __future__ import annotations

import numpy as np

from . import api as A

SOLVENT_FIELDS = ("pos", "vel", "image", "id", "species", "flags", "force", "force_old")
COLLOID_FIELDS = ("pos", "vel", "image", "id", "species", "flags", "force", "force_old")


def _dump(prefix: str, p: A.ParticleSystem, fields, out: dict):
    for f in fields:
        out[f"{prefix}/{f}"] = p.download(f)


def _load(prefix: str, p: A.ParticleSystem, fields, data):
    for f in fields:
        p.upload(f, data[f"{prefix}/{f}"])


# ---------------------------------------------------------------- bulk fluid
def save_bulk(path, p: A.ParticleSystem, cells: A.CellSystem, rng: A.Rng) -> None:
    """A bulk fluid after rmpcd_bulk_run (sorted for the final origin)."""
    out = {"kind": np.asarray("bulk"), "L": cells.L, "precision": np.asarray(p.precision),
           "n_species": np.asarray(p.n_species), "origin": cells.origin,
           "rng": np.asarray([rng.seed, rng.step], dtype=np.uint64)}
    _dump("solvent", p, ("pos", "vel", "image", "id", "species", "flags"), out)
    np.savez(path, **out)


def load_bulk(path):
    """(ParticleSystem, CellSystem, Rng) as saved by save_bulk."""
    d = np.load(path)
    if str(d["kind"]) != "bulk":
        raise ValueError(f"{path}: not a bulk-fluid checkpoint")
    cells = A.CellSystem(d["L"], 1.0)
    n = len(d["solvent/pos"])
    p = A.ParticleSystem(n, int(d["n_species"]), None, int(d["precision"]))
    _load("solvent", p, ("pos", "vel", "image", "id", "species", "flags"), d)
    cells.origin = d["origin"]
    p.sort(cells)
    seed, step = (int(x) for x in d["rng"])
    rng = A.Rng(seed, step)
    return p, cells, rng


# ------------------------------------------------------- single_dimer_pbc
def save_dimer(path, g) -> None:
    """A programs.SingleDimerPBC between two intervals."""
    out = {"kind": np.asarray("single_dimer_pbc"), "init": np.asarray(repr(g._init_kwargs)),
           "origin": g.cells.origin, "rng": np.asarray([g.rng.seed, g.rng.step], dtype=np.uint64),
           "counters": np.asarray([g.n_extra_sorting, g.md_steps]),
           "energies": np.asarray([np.nan if g.e1 is None else g.e1, np.nan if g.e2 is None else g.e2])}
    _dump("solvent", g.solvent, SOLVENT_FIELDS, out)
    _dump("colloids", g.colloids, COLLOID_FIELDS, out)
    np.savez(path, **out)


def load_dimer(path):
    """The programs.SingleDimerPBC saved by save_dimer, ready for its next interval."""
    from .programs import SingleDimerPBC

    d = np.load(path)
    if str(d["kind"]) != "single_dimer_pbc":
        raise ValueError(f"{path}: not a single_dimer_pbc checkpoint")
    g = SingleDimerPBC(**_kwargs(d))
    _restore_program(g, d)
    g.neigh.update_list(g.colloids, g.solvent, g.max_cut + g.skin, g.cells, g.solvent_colloid_lj)
    g.solvent.copy_pos_old()
    g.colloids.copy_pos_old()
    g.n_extra_sorting, g.md_steps = (int(x) for x in d["counters"])
    g.e1, g.e2 = (float(x) for x in d["energies"])
    return g


# --------------------------------------------------------- n_colloids_pbc
def save_ncolloids(path, g) -> None:
    """A programs.NColloidsPBC between two intervals."""
    out = {"kind": np.asarray("n_colloids_pbc"), "init": np.asarray(repr(g._init_kwargs)),
           "origin": g.cells.origin, "rng": np.asarray([g.rng.seed, g.rng.step], dtype=np.uint64),
           "counters": np.asarray([g.t, g.last_sort, g.n_extra_sorting]),
           "energies": np.asarray([g.e1, g.e2])}
    _dump("solvent", g.solvent, SOLVENT_FIELDS, out)
    _dump("colloids", g.colloids, COLLOID_FIELDS, out)
    np.savez(path, **out)


def load_ncolloids(path):
    from .programs import NColloidsPBC

    d = np.load(path)
    if str(d["kind"]) != "n_colloids_pbc":
        raise ValueError(f"{path}: not an n_colloids_pbc checkpoint")
    g = NColloidsPBC(**_kwargs(d))
    _restore_program(g, d)
    g.neigh.update_list(g.colloids, g.solvent, g.radius, g.cells)
    g.solvent.copy_pos_old()
    g.colloids.copy_pos_old()
    g.t, g.last_sort, g.n_extra_sorting = (int(x) for x in d["counters"])
    g.e1, g.e2 = (float(x) for x in d["energies"])
    return g


def _kwargs(d) -> dict:
    import ast

    return ast.literal_eval(str(d["init"]))


def _restore_program(g, d):
    _load("solvent", g.solvent, SOLVENT_FIELDS, d)
    _load("colloids", g.colloids, COLLOID_FIELDS, d)
    g.cells.origin = d["origin"]
    g.solvent.sort(g.cells)
    seed, step = (int(x) for x in d["rng"])
    g.rng.seed, g.rng.step = seed, step
