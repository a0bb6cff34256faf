"""Shared helpers for the GPU parity tests: build an oracle system and a CUDA
system with identical state, and compare their arrays."""
import numpy as np

SOLVENT_FIELDS = ("pos", "vel", "image", "id", "species", "flags")


def make_pair(rm, oracle, L, N, seed=0, precision=64, n_species=2, walls=False, species=None, origin=None,
              vel_scale=np.sqrt(1 / 3), mass=None, sorted_=True):
    L = np.asarray(L)
    rng = np.random.default_rng(seed)
    oc = oracle.Cells(L, 1.0, walls)
    op = oracle.Particles(N, n_species, mass)
    edges = oc.edges
    op.pos[:] = rng.random((N, 3)) * edges
    op.vel[:] = rng.normal(size=(N, 3)) * vel_scale
    op.species[:] = 1 if species is None else species
    if origin is not None:
        oc.origin = origin
    gc = rm.CellSystem(L, 1.0, walls)
    gp = rm.ParticleSystem(N, n_species, mass, precision)
    if origin is not None:
        gc.origin = origin
    upload(gp, op)
    if sorted_:
        op.sort(oc)
        gp.sort(gc)
    return (oc, op), (gc, gp)


def upload(gp, op, fields=("pos", "vel", "image", "id", "species", "flags")):
    for f in fields:
        gp.upload(f, getattr(op, f))


def assert_same(gp, op, fields=SOLVENT_FIELDS, exact=True, rtol=0.0, atol=0.0):
    for f in fields:
        a = gp.download(f)
        b = getattr(op, f)
        assert a.shape == b.shape, f"{f}: shape {a.shape} vs {b.shape}"
        if a.size == 0:
            continue
        if exact:
            bad = np.nonzero((a != b).reshape(len(a), -1).any(1))[0]
            assert bad.size == 0, f"{f}: {bad.size} rows differ, first {bad[:5]}: gpu {a[bad[:3]]} oracle {b[bad[:3]]}"
        else:
            np.testing.assert_allclose(a, b, rtol=rtol, atol=atol, err_msg=f)


def assert_cells_same(gc, oc):
    assert np.array_equal(gc.cell_count, oc.cell_count), "cell_count"
    assert np.array_equal(gc.cell_start, oc.cell_start), "cell_start"
