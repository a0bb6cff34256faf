"""Rigid-body colloids (src/md.f90:321-700): multi-link RATTLE, the elastic
network and the quaternion rigid body.

CPU tests pin the oracle to the properties the routines exist for
(constraints met to the requested precision, momentum and energy bookkeeping,
rigid motion, angular momentum conservation); GPU tests require the CUDA
path to equal the oracle bit for bit.  The bodies are bead clusters placed
across a periodic boundary, linked pairwise within 2.5 sigma, as the Janus
bodies of programs/single_body.f90 are.
"""
import numpy as np
import pytest

EDGES = np.array([12.0, 10.0, 14.0])


def cluster(n=12, seed=3, center=(11.5, 0.3, 7.0)):
    """n beads inside a sphere of radius 1.6 around center (wrapped into the
    box), two species, and the links between beads closer than 2.5."""
    r = np.random.default_rng(seed)
    pts = []
    while len(pts) < n:
        x = r.uniform(-1.6, 1.6, 3)
        if np.linalg.norm(x) < 1.6 and all(np.linalg.norm(x - p) > 0.6 for p in pts):
            pts.append(x)
    rel = np.array(pts)
    links = [(a + 1, b + 1) for a in range(n) for b in range(a + 1, n) if np.linalg.norm(rel[a] - rel[b]) < 2.5]
    dist = np.array([np.linalg.norm(rel[a - 1] - rel[b - 1]) for a, b in links])
    pos = np.mod(rel + np.asarray(center), EDGES)
    species = (np.arange(n) % 2 + 1).astype(np.int32)
    return pos, rel, np.array(links, np.int32), dist, species


def make_oracle(oracle, n, pos, species, mass=(2.0, 3.5)):
    p = oracle.Particles(n, 2, list(mass))
    p.pos[:] = pos
    p.species[:] = species
    return p


def min_image(d):
    return d - EDGES * np.round(d / EDGES)


def link_error(pos, links, dist):
    d = min_image(pos[links[:, 0] - 1] - pos[links[:, 1] - 1])
    return np.abs(np.linalg.norm(d, axis=1) - dist).max()


def test_rattle_body_meets_the_constraints(oracle):
    n = 12
    pos, rel, links, dist, sp = cluster(n)
    p = make_oracle(oracle, n, pos, sp)
    r = np.random.default_rng(4)
    p.pos_rattle[:] = p.pos
    p.vel[:] = r.normal(size=(n, 3)) * 0.3
    dt = 0.01
    p.pos[:] = np.mod(p.pos + dt * p.vel + r.normal(size=(n, 3)) * 1e-3, EDGES)
    assert link_error(p.pos, links, dist) > 1e-4
    it = oracle.rattle_body_pos(p, links, dist, dt, EDGES, 1e-10)
    assert 1 < it < 1001
    assert link_error(p.pos, links, dist) < 1e-10
    it = oracle.rattle_body_vel(p, links, dist, dt, EDGES, 1e-12)
    assert 1 <= it < 1001
    s = min_image(p.pos[links[:, 0] - 1] - p.pos[links[:, 1] - 1])
    dv = p.vel[links[:, 0] - 1] - p.vel[links[:, 1] - 1]
    assert np.abs((dv * s).sum(1)).max() < 1e-10
    # momentum is exchanged along the links only: total momentum unchanged
    m = np.where(sp == 1, 2.0, 3.5)[:, None]
    p2 = make_oracle(oracle, n, p.pos.copy(), sp)
    p2.vel[:] = r.normal(size=(n, 3))
    mom = (m * p2.vel).sum(0)
    oracle.rattle_body_vel(p2, links, dist, dt, EDGES, 1e-12)
    assert np.allclose((m * p2.vel).sum(0), mom, atol=1e-12)


def test_elastic_network_is_minus_the_gradient(oracle):
    n = 8
    pos, rel, links, dist, sp = cluster(n, seed=5)
    r = np.random.default_rng(6)
    p = make_oracle(oracle, n, np.mod(pos + r.normal(size=(n, 3)) * 0.05, EDGES), sp)
    k = 7.0
    e = oracle.elastic_network(p, links, dist, k, EDGES)
    f = p.force.copy()
    assert np.allclose(f.sum(0), 0, atol=1e-12)
    h = 1e-6
    for i in (0, 3):
        for c in range(3):
            q = make_oracle(oracle, n, p.pos.copy(), sp)
            q.pos[i, c] += h
            ep = oracle.elastic_network(q, links, dist, k, EDGES)
            q = make_oracle(oracle, n, p.pos.copy(), sp)
            q.pos[i, c] -= h
            em = oracle.elastic_network(q, links, dist, k, EDGES)
            assert abs(-(ep - em) / (2 * h) - f[i, c]) < 1e-5
    d = np.linalg.norm(min_image(p.pos[links[:, 0] - 1] - p.pos[links[:, 1] - 1]), axis=1)
    assert abs(e - (k * (d - dist) ** 2 / 2).sum()) < 1e-12


def rigid_setup(oracle, n=10, seed=7):
    pos, rel, links, dist, sp = cluster(n, seed=seed)
    p = make_oracle(oracle, n, pos, sp)
    p.image[:] = np.floor((rel + np.array([11.5, 0.3, 7.0])) / EDGES).astype(np.int32)
    return p


def test_rigid_body_free_rotation(oracle):
    n = 10
    p = rigid_setup(oracle, n)
    body = oracle.RigidBody(p, 1, n, EDGES)
    st = body.state()
    m = np.where(p.species == 1, 2.0, 3.5)
    unwrapped = p.pos + p.image * EDGES
    assert np.isclose(st["mass"], m.sum())
    assert np.allclose(st["pos"], (m[:, None] * unwrapped).sum(0) / m.sum())
    assert np.allclose(st["q"], [1, 0, 0, 0])
    # spin the body: angular momentum L, no force or torque
    body.st[14:17] = [0.8, -0.3, 0.5]
    L0 = body.st[14:17].copy()
    pair = lambda x: np.linalg.norm(min_image(x[:, None, :] - x[None, :, :]), axis=2)
    d0 = pair(p.pos)
    dt = 0.01
    for _ in range(50):
        body.vv1(p, dt, 1e-12, EDGES)
        p.force[:] = 0
        body.compute_force_torque(p)
        body.vv2(p, dt)
    st = body.state()
    assert np.allclose(st["L"], L0, atol=1e-13)
    assert abs(np.linalg.norm(st["q"]) - 1) < 1e-14
    assert not np.allclose(st["q"], [1, 0, 0, 0])  # it turned
    assert np.abs(pair(p.pos) - d0).max() < 1e-10  # rigidly
    # bead velocities are those of the rigid motion v + omega x r
    omega = st["omega_body"]
    assert np.all(np.isfinite(omega)) and np.linalg.norm(omega) > 0


# ---------------------------------------------------------------------------
# GPU parity
# ---------------------------------------------------------------------------
def upload_pair(rm, oracle, n, pos, sp, mass=(2.0, 3.5)):
    p = make_oracle(oracle, n, pos, sp, mass)
    g = rm.ParticleSystem(n, 2, list(mass))
    g.upload("pos", p.pos)
    g.upload("species", p.species)
    return p, g


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [1e-10, 1e-3])
def test_rattle_body_gpu_equals_oracle(rm, oracle, precision):
    n = 12
    pos, rel, links, dist, sp = cluster(n)
    p, g = upload_pair(rm, oracle, n, pos, sp)
    r = np.random.default_rng(4)
    p.pos_rattle[:] = p.pos
    p.vel[:] = r.normal(size=(n, 3)) * 0.3
    dt = 0.01
    p.pos[:] = np.mod(p.pos + dt * p.vel + r.normal(size=(n, 3)) * 1e-3, EDGES)
    for f in ("pos", "vel", "pos_rattle"):
        g.upload(f, getattr(p, f))
    it_o = oracle.rattle_body_pos(p, links, dist, dt, EDGES, precision)
    it_g = rm.rattle_body_pos(g, links, dist, dt, EDGES, precision)
    assert it_g == it_o
    for f in ("pos", "vel", "pos_rattle"):
        assert np.array_equal(g.download(f), getattr(p, f)), f
    it_o = oracle.rattle_body_vel(p, links, dist, dt, EDGES, precision * 1e-2)
    it_g = rm.rattle_body_vel(g, links, dist, dt, EDGES, precision * 1e-2)
    assert it_g == it_o
    for f in ("pos", "vel"):
        assert np.array_equal(g.download(f), getattr(p, f)), f


@pytest.mark.gpu
def test_rattle_body_not_converging_reports_1001(rm, oracle):
    n = 6
    pos, rel, links, dist, sp = cluster(n, seed=9)
    p, g = upload_pair(rm, oracle, n, pos, sp)
    p.pos_rattle[:] = p.pos
    p.pos[:] = np.mod(p.pos + np.random.default_rng(2).normal(size=(n, 3)) * 1e-3, EDGES)
    for f in ("pos", "pos_rattle"):
        g.upload(f, getattr(p, f))
    # precision 0 is never reached: the loop runs its 1000 sweeps
    assert oracle.rattle_body_pos(p, links, dist, 0.01, EDGES, 0.0) == 1001
    assert rm.rattle_body_pos(g, links, dist, 0.01, EDGES, 0.0) == 1001
    assert np.array_equal(g.download("pos"), p.pos)


@pytest.mark.gpu
def test_elastic_network_gpu_equals_oracle(rm, oracle):
    n = 8
    pos, rel, links, dist, sp = cluster(n, seed=5)
    r = np.random.default_rng(6)
    p, g = upload_pair(rm, oracle, n, np.mod(pos + r.normal(size=(n, 3)) * 0.05, EDGES), sp)
    p.force[:] = r.normal(size=(n, 3))
    g.upload("force", p.force)
    e_o = oracle.elastic_network(p, links, dist, 7.0, EDGES)
    e_g = rm.elastic_network(g, links, dist, 7.0, EDGES)
    assert e_g == e_o
    assert np.array_equal(g.download("force"), p.force)


@pytest.mark.gpu
def test_rigid_body_gpu_equals_oracle(rm, oracle):
    n = 10
    p = rigid_setup(oracle, n)
    r = np.random.default_rng(8)
    p.vel[:] = r.normal(size=(n, 3)) * 0.1
    g = rm.ParticleSystem(n, 2, [2.0, 3.5])
    for f in ("pos", "vel", "image", "species"):
        g.upload(f, getattr(p, f))
    bo = oracle.RigidBody(p, 1, n, EDGES)
    bg = rm.RigidBody(g, 1, n, EDGES)
    so, sg = bo.state(), bg.state()
    for k in so:
        assert np.array_equal(np.asarray(sg[k]), np.asarray(so[k])), k
    assert np.array_equal(bg.pos_body(), bo.pos_body)
    bo.st[14:17] = [0.8, -0.3, 0.5]
    bg.set_state(L=[0.8, -0.3, 0.5])
    dt = 0.01
    for step in range(20):
        bo.vv1(p, dt, 1e-12, EDGES)
        bg.vv1(g, dt, 1e-12, EDGES)
        # a force field on the beads, the same on both sides
        f = np.cos(np.arange(3 * n).reshape(n, 3) * 0.7 + step) * 0.05
        p.force[:] = f
        g.upload("force", f)
        bo.compute_force_torque(p)
        bg.compute_force_torque(g)
        bo.vv2(p, dt)
        bg.vv2(g, dt)
    so, sg = bo.state(), bg.state()
    for k in so:
        assert np.array_equal(np.asarray(sg[k]), np.asarray(so[k])), k
    assert np.array_equal(g.download("pos"), p.pos)
    assert np.array_equal(g.download("vel"), p.vel)
