"""Full-size runs of the configurations the parity tests check in small:
properties that hold at any size -- id permutations, sorted Morton codes
with a stable permutation, momentum of a system started at rest, the FP64
force error, bit-for-bit determinism, and ensemble instances equal to
their standalone runs."""
import numpy as np
import pytest

from conftest import same_bits

pytestmark = pytest.mark.gpu


def check_state(s, n):
    assert np.array_equal(np.sort(s["id"]), np.arange(n))
    for f in ("px", "py", "vx", "vy", "ax", "ay"):
        assert np.isfinite(s[f]).all(), f


def check_morton(sim):
    codes, perm = sim.morton()
    n = len(codes)
    assert np.array_equal(np.sort(perm), np.arange(n))
    c = codes[perm]
    assert np.all(c[1:] >= c[:-1])
    tie = c[1:] == c[:-1]  # stable: equal codes keep their input order
    assert np.all(perm[1:][tie] > perm[:-1][tie])


def momentum_ratio(sim, s):
    em = sim.energy_momentum()
    mv = float(np.sum(s["mass"].astype(np.float64)
                      * np.hypot(s["vx"].astype(np.float64), s["vy"].astype(np.float64))))
    return float(np.hypot(em[1], em[2])) / mv


def test_cold_square_4m(nbx):
    """4,194,304 unit masses at rest in the cold square (softening scaled to
    1e-3 of the half-width), theta 0.5, collisions on."""
    n = 1 << 22
    b = nbx.cold_square(n, 0)
    eps = 1e-3 * 3.0 * np.sqrt(n)
    sim = nbx.Simulation(b, theta=0.5, epsilon=eps)
    sim.step(20)
    s = sim.download()
    check_state(s, n)
    assert momentum_ratio(sim, s) < 1e-3  # from rest: gravity + collisions
    em = sim.energy_momentum()
    assert em[4] == n  # total mass, exact
    sim.phase("build")
    check_morton(sim)
    sim.phase("forces")
    t = np.random.default_rng(12345).choice(n, 4096, replace=False).astype(np.uint32)
    err, _ = sim.force_error(t)
    # theta 0.5 in a uniform square: net forces nearly cancel inside, so the
    # relative tail is the method's own (median ~2%, p99 ~10%)
    assert err["median"] < 0.03 and err["p99"] < 0.2, err
    again = nbx.Simulation(b, theta=0.5, epsilon=eps)
    again.step(20)
    sim.sync()
    sim.close()
    s2 = again.download()
    again.close()
    # the first handle ran one extra build and force pass on its state, which
    # leaves positions and velocities untouched
    a, a2 = s[np.argsort(s["id"])], s2[np.argsort(s2["id"])]
    for f in ("px", "py", "vx", "vy", "mass", "radius", "id"):
        assert same_bits(a[f], a2[f]), f


def test_two_discs_1m_50_steps(nbx):
    n = 1 << 20
    b = nbx.two_discs(n, 0, 0.2)
    outs = []
    for _ in range(2):
        sim = nbx.Simulation(b, theta=0.5)
        sim.step(50)
        outs.append(sim.download())
        if len(outs) == 1:
            check_state(outs[0], n)
            check_morton(sim)
            t = np.random.default_rng(12345).choice(n, 4096, replace=False)
            pos = np.empty(n, np.int64)
            pos[outs[0]["id"]] = np.arange(n)
            err, _ = sim.force_error(pos[t].astype(np.uint32))
            assert err["p99"] < 0.04 and err["median"] < 6e-3, err
        sim.close()
    assert same_bits(outs[0], outs[1])  # deterministic, collisions included


def test_ensemble_512_instances(nbx):
    """The 512-instance ensemble (log-uniform sizes in [2000, 200000]): every
    checked instance equals its standalone run bit for bit."""
    sizes = nbx.ensemble_sizes(512)
    bodies = nbx.ensemble_bodies(sizes)
    h = nbx.Handle(sizes, theta=0.5)
    h.upload(bodies)
    h.step(3)
    g = h.download()
    h.close()
    for f in ("px", "py", "vx", "vy", "ax", "ay"):
        assert np.isfinite(g[f]).all(), f
    starts = np.concatenate([[0], np.cumsum(sizes.astype(np.int64))]).astype(np.int64)
    for k in (0, 137, 300, 511):
        part = bodies[starts[k]:starts[k + 1]]
        sim = nbx.Simulation(part, theta=0.5)
        sim.step(3)
        assert same_bits(sim.download(), g[starts[k]:starts[k + 1]]), k
        sim.close()
    for k in range(512):  # every instance keeps its own bodies
        seg = g[starts[k]:starts[k + 1]]
        assert np.array_equal(np.sort(seg["id"]), np.arange(len(seg)))


def test_cold_square_4m_build_bit_exact(nbx, oracle):
    """Morton codes, permutation and tree of the 4,194,304-body cold square
    against the oracle, bit for bit (the same check as the small states)."""
    b = nbx.cold_square(1 << 22, 0)
    sim = nbx.Simulation(b, theta=0.5)
    sim.phase("build")
    codes, perm = sim.morton()
    root, ocodes, operm, sb, tree = oracle.morton_build(b)
    assert np.array_equal(codes, ocodes) and np.array_equal(perm, operm)
    t = sim.tree()
    assert t["node_count"] == tree.node_count and t["level_count"] == tree.level_count
    for k, v in tree.trimmed().items():
        assert same_bits(t[k], v), k
    assert np.array_equal(sim.download()["id"], sb["id"])
    sim.close()


def collide_at_scale_cases(nbx):
    # a compressed 1M cold square: most boxes overlap several neighbours
    c = nbx.cold_square(1 << 20, 4)
    c["px"] *= np.float32(0.35)
    c["py"] *= np.float32(0.35)
    yield "cold_dense_1M", c
    # the headline two discs late in a run (contacts have piled up)
    sim = nbx.Simulation(nbx.two_discs(1 << 20, 0, 0.2), theta=0.5)
    sim.step(1000)
    sim.phase("iterate")
    yield "two_discs_1M_step1000", sim.download()
    sim.close()
    # the 4M cold square (its configuration's softening) 600 steps in
    n = 1 << 22
    sim = nbx.Simulation(nbx.cold_square(n, 0), theta=0.5, epsilon=1e-3 * 3.0 * np.sqrt(n))
    sim.step(600)
    sim.phase("iterate")
    yield "cold_4M_step600", sim.download()
    sim.close()


def test_collisions_bit_exact_at_scale(nbx, oracle):
    """Candidate pairs (set and pairLess order) and the resolved state bit
    for bit against the oracle's sequential collide() on collision-heavy
    states at the configurations' full sizes."""
    for label, st in collide_at_scale_cases(nbx):
        sim = nbx.Simulation(st)
        sim.phase("collide")
        gl, ge = sim.pairs()
        pairs, depth = sim.collision_stats()
        ol, oe = oracle.collision_pairs(st)
        assert len(ol) > 100000, (label, len(ol))
        assert pairs == len(ol), label
        assert np.array_equal(gl, ol) and np.array_equal(ge, oe), label
        out = sim.download()
        ref, _ = oracle.collide(st)
        assert same_bits(out, ref), (label, int((out != ref).sum()), depth)
        sim.close()
