"""Pins the CPU restatement to the reference itself at more sizes than the
fixtures hold (runs where oracle/_ref was built from the reference)."""
import numpy as np
import pytest

from conftest import same_bits

from oracle import Reference

pytestmark = pytest.mark.skipif(not Reference.available("parity"),
                                reason="reference build (oracle/_ref) absent")


@pytest.fixture(scope="module")
def ref():
    return Reference("parity")


@pytest.mark.parametrize("n", [1, 17, 2000, 50000, 200000])
def test_morton_tree_forces(oracle, ref, n):
    b = ref.uniform_disc(n)
    root, codes, perm, sb, tree = oracle.morton_build(b)
    assert np.array_equal(codes, ref.morton(b["px"], b["py"], root))
    t2 = ref.build_tree(codes[perm], sb["px"], sb["py"], sb["mass"], root)
    assert tree.node_count == t2.node_count and tree.level_count == t2.level_count
    for k, v in tree.trimmed().items():
        assert same_bits(v, t2.trimmed()[k]), k
    for theta in (1.0, 0.5):
        a = oracle.tree_forces(sb["px"], sb["py"], sb["mass"], tree, theta, 1.0)
        r = ref.tree_forces(sb["px"], sb["py"], sb["mass"], t2, theta, 1.0)
        assert same_bits(np.stack(a), np.stack(r))


@pytest.mark.parametrize("n", [3000, 20000])
def test_collide_and_step(oracle, ref, n):
    b = ref.uniform_disc(n)
    st, _ = ref.simulate(b, steps=100)
    st = ref.iterate(st, 0.05)
    out, k = oracle.collide(st)
    assert k > 0
    assert same_bits(out, ref.collide(st))
    q = oracle.quadtree_forces(st, 0.7, 1.0)
    assert same_bits(q, ref.quadtree_forces(st, 0.7, 1.0))


@pytest.mark.parametrize("n", [1, 2, 257, 3000])
def test_naive_forces_and_steps(oracle, ref, n):
    """NaiveSimulation::attract and ::step restated (nbody_oracle.c) against
    the reference's own NaiveSimulation.cpp, bit for bit."""
    b = ref.uniform_disc(n)
    r = ref.naive_attract(b)
    ax, ay = oracle.naive_forces(b["px"], b["py"], b["mass"], 1.0)
    assert same_bits(ax, r["ax"]) and same_bits(ay, r["ay"])
    o = oracle.naive_step(b, steps=3)
    r3, _ = ref.naive_simulate(b, steps=3)
    assert same_bits(o, r3)
