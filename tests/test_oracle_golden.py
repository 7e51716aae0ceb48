"""The CPU oracle against fixtures written by the reference itself
(tests/golden/make_golden.py).  Bit-exact: the oracle and the reference's
IEEE build evaluate the same float operations."""
import hashlib

import numpy as np

from conftest import same_bits


def test_morton_codes_and_perm(oracle, golden):
    d = golden["disc4096"]
    root = oracle.root_square(d["px"], d["py"])
    assert same_bits(root, golden["root"])
    codes = oracle.morton(d["px"], d["py"], root)
    assert np.array_equal(codes, golden["codes"])
    assert np.array_equal(oracle.stable_perm(codes), golden["perm"])


def test_tree_topology_and_mass(oracle, golden):
    _, _, _, _, tree = oracle.morton_build(golden["disc4096"])
    t = tree.trimmed()
    assert tree.level_count == int(golden["tree_levels"][0])
    for k, v in t.items():
        assert same_bits(v, golden["tree_" + k]), k


def test_tree_forces_bit_exact(oracle, golden):
    _, _, _, sb, tree = oracle.morton_build(golden["disc4096"])
    for theta in (1.0, 0.5):
        ax, ay = oracle.tree_forces(sb["px"], sb["py"], sb["mass"], tree, theta, 1.0)
        assert same_bits(np.stack([ax, ay]), golden[f"forces_t{theta}"])


def test_quadtree_partition_forces_bit_exact(oracle, golden):
    for theta in (1.0, 0.5):
        q = oracle.quadtree_forces(golden["disc4096"], theta, 1.0)
        assert same_bits(q, golden[f"quadtree_t{theta}"])


def test_collide_bit_exact(oracle, golden):
    st = golden["collide_in"]
    out, pairs = oracle.collide(st)
    assert pairs > 0
    assert same_bits(out, golden["collide_out"])


def test_collision_pairs_are_all_overlaps(oracle, golden):
    """The candidate set is every overlapping box pair (brute force, as
    cpuContacts, CheckCuda.cu:135-184) oriented by before()."""
    st = golden["collide_in"]
    later, earlier = oracle.collision_pairs(st)
    r = st["radius"]
    minx, maxx = st["px"] - r, st["px"] + r
    miny, maxy = st["py"] - r, st["py"] + r
    n = len(st)
    idx = np.arange(n)
    brute = set()
    for i in range(n):
        j = idx[i + 1:]
        # orientation: earlier = smaller (minX, index)
        i_first = (minx[i] < minx[j]) | ((minx[i] == minx[j]) & (i < j))
        e = np.where(i_first, i, j)
        l = np.where(i_first, j, i)
        ov = (maxx[e] >= minx[l]) & (miny[l] <= maxy[e]) & (miny[e] <= maxy[l])
        for a, b in zip(l[ov], e[ov]):
            brute.add((int(a), int(b)))
    assert set(zip(later.tolist(), earlier.tolist())) == brute
    # pairLess order: by later's (minX, index), then earlier's
    key = np.lexsort((earlier, minx[earlier], later, minx[later]))
    assert np.array_equal(key, np.arange(len(later)))


def test_oracle_step_tracks_reference_simulation(oracle, golden):
    """10 Simulation::steps: the oracle's Morton tree vs the reference's
    partition tree differ only in summation order inside leaves."""
    for theta in (1.0, 0.5):
        ref = golden[f"sim10_t{theta}"]
        got = oracle.step(golden["sim_in"], steps=10, theta=theta)
        g = np.sort(got, order="id")
        r = np.sort(ref, order="id")
        err = np.hypot(g["px"] - r["px"], g["py"] - r["py"]) / np.hypot(r["px"], r["py"])
        assert np.isfinite(err).all()
        assert np.median(err) < 1e-4 and err.max() < 1e-3, (np.median(err), err.max())


def test_naive_forces_and_steps_bit_exact(oracle, golden):
    """NaiveSimulation::attract / ::step (the reference's own outputs)."""
    b = golden["sim_in"]
    ax, ay = oracle.naive_forces(b["px"], b["py"], b["mass"], 1.0)
    assert same_bits(np.stack([ax, ay]), golden["naive_acc"])
    assert same_bits(oracle.naive_step(golden["naive_in"], steps=5), golden["naive5"])
