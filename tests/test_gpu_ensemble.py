"""Batched ensemble: many instances of uneven size in one handle (one launch
per phase for all of them) give exactly the single-instance results."""
import numpy as np
import pytest

from conftest import same_bits

pytestmark = pytest.mark.gpu


def test_ensemble_equals_looped_instances(nbx, oracle):
    sizes = nbx.ensemble_sizes(24, 200, 20000)
    bodies = nbx.ensemble_bodies(sizes)
    ens = nbx.Handle(sizes, exact_math=1, theta=0.5)
    ens.upload(bodies)
    ens.step(5)
    ens.sync()
    got = ens.download(id_order=True)
    start = 0
    for i, n in enumerate(sizes):
        n = int(n)
        sim = nbx.Simulation(bodies[start:start + n], exact_math=1, theta=0.5)
        sim.step(5)
        one = sim.download(id_order=True)
        sim.close()
        assert same_bits(got[start:start + n], one), i
        if i < 3:  # and against the CPU oracle
            ref = np.sort(oracle.step(bodies[start:start + n], steps=5, theta=0.5),
                          order="id")
            assert same_bits(one, ref), i
        start += n
    ens.close()


def test_ensemble_introspection_per_instance(nbx, oracle):
    sizes = nbx.ensemble_sizes(6, 500, 5000)
    bodies = nbx.ensemble_bodies(sizes)
    ens = nbx.Handle(sizes)
    ens.upload(bodies)
    ens.phase("build")
    start = 0
    for i, n in enumerate(sizes):
        n = int(n)
        b = bodies[start:start + n]
        codes, perm = ens.morton(i)
        root, ocodes, operm, sb, tree = oracle.morton_build(b)
        assert np.array_equal(codes, ocodes) and np.array_equal(perm, operm)
        t = ens.tree(i)
        for k, v in tree.trimmed().items():
            assert same_bits(t[k], v), (i, k)
        start += n
    ens.close()


def test_ensemble_collisions_and_fast_math(nbx):
    sizes = nbx.ensemble_sizes(8, 1000, 8000)
    bodies = nbx.ensemble_bodies(sizes)
    ens = nbx.Handle(sizes, theta=0.5)
    ens.upload(bodies)
    ens.step(40)
    ens.sync()
    got = ens.download(id_order=True)
    start = 0
    for i, n in enumerate(sizes):
        n = int(n)
        sim = nbx.Simulation(bodies[start:start + n], theta=0.5)
        sim.step(40)
        assert same_bits(got[start:start + n], sim.download(id_order=True)), i
        sim.close()
        start += n
    ens.close()


def test_autotune_restores_state(nbx):
    sizes = nbx.ensemble_sizes(16, 1000, 20000)
    bodies = nbx.ensemble_bodies(sizes)
    h = nbx.Handle(sizes, theta=0.5)
    h.upload(bodies)
    h.step(2)
    before = h.download()
    best = h.autotune(allow_leaf=False, steps=2)
    assert best["leaf_capacity"] == 16 and best["ms_per_step"] > 0
    # all three axes reported: grid, block shape, leaf width
    assert best["force_block"] in (128, 256, 512) and best["leaf_pairs"] in (0, 1)
    assert same_bits(h.download(), before)
    # stepping with the tuned launch equals a fresh handle with the same
    # parameters bit for bit (grid and block shape change nothing; the leaf
    # width only the summation order, checked against the default below)
    h.step(3)
    ref = nbx.Handle(sizes, theta=0.5)
    ref.upload(bodies)
    ref.step(2)
    ref.set_params(force_blocks=best["force_blocks"], force_block=best["force_block"],
                   leaf_pairs=best["leaf_pairs"])
    ref.step(3)
    assert same_bits(h.download(), ref.download())
    h.close()
    ref.close()


@pytest.mark.parametrize("threads", [128, 256, 512])
@pytest.mark.parametrize("pairs", [0, 1])
def test_plain_walk_shapes(nbx, oracle, threads, pairs):
    """Every block shape and leaf width of the default walk against the
    reference traversal (the bars of the default arithmetic), and block
    shapes bit-identical to each other at one leaf width."""
    from conftest import rel_err
    b = nbx.uniform_disc(20000)
    _, _, _, sb, tree = oracle.morton_build(b)
    ox, oy = oracle.tree_forces(sb["px"], sb["py"], sb["mass"], tree, 0.5, 1.0)
    sim = nbx.Simulation(b, theta=0.5, force_block=threads, leaf_pairs=pairs)
    sim.phase("attract")
    g = sim.download()
    e = rel_err(g["ax"], g["ay"], ox, oy)
    assert np.percentile(e, 99) < 1e-5 and e.max() < 1e-4, (np.percentile(e, 99), e.max())
    base = nbx.Simulation(b, theta=0.5, force_block=256, leaf_pairs=pairs)
    base.phase("attract")
    assert same_bits(g, base.download())
    sim.close()
    base.close()


def test_ensemble_step_io(nbx):
    """The host-body step of a many-instance handle (force ranges that cut
    across instances, each range's records copied while later ranges
    compute) equals upload + step + download, bit for bit."""
    import torch

    sizes = nbx.ensemble_sizes(16, 5000, 40000)
    bodies = nbx.ensemble_bodies(sizes)
    n = int(np.sum(sizes))
    assert n >= 2 * 65536  # more than one force range
    ref = nbx.Handle(sizes, theta=0.5)
    cur = bodies.copy()
    expect = []
    for _ in range(3):
        ref.upload(cur)
        ref.step(1)
        cur = ref.download()
        expect.append(cur)
    ref.close()
    pinned = torch.empty(n * 36, dtype=torch.uint8, pin_memory=True)
    hb = pinned.numpy().view(nbx.BODY_DTYPE)
    hb[:] = bodies
    ens = nbx.Handle(sizes, theta=0.5)
    for k in range(3):
        ens.step_io_ptr(pinned.data_ptr(), pinned.data_ptr(), n)
        assert same_bits(hb, expect[k]), k
    ens.close()
