"""GPU parity of the direct all-pairs law (force_law = 1, NaiveSimulation)
against the CPU oracle, which is pinned to the reference's own
NaiveSimulation.cpp (test_oracle_ref.py, golden fixture)."""
import numpy as np
import pytest

from conftest import rel_err, same_bits

pytestmark = pytest.mark.gpu


def naive_sim(nbx, bodies, **kw):
    return nbx.Simulation(bodies, force_law=1, **kw)


@pytest.mark.parametrize("n", [1, 2, 511, 512, 5000])
def test_naive_forces_exact_bit_identical(nbx, oracle, n):
    b = nbx.uniform_disc(n)
    sim = naive_sim(nbx, b, exact_math=1)
    sim.phase("attract")
    g = sim.download()
    ax, ay = oracle.naive_forces(b["px"], b["py"], b["mass"], 1.0)
    assert same_bits(g["ax"], ax) and same_bits(g["ay"], ay)
    assert same_bits(g["px"], b["px"]) and same_bits(g["id"], b["id"])  # order kept
    sim.close()


@pytest.mark.parametrize("n", [5000, 40000])
def test_naive_forces_fast_tolerance(nbx, oracle, n):
    b = nbx.uniform_disc(n)
    sim = naive_sim(nbx, b)
    sim.phase("attract")
    g = sim.download()
    ax, ay = oracle.naive_forces(b["px"], b["py"], b["mass"], 1.0)
    e = rel_err(g["ax"], g["ay"], ax, ay)
    assert np.percentile(e, 99) < 1e-5 and e.max() < 1e-3, (np.percentile(e, 99), e.max())
    sim.close()


def test_naive_steps_match_reference_fixture(nbx, golden):
    """Five NaiveSimulation::steps (iterate, collide, attract) against the
    reference's own output, bit for bit with exact arithmetic."""
    sim = naive_sim(nbx, golden["naive_in"], exact_math=1)
    sim.step(5)
    sim.sync()
    assert same_bits(sim.download(), golden["naive5"])
    sim.close()


def test_naive_ten_steps_with_collisions(nbx, oracle):
    b = nbx.uniform_disc(3000)
    o = oracle.naive_step(b, steps=10)
    sim = naive_sim(nbx, b, exact_math=1)
    sim.step(10)
    assert same_bits(sim.download(), o)
    sim.close()
    sim = naive_sim(nbx, b)
    sim.step(10)
    g = sim.download()
    e = rel_err(g["px"], g["py"], o["px"], o["py"])
    assert e.max() < 1e-3 and np.median(e) < 1e-5
    sim.close()


def test_naive_ensemble_instances_independent(nbx, oracle):
    """Instances straddle thread blocks: every body sums only its own
    instance, in index order."""
    sizes = [1000, 2500, 777, 1]
    parts = [nbx.uniform_disc(s, i) for i, s in enumerate(sizes)]
    h = nbx.Handle(sizes, force_law=1, exact_math=1)
    h.upload(np.concatenate(parts))
    h.phase("attract")
    g = h.download()
    off = 0
    for p in parts:
        ax, ay = oracle.naive_forces(p["px"], p["py"], p["mass"], 1.0)
        assert same_bits(g["ax"][off:off + len(p)], ax)
        assert same_bits(g["ay"][off:off + len(p)], ay)
        off += len(p)
    h.set_params(exact_math=0)
    h.phase("attract")
    g = h.download()
    off = 0
    for p in parts:
        ax, ay = oracle.naive_forces(p["px"], p["py"], p["mass"], 1.0)
        e = rel_err(g["ax"][off:off + len(p)], g["ay"][off:off + len(p)], ax, ay)
        assert len(p) == 1 or np.percentile(e, 99) < 1e-5
        off += len(p)
    h.close()


def test_naive_zero_softening_skips_self(nbx, oracle):
    b = nbx.uniform_disc(700)
    sim = naive_sim(nbx, b, epsilon=0.0)
    sim.phase("attract")
    g = sim.download()
    assert np.isfinite(g["ax"]).all() and np.isfinite(g["ay"]).all()
    ax, ay = oracle.naive_forces(b["px"], b["py"], b["mass"], 0.0)
    e = rel_err(g["ax"], g["ay"], ax, ay)
    assert np.percentile(e, 99) < 1e-5
    sim.close()


def test_naive_fp64_error_uses_plummer_law(nbx, oracle):
    """Against the FP64 Plummer sum the GPU is as accurate as the
    reference's own single-precision sequential sum (whose error grows with
    n: p99 ~2e-4 at 2^16 bodies)."""
    n = 1 << 16
    b = nbx.uniform_disc(n)
    sim = naive_sim(nbx, b)
    sim.phase("attract")
    t = np.random.default_rng(5).choice(n, 256, replace=False).astype(np.uint32)
    stats, err = sim.force_error(t)
    rx, ry = sim.direct_fp64(t)
    ax, ay = oracle.naive_forces(b["px"], b["py"], b["mass"], 1.0)
    ref_err = np.hypot(ax[t] - rx, ay[t] - ry) / np.hypot(rx, ry)
    assert stats["p99"] <= 1.5 * np.percentile(ref_err, 99) + 1e-6, (stats, np.percentile(ref_err, 99))
    assert stats["p99"] < 1e-3
    sim.close()


def test_naive_has_no_tree(nbx):
    sim = naive_sim(nbx, nbx.uniform_disc(1000))
    sim.step(1)
    with pytest.raises(nbx.NbxError):
        sim.morton()
    with pytest.raises(nbx.NbxError):
        naive_sim(nbx, nbx.uniform_disc(10), use_mlp=2)
    sim.close()


def test_direct_fp64_sums_own_instance(nbx, oracle):
    """The FP64 check of an ensemble sums each target's own instance only."""
    sizes = [3000, 5000, 2000]
    parts = [nbx.uniform_disc(s, i) for i, s in enumerate(sizes)]
    h = nbx.Handle(sizes)
    h.upload(np.concatenate(parts))
    cur = h.download()
    tg = np.array([3000 + 17, 3000 + 4999, 8000, 9999, 5], np.uint32)
    ax, ay = h.direct_fp64(tg)
    starts = np.cumsum([0] + sizes)
    for k, t in enumerate(tg):
        inst = int(np.searchsorted(starts, t, side="right") - 1)
        own = cur[starts[inst]:starts[inst + 1]]
        rx, ry = oracle.direct_fp64(own, 1.0, [t - starts[inst]])
        assert abs(ax[k] - rx[0]) <= 1e-12 * max(1.0, abs(rx[0]))
        assert abs(ay[k] - ry[0]) <= 1e-12 * max(1.0, abs(ry[0]))
    h.close()
