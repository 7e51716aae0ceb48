"""The viewer-facing calls on the GPU: the attractor term fused into the
force pass (attractorKernel, CudaSimulation.cu:14-31) and handle reset
(CudaSimulation::reset), against the oracle."""
import numpy as np
import pytest

from conftest import rel_err, same_bits

pytestmark = pytest.mark.gpu

AT = (300.0, -200.0)


def expected_tree(oracle, bodies, theta, at=None, mass=1e6, soft=50.0):
    _, _, _, sb, tree = oracle.morton_build(bodies)
    ax, ay = oracle.tree_forces(sb["px"], sb["py"], sb["mass"], tree, theta, 1.0)
    if at is not None:
        ax, ay = oracle.attractor(sb["px"], sb["py"], ax, ay, at, mass, soft)
    return ax, ay


@pytest.mark.parametrize("theta", [1.0, 0.5])
def test_attractor_tree_exact(nbx, oracle, theta):
    b = nbx.uniform_disc(20000)
    sim = nbx.Simulation(b, theta=theta, exact_math=1)
    sim.set_attractor(True, *AT, mass=2e6, softening=40.0)
    sim.phase("attract")
    g = sim.download()
    ax, ay = expected_tree(oracle, b, theta, AT, 2e6, 40.0)
    assert same_bits(g["ax"], ax) and same_bits(g["ay"], ay)
    sim.set_attractor(True, *AT, mass=2e6, softening=40.0)
    sim.set_params(exact_math=0)
    sim.phase("forces")
    g = sim.download()
    e = rel_err(g["ax"], g["ay"], ax, ay)
    assert np.percentile(e, 99) < 1e-5 and e.max() < 1e-4
    sim.close()


def test_attractor_naive_exact(nbx, oracle):
    b = nbx.uniform_disc(3000)
    sim = nbx.Simulation(b, force_law=1, exact_math=1)
    sim.set_attractor(True, *AT)
    sim.phase("attract")
    g = sim.download()
    ax, ay = oracle.naive_forces(b["px"], b["py"], b["mass"], 1.0)
    ax, ay = oracle.attractor(b["px"], b["py"], ax, ay, AT)
    assert same_bits(g["ax"], ax) and same_bits(g["ay"], ay)
    sim.close()


def test_attractor_moves_between_graph_steps(nbx, oracle):
    """Steps run from captured graphs; moving or switching off the attractor
    between them takes effect without re-capture."""
    b = nbx.uniform_disc(20000)
    sim = nbx.Simulation(b, theta=0.5, exact_math=1)
    sim.set_attractor(True, 1000.0, 0.0)
    sim.step(2)
    sim.set_attractor(True, *AT)
    sim.step(1)
    g = sim.download()  # Morton order of the last build: the oracle keeps it
    ax, ay = expected_tree(oracle, g, 0.5, AT)
    assert same_bits(g["ax"], ax) and same_bits(g["ay"], ay)
    sim.set_attractor(False, *AT)
    sim.step(1)
    g = sim.download()
    ax, ay = expected_tree(oracle, g, 0.5)
    assert same_bits(g["ax"], ax) and same_bits(g["ay"], ay)
    sim.close()


def test_attractor_off_changes_nothing(nbx):
    b = nbx.uniform_disc(10000)
    outs = []
    for toggle in (False, True):
        sim = nbx.Simulation(b)
        if toggle:
            sim.set_attractor(True, *AT)
            sim.set_attractor(False, *AT)
        sim.step(5)
        outs.append(sim.download())
        sim.close()
    assert same_bits(outs[0], outs[1])


def test_reset_matches_fresh_handle(nbx):
    """Reset to another body count keeps the parameters and the attractor;
    the following steps equal those of a fresh handle."""
    first = nbx.uniform_disc(3000)
    second = nbx.make_scenario("two_galaxies", 5001, 4)
    sim = nbx.Simulation(first, theta=0.5)
    sim.set_attractor(True, *AT)
    sim.step(2)
    sim.reset(second)
    assert sim.params.theta == 0.5
    sim.step(3)
    got = sim.download()
    ref = nbx.Simulation(second, theta=0.5)
    ref.set_attractor(True, *AT)
    ref.step(3)
    assert same_bits(got, ref.download())
    ref.close()
    sim.reset(first[:17])  # shrink
    sim.step(1)
    assert len(sim.download()) == 17
    sim.close()


def test_reset_keeps_network_and_rejects_ensembles(nbx):
    sim = nbx.Simulation(nbx.uniform_disc(1000))
    sim.mlp_init(3)
    before = sim.mlp_get_params()
    sim.reset(nbx.uniform_disc(2000, 1))
    assert same_bits(sim.mlp_get_params(), before)
    sim.close()
    h = nbx.Handle([100, 200])
    h.upload(np.concatenate([nbx.uniform_disc(100), nbx.uniform_disc(200, 1)]))
    with pytest.raises(nbx.NbxError):
        h.reset(nbx.uniform_disc(50))
    h.close()
