"""Learned far-field correction: the FP64 reference's analytic gradient
(CPU), and the GPU training / inference kernels against it."""
import numpy as np
import pytest

import mlp_ref


def random_rows(n, seed=0):
    rng = np.random.default_rng(seed)
    rows = np.zeros((n, 12), np.float32)
    rows[:, :9] = rng.normal(0, 0.5, (n, 9))
    rows[:, 9:11] = rng.normal(0, 0.05, (n, 2))
    rows[:, 11] = rng.uniform(0.5, 1.5, n)
    return rows


def random_params(seed=1):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 0.3, mlp_ref.N_PARAMS).astype(np.float32)


def test_reference_gradient_matches_finite_differences():
    rows = random_rows(40, 3)
    P = random_params(4).astype(np.float64)
    _, g = mlp_ref.loss_and_grad(P, rows, rounding=False)
    rng = np.random.default_rng(5)
    for k in rng.choice(mlp_ref.N_PARAMS, 60, replace=False):
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        # the reference rounds P to float32: difference the float64 path
        lp = _loss64(Pp, rows)
        lm = _loss64(Pm, rows)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])) + 1e-7, (k, fd, g[k])


def _loss64(P, rows):
    p = {k: P[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in mlp_ref.OFF.items()}
    X, T, w = rows[:, :9].astype(np.float64), rows[:, 9:11], rows[:, 11:12]
    h1 = mlp_ref.silu(X @ p["W1"].T + p["b1"])
    h2 = mlp_ref.silu(h1 @ p["W2"].T + p["b2"])
    y = h2 @ p["W3"].T + p["b3"]
    return float((w * (y - T) ** 2).sum() / len(rows))


@pytest.mark.gpu
def test_gpu_gradient_matches_fp64(nbx):
    rows = random_rows(1000, 7)
    P = random_params(8)
    h = nbx.Handle([64])
    h.mlp_set_params(P)
    g, loss = h.mlp_gradient(rows)
    rl, rg = mlp_ref.loss_and_grad(P, rows)
    assert abs(loss - rl) <= 1e-4 * abs(rl)
    rel = np.linalg.norm(g - rg) / np.linalg.norm(rg)
    assert rel < 1e-4, rel
    assert np.max(np.abs(g - rg)) <= 1e-3 * np.max(np.abs(rg))
    h.close()


@pytest.mark.gpu
def test_gpu_eval_paths(nbx):
    rows = random_rows(3000, 9)
    P = random_params(10) * np.float32(0.5)
    h = nbx.Handle([64])
    h.mlp_set_params(P)
    y_ref, _ = mlp_ref.forward(P, rows[:, :9])
    simt = h.mlp_eval(rows[:, :9], tensor_cores=False)
    assert np.max(np.abs(simt - y_ref)) <= 1e-4 * max(1.0, np.max(np.abs(y_ref)))
    tc = h.mlp_eval(rows[:, :9], tensor_cores=True)
    # tensor cores: BF16 SiLU (tanh.approx) between layers
    scale = np.max(np.abs(y_ref))
    assert np.max(np.abs(tc - y_ref)) <= 3e-2 * scale, np.max(np.abs(tc - y_ref)) / scale
    h.close()


@pytest.mark.gpu
def test_training_reduces_loss(nbx):
    rng = np.random.default_rng(11)
    rows = random_rows(8192, 12)
    # a smooth target the network can learn
    X = rows[:, :9]
    rows[:, 9] = 0.3 * np.tanh(X[:, 0] + 0.5 * X[:, 6]) * X[:, 3]
    rows[:, 10] = 0.2 * X[:, 1] * X[:, 5]
    rows[:, 11] = 1.0
    h = nbx.Handle([64])
    losses = h.mlp_train(rows, epochs=8, batch=512, lr=3e-3, seed=1)
    assert losses[-1] < 0.3 * losses[0], losses
    # deterministic
    h2 = nbx.Handle([64])
    losses2 = h2.mlp_train(rows, epochs=8, batch=512, lr=3e-3, seed=1)
    assert np.array_equal(h.mlp_get_params(), h2.mlp_get_params())
    h.close()
    h2.close()


def _errors(nbx, state, theta, use, band=0.5, weights=None, m=2048):
    n = len(state)
    sim = nbx.Simulation(state, theta=theta, use_mlp=use, mlp_band=band)
    if weights is not None:
        sim.mlp_set_params(weights)
    sim.phase("attract")
    s = sim.download()
    ids = np.random.default_rng(3).choice(n, m, replace=False)
    pos = np.empty(n, np.int64)
    pos[s["id"]] = np.arange(n)
    stats, _ = sim.force_error(pos[ids].astype(np.uint32))
    sim.close()
    return stats


@pytest.mark.gpu
def test_trained_network_and_quadrupole_gain(nbx):
    """What the corrections gain over the uncorrected method at the same MAC:
    the committed network (trained by train_farfield.py with the library's
    own kernels) and the analytic quadrupole control both lower the force
    error against the FP64 direct sum."""
    import os
    w = np.fromfile(os.path.join(os.path.dirname(nbx.__file__), "weights",
                                 "farfield_mlp.f32"), "<f4")
    # the headline two-disc system after 50 steps (a state the network was
    # not trained on: its training rows come from steps 0 and 200)
    sim = nbx.Simulation(nbx.two_discs(1 << 20, 0, 0.2), theta=0.5)
    sim.step(50)
    state = sim.download()
    sim.close()
    plain = _errors(nbx, state, 0.7, 0)
    learned = _errors(nbx, state, 0.7, 1, weights=w)
    quad = _errors(nbx, state, 0.7, 2)
    assert learned["median"] < 0.8 * plain["median"], (learned, plain)
    assert learned["p99"] < plain["p99"], (learned, plain)
    assert quad["median"] < 0.8 * plain["median"], (quad, plain)
