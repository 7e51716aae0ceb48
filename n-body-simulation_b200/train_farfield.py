"""Trains the learned far-field correction and measures it.

    python train_farfield.py [--out weights/farfield_mlp.f32] [--rows 4194304]

1. Harvest: (cell, target) rows from trees of three workloads -- a 10,000-body
   disc, the 1,048,576-body two-disc system (initial and after 200 steps) and
   a 4,194,304-body cold square (initial and after 100 steps) -- with the MAC
   at theta 1.1 and every accepted cell with size/distance >= 0.3, targets
   from FP64 direct sums over each cell's bodies (nbx_mlp_harvest).
2. Train: Adam on the GPU with the library's own forward/backward kernels
   (nbx_mlp_train).
3. Sweep: on the two-disc system, force error against the FP64 direct sum on
   4096 sampled bodies and the force-pass time, for plain Barnes-Hut and the
   learned form at theta in {0.5, 0.7, 0.9, 1.1}; whole-step throughput for
   plain theta 0.5 and the learned form at each theta.

Writes the weights (1442 float32) and a JSON report next to them.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import nbx  # noqa: E402

HARVEST_THETA = 1.1
HARVEST_BAND = 0.3


def harvest(bodies, steps, n_targets, eps, seed, theta=0.5, max_rows=1 << 22):
    sim = nbx.Simulation(bodies, theta=theta, epsilon=eps)
    if steps:
        sim.step(steps)
    sim.phase("build")
    rng = np.random.default_rng(seed)
    t = rng.choice(len(bodies), min(n_targets, len(bodies)), replace=False)
    rows = sim.mlp_harvest(t.astype(np.uint32), HARVEST_THETA, HARVEST_BAND, max_rows)
    sim.close()
    return rows[rows[:, 11] > 0]


def force_error(sim, n, targets_ids):
    s = sim.download()
    pos = np.empty(n, np.int64)
    pos[s["id"]] = np.arange(n)
    stats, _ = sim.force_error(pos[targets_ids].astype(np.uint32))
    return stats


def timed(fn, reps):
    fn()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    return (time.perf_counter() - t0) / reps * 1e3


FORMS = {"plain": (0, 0.5), "mlp": (1, 0.5), "quad": (2, 0.5),
         "quad0.3": (2, 0.3)}


def sweep(weights, n=1 << 20, thetas=(0.5, 0.7, 0.9, 1.1), pre_steps=50,
          step_reps=30):
    bodies = nbx.two_discs(n, 0, 0.2)
    ids = np.random.default_rng(12345).choice(n, 4096, replace=False)
    base = nbx.Simulation(bodies, theta=0.5)
    base.step(pre_steps)
    state = base.download()
    base.close()
    out = []
    for theta in thetas:
        for mode, (use, band) in FORMS.items():
            sim = nbx.Simulation(state, theta=theta, use_mlp=use, mlp_band=band)
            if use == 1:
                sim.mlp_set_params(weights)
            sim.phase("attract")
            err = force_error(sim, n, ids)
            inter = sim.interactions()
            fms = timed(lambda: sim.phase("forces"), 5)
            sim.step(3)
            sim.sync()
            t0 = time.perf_counter()
            sim.step(step_reps)
            sim.sync()
            sms = (time.perf_counter() - t0) / step_reps * 1e3
            out.append({"theta": theta, "form": mode, "band": band,
                        "p50": float(err["median"]), "p99": float(err["p99"]),
                        "max": float(err["max"]), "force_ms": fms, "step_ms": sms,
                        "body_steps_per_s": n / (sms * 1e-3),
                        "interactions_per_body":
                            float((inter["far"] + inter["near"]) / n)})
            print(json.dumps(out[-1]), flush=True)
            sim.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "farfield_mlp.f32"))
    ap.add_argument("--rows", type=int, default=1 << 22)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--sweep-only", default=None,
                    help="skip harvest/training; sweep with these weights")
    args = ap.parse_args()
    os.makedirs(os.path.dirname(args.out), exist_ok=True)

    if args.sweep_only:
        w = np.fromfile(args.sweep_only, "<f4")
        rep = {"sweep": sweep(w)}
        with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
            json.dump(rep, f, indent=1)
        return
    t0 = time.time()
    parts = []
    parts.append(harvest(nbx.uniform_disc(10000), 0, 10000, 1.0, 1))
    two = nbx.two_discs(1 << 20, 0, 0.2)
    parts.append(harvest(two, 0, 24000, 1.0, 2))
    parts.append(harvest(two, 200, 24000, 1.0, 3))
    cold = nbx.cold_square(1 << 22, 0)
    eps_cold = 1e-3 * 3.0 * np.sqrt(1 << 22)  # 1e-3 of the square's half-width
    parts.append(harvest(cold, 0, 12000, float(eps_cold), 4))
    parts.append(harvest(cold, 100, 12000, float(eps_cold), 5))
    rows = np.concatenate(parts)
    rng = np.random.default_rng(0)
    if len(rows) > args.rows:
        rows = rows[rng.choice(len(rows), args.rows, replace=False)]
    print(f"harvested {len(rows)} rows from {[len(p) for p in parts]} "
          f"in {time.time() - t0:.1f} s", flush=True)

    h = nbx.Handle([64])
    h.mlp_init(7)
    t1 = time.time()
    losses = list(h.mlp_train(rows, epochs=args.epochs, batch=4096, lr=2e-3, seed=1))
    losses += list(h.mlp_train(rows, epochs=max(2, args.epochs // 3), batch=4096,
                               lr=4e-4, seed=2))
    print("epoch losses", [f"{l:.3e}" for l in losses],
          f"({time.time() - t1:.1f} s)", flush=True)
    zero = float(np.mean(np.sum(rows[:, 9:11] ** 2, axis=1)))
    weights = h.mlp_get_params()
    h.close()
    weights.astype("<f4").tofile(args.out)

    report = {"rows": int(len(rows)), "harvest_theta": HARVEST_THETA,
              "harvest_band": HARVEST_BAND,
              "epoch_loss": [float(v) for v in losses],
              "loss_of_zero_correction": zero}
    if not args.no_sweep:
        report["sweep"] = sweep(weights)
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(report, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
