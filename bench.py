"""Benchmark of the B200 Simulation::step path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (the headline configuration): two rotating discs of 2^19 bodies
each (1,048,576 total), centres 6R apart on x, bulk velocities +-0.2 of the
circular speed on y, opposite spins; FP32; theta = 0.5, epsilon = 1,
dt = 0.05, leaf capacity 16, collisions on.  A "step" is one
Simulation::step (iterate -> collide -> tree build -> forces) of that
system.  Inputs are synthetic (the reference uses no dataset).

value: body-steps/s with the state resident in HBM, timed with CUDA events
on the library's stream over K steps (one captured graph per step),
barrier + synchronize on both sides, max over ranks.  With N GPUs each rank
advances its own replica (the single simulation does not shard), so the
whole-job value is N x bodies / step time ("scaling": "weak").

e2e: the same metric through the C ABI as a drop-in Simulation::step with a
host-owned body array (nbx_step_io, the call the drop-in makes): per step
the 36-byte Body records go host -> device (pinned), one step runs, and they
come back device -> host, the copy back overlapped with the force pass's
later target ranges.  The same loop through three calls (upload, step,
download) is reported beside it.

--impl reference times the reference's own OpenMP CPU implementation
(oracle/_ref/libref_omp.so, built from the reference's sources with its own
flags) on the same workload; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "n-body-simulation_b200")
sys.path.insert(0, PKG)

METRIC = "body-steps/s at 1M: plain vs learned-theta at equal FP64 force error; ensemble"
UNIT = "body-steps/s"
N_BODIES = 1 << 20
THETA = 0.5
WORKLOAD = {
    "workload": "two discs 2x2^19 bodies (1,048,576), centres 6R apart, "
                "+-0.2 v_circ bulk, opposite spin; theta 0.5, eps 1, dt 0.05, "
                "leaf 16, collisions on",
    "bodies": N_BODIES, "theta": THETA, "epsilon": 1.0, "dt": 0.05,
    "leaf_capacity": 16, "collisions": True,
    "l2": "no flush: the per-step working set (~0.3 GB) exceeds the 126 MB L2",
}
# Algorithmic FLOPs per interaction (GPU Gems 3 ch. 31 convention).
FLOP_PER_INTERACTION = 20.0
# Compulsory HBM bytes per body-step of every phase except the force pass
# (FP32 state; one read + one write where a phase must move the data):
# integrate 40, bounds 8, Morton 20, one sort pass 24, gather 56,
# build + upward ~33, collision 88.
ALG_BYTES_PER_BODY_STEP = 285.0 - 16.0  # the force pass's 16 B excluded
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_forces
# launch on the two-disc 1M workload, from an ncu capture of its third launch.
FORCE_TRAFFIC_BYTES = 23.705856e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_BODIES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="headline workload only (no learned/ensemble legs)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default launch parameters (profiling: no tuner trials "
                         "before the timed steps)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200", "-i",
                 str(self.gpu)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------ distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local, dist


def max_over_ranks(dist, local, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def parallelism(world: int) -> str:
    """Both arms name the same layout: one replica of the simulation per GPU."""
    return f"replicas{world}" if world > 1 else "single"


# ------------------------------------------------------------- reference
def reference_rate(n, steps, warmup, bodies=None):
    """The reference's OpenMP Simulation::step (its own flags), all cores.
    Without `bodies` the workload is built by the reference's own
    uniformDisc (oracle/_ref), so that this arm maps no product code."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    R = Reference("omp")
    b = bodies if bodies is not None else R.two_discs(n, 0, 0.2)
    if warmup:
        b, _ = R.simulate(b, theta=THETA, steps=warmup)
    _, ms = R.simulate(b, theta=THETA, steps=steps)
    return n * steps / (ms * 1e-3), R.threads(), ms / steps


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = max(1, min(args.steps, 20))
    warm = max(3, min(args.warmup, 5))
    value, cores, ms = reference_rate(args.n, steps, warm)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": dict(WORKLOAD, parallelism=parallelism(args.gpus)),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                         "kind": "reference", "host": host_cpu(),
                         "sample": f"{steps} Simulation::step calls of the "
                                   f"{args.n}-body workload after {warm} warm-up "
                                   "steps (requested steps capped at 20)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------- extra legs
WEIGHTS = os.path.join(PKG, "weights", "farfield_mlp.f32")


def time_steps(torch, h, stream, steps):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    h.sync()
    e0.record(stream)
    h.step(steps)
    e1.record(stream)
    e1.synchronize()
    h.sync()
    return e0.elapsed_time(e1) / steps


def forms_leg(nbx, torch, sim, n, local, ids, args):
    """Plain Barnes-Hut against the learned far-field correction and the
    analytic quadrupole control on the same state, swept over theta in
    {0.5, 0.7, 0.9, 1.1} (plus the points nearest plain theta 0.5's cost):
    body-steps/s and the force error against the FP64 direct sum on the
    same 4096 sampled bodies.  Also the error floor of the reference's law
    itself (fastInvSqrt against the exact law, FP64 sums over every body) on
    1024 of those bodies."""
    state = sim.download()
    pos = np.empty(n, np.int64)
    pos[state["id"]] = np.arange(n)
    tg = pos[ids].astype(np.uint32)
    weights = np.fromfile(WEIGHTS, "<f4")
    steps = max(5, min(args.steps, 200))
    out = []
    configs = []
    for theta in (0.5, 0.7, 0.9, 1.1):
        configs += [("plain", theta, 0, 0.5), ("learned", theta, 1, 0.5),
                    ("quadrupole", theta, 2, 0.4)]
    # the corrected forms nearest plain theta 0.5's cost, and plain 0.45
    configs += [("plain", 0.45, 0, 0.5), ("quadrupole", 0.65, 2, 0.4),
                ("quadrupole", 0.6, 2, 0.4), ("quadrupole", 0.55, 2, 0.3)]
    for name, theta, use, band in configs:
        h = nbx.Simulation(state, theta=theta, use_mlp=use, mlp_band=band, device=local)
        if use == 1:
            h.mlp_set_params(weights)
        h.phase("attract")
        err, _ = h.force_error(tg)
        stream = torch.cuda.ExternalStream(h.stream(), device=local)
        h.step(2)
        ms = time_steps(torch, h, stream, steps)
        out.append({"form": name, "theta": theta, "band": band,
                    "body_steps_per_s": n / (ms * 1e-3), "ms_per_step": ms,
                    "p50": err["median"], "p99": err["p99"], "steps": steps})
        h.close()
    # the floor under every form: the reference's fastInvSqrt law against
    # the exact law, both summed over every body in FP64
    h = nbx.Simulation(state, theta=0.5, device=local)
    fl = h.law_error(tg[:1024])
    h.close()
    floor = {"form": "law floor: fastInvSqrt law vs exact law, both FP64 all-body sums",
             "samples": 1024, "p50": fl["median"], "p99": fl["p99"], "max": fl["max"]}
    return {"forms": out, "law_floor": floor}


def render_leg(nbx, sim, n):
    """The headless splat renderer on the headline state: 1920x1080, both
    colour modes, camera fitted to the bodies; wall time per frame (each
    call synchronises)."""
    st = sim.body_stats()
    res = {"width": 1920, "height": 1080, "bodies": n}
    s = sim.download()
    span = max(float(np.ptp(s["px"])), float(np.ptp(s["py"])), 1.0) * 1.1
    for mode in ("glow", "speed"):
        for _ in range(3):
            sim.render(1920, 1080, (st["com_x"], st["com_y"]), 1080 / span, mode=mode)
        t0 = time.perf_counter()
        reps = 10
        for _ in range(reps):
            sim.render(1920, 1080, (st["com_x"], st["com_y"]), 1080 / span, mode=mode)
        res[f"{mode}_ms_per_frame"] = (time.perf_counter() - t0) * 1e3 / reps
    return res


def cold_square_leg(nbx, torch, local, steps=2000, every=100, samples=16384):
    """The collision-heavy cold-square collapse at its full size and
    configured length: 4,194,304 unit masses at rest (the viewer's
    ColdSquare geometry, softening 1e-3 of the half-width), theta 0.5,
    collisions on, 2000 steps through the densest-core phase.  Every `every`
    steps: ms/step of the graph steps, one eagerly profiled step (the
    ordered resolution's share of it), the contact pairs and the longest
    chain of dependent pairs.  Energy drift: compensated FP64 kinetic energy
    of all bodies plus the FP64 potential of the tree law estimated from
    the same `samples` bodies (by id) at the start and the end."""
    n = 1 << 22
    eps = 1e-3 * 3.0 * float(np.sqrt(n))
    sim = nbx.Simulation(nbx.cold_square(n, 0), theta=0.5, epsilon=eps, device=local)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    rng = np.random.default_rng(777)
    sample_ids = rng.choice(n, samples, replace=False)

    def energy():
        st = sim.download()
        where = np.empty(n, np.int64)
        where[st["id"]] = np.arange(n)
        tg = where[sample_ids].astype(np.uint32)
        u, phi = sim.potential(tg)
        mphi = st["mass"][tg].astype(np.float64) * phi
        u_err = 0.5 * n * float(np.std(mphi)) / np.sqrt(samples)
        em = sim.energy_momentum()
        mv = float(np.sum(st["mass"].astype(np.float64)
                          * np.hypot(st["vx"].astype(np.float64), st["vy"].astype(np.float64))))
        return em, u, u_err, mv

    em0, u0, u0_err, _ = energy()
    trace = []
    total_ms = 0.0
    done = 0
    while done < steps:
        k = min(every, steps - done)
        ms = time_steps(torch, sim, stream, k - 1) if k > 1 else 0.0
        prof = sim.profile_step()
        pairs, depth = sim.collision_stats()
        step_ms = sum(prof.values())
        total_ms += ms * (k - 1) + step_ms
        done += k
        trace.append({"step": done, "ms_per_step": ms if k > 1 else step_ms,
                      "resolve_share": prof.get("collide.resolve", 0.0) / step_ms,
                      "contact_pairs": pairs, "chain_depth": depth})
    sim.sync()
    em, u, u_err, mv = energy()
    sim.close()
    e0 = em0[0] + u0
    e1 = em[0] + u
    return {"bodies": n, "steps": steps, "epsilon": eps, "theta": 0.5,
            "ms_per_step": total_ms / steps,
            "body_steps_per_s": n * steps / (total_ms * 1e-3),
            "per_100_steps": trace,
            "kinetic_energy_fp64": [float(em0[0]), float(em[0])],
            "potential_energy_fp64": [u0, u],
            "potential_sample_stderr": [u0_err, u_err],
            "energy_drift_rel": (e1 - e0) / abs(e0),
            "energy_drift_rel_stderr": float(np.hypot(u0_err, u_err)) / abs(e0),
            "energy_note": "potential from the FP64 tree-law direct sum at the "
                           f"same {samples} bodies (by id) at both ends, scaled "
                           "to all pairs; collisions are inelastic, so total "
                           "energy falls physically",
            "momentum_drift_rel": float(np.hypot(em[1] - em0[1], em[2] - em0[2])) / mv,
            "angular_momentum_drift_rel": float(abs(em[3] - em0[3])) / (mv * 3.0 * np.sqrt(n)),
            "mass_exact": bool(em[4] == em0[4])}


def host_cpu():
    """Model name and logical CPU count of this host (lscpu's figures)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def _ref_gpu_child(n, kind, theta, warmup, steps, q):
    """Child process: the reference's CudaSimulation (oracle/_ref/
    libref_cuda.so) on its own CUDA context; the reference exits on any CUDA
    error, which the parent then sees as a dead child."""
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Reference, ReferenceCuda
        R = Reference("omp")
        b = R.two_discs(n, 0, 0.2) if kind == "two_discs" else R.uniform_disc(n, 0)
        _, ms = ReferenceCuda().simulate(b, theta=theta, warmup=warmup, steps=steps)
        q.put({"ms": ms})
    except Exception as ex:  # reference build absent
        q.put({"unavailable": str(ex)})


def reference_gpu(n, kind, theta, warmup, steps):
    """ms/step of the reference's own CUDA path (CudaSimulation::step,
    built for sm_100a from its unmodified sources) on the same GPU, run in a
    child process; its collisions are resolved Jacobi-style, every contact
    of a body against the step's start state, by design
    (accumulatePair, CollisionKernels.cuh:197-235)."""
    import multiprocessing as mpc
    ctx = mpc.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_gpu_child, args=(n, kind, theta, warmup, steps, q))
    p.start()
    p.join(600)
    if p.is_alive():
        p.kill()
        return {"unavailable": "timed out"}
    if p.exitcode != 0 or q.empty():
        return {"unavailable": f"reference exited with code {p.exitcode}"}
    r = q.get()
    if "ms" in r:
        if r["ms"] < 0:
            return {"unavailable": "CUDA error in the reference path"}
        ms = r["ms"] / steps
        return {"ms_per_step": ms, "body_steps_per_s": n / (ms * 1e-3),
                "steps": steps, "warmup": warmup}
    return r


def c0_leg(nbx, torch, local):
    """The reference's own CPU-runnable case: uniformDisc(10,000), dt 0.05,
    eps 1, leaf 16, collisions on, 100 steps, at theta 1.0 (the reference's
    default, what its `sim` CLI runs) and 0.5.  The product (device-resident
    step graphs, CUDA events) against the reference's serial and OpenMP
    builds (its own flags; the CLIs' avg_compute_step at theta 1.0 as well)
    and its CUDA path on the same GPU."""
    n, steps = 10000, 100
    res = {"bodies": n, "steps": steps, "host": host_cpu()}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    for theta in (1.0, 0.5):
        row = {}
        sim = nbx.Simulation(nbx.uniform_disc(n), theta=theta, device=local)
        stream = torch.cuda.ExternalStream(sim.stream(), device=local)
        sim.step(3)
        ms = time_steps(torch, sim, stream, steps)
        sim.close()
        row["b200"] = {"ms_per_step": ms, "body_steps_per_s": n / (ms * 1e-3)}
        try:
            from oracle import Reference
            for kind in ("serial", "omp"):
                R = Reference(kind)
                _, rms = R.simulate(nbx.uniform_disc(n), theta=theta, steps=steps)
                row[f"reference_{kind}"] = {"ms_per_step": rms / steps,
                                            "body_steps_per_s": n * steps / (rms * 1e-3),
                                            "threads": R.threads()}
        except Exception as ex:
            row["reference_cpu"] = {"unavailable": str(ex)}
        row["reference_cuda"] = reference_gpu(n, "disc", theta, 3, steps)
        res[f"theta_{theta}"] = row
    # the reference CLIs themselves (theta 1.0), their own timing line
    for exe in ("sim_serial", "sim"):
        path = os.path.join(ROOT, "oracle", "_ref", exe)
        try:
            out = subprocess.run([path, str(n), str(steps), "1"], capture_output=True,
                                 text=True, timeout=300).stderr
            avg = float(out.split("avg_compute_step=")[1].split()[0])
            res[f"cli_{exe}"] = {"avg_compute_step_ms": avg,
                                 "body_steps_per_s": n / (avg * 1e-3)}
        except (OSError, IndexError, ValueError, subprocess.SubprocessError) as ex:
            res[f"cli_{exe}"] = {"unavailable": str(ex)}
    return res


NAIVE_N = 1 << 18


def naive_leg(nbx, torch, local, args):
    """The direct all-pairs law (force_law = 1, NaiveSimulation) on a
    2^18-body disc: a second roofline anchor (pure FP32/MUFU issue, n(n-1)
    interactions per step, 20 FLOP each), against the reference's own
    OpenMP NaiveSimulation on a smaller disc."""
    n = NAIVE_N
    sim = nbx.Simulation(nbx.uniform_disc(n), force_law=1, device=local)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    sim.step(3)
    sim.sync()
    steps = 10
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step_timed(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    fms = sim.force_times(steps)
    inter = float(n) * (n - 1)
    tflops = FLOP_PER_INTERACTION * inter / (float(fms.mean()) * 1e-3) / 1e12
    peak = nbx.fp32_peak_tflops()
    rng = np.random.default_rng(12345)
    err, _ = sim.force_error(rng.choice(n, 1024, replace=False).astype(np.uint32))
    sim.close()
    res = {"bodies": n, "steps": steps, "ms_per_step": ms,
           "body_steps_per_s": n / (ms * 1e-3),
           "force_ms": float(fms.mean()), "interactions_per_s": inter / (float(fms.mean()) * 1e-3),
           "achieved_tflops": tflops, "peak_tflops": peak,
           "frac": tflops / peak if peak else None,
           "force_error_fp64_p99": err["p99"]}
    try:  # the reference's own NaiveSimulation (OpenMP, its flags), smaller disc
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Reference
        R = Reference("omp")
        nc = 1 << 15
        _, cms = R.naive_simulate(nbx.uniform_disc(nc), steps=2)
        res["reference_cpu"] = {"bodies": nc, "ms_per_step": cms / 2,
                                "interactions_per_s": nc * (nc - 1) / (cms / 2 * 1e-3),
                                "cores": R.threads()}
    except Exception as ex:  # reference build absent
        res["reference_cpu"] = {"unavailable": str(ex)}
    return res


def ensemble_leg(nbx, torch, world, rank, local, dist, args):
    """512 discs of log-uniform size in [2000, 200000] advanced by one
    handle, against looping the single-instance solver over the same
    instances (one handle and captured graph per instance, launched
    back to back without host synchronisation between instances)."""
    sys.path.insert(0, PKG)
    import ensemble
    sizes = nbx.ensemble_sizes(512)
    mine = ensemble.partition_instances(sizes, world)[rank]
    my_sizes = sizes[mine]
    bodies = np.concatenate([nbx.uniform_disc(int(sizes[i]), i) for i in mine])
    steps = max(3, min(args.steps, 10))
    h = nbx.Handle(my_sizes, theta=0.5, device=local)
    h.upload(bodies)
    stream = torch.cuda.ExternalStream(h.stream(), device=local)
    h.step(2)
    kernels = h.step_kernels()
    ms = max_over_ranks(dist, local, time_steps(torch, h, stream, steps))
    total = int(sizes.sum())
    res = {"instances": int(len(sizes)), "bodies": total, "theta": 0.5,
           "steps": steps, "ms_per_step": ms,
           "body_steps_per_s": total / (ms * 1e-3),
           "kernels_per_step": kernels}
    if dist is not None:
        # the run's only collective: per-instance metrics to every rank
        metrics = ensemble.gather_metrics(
            dist, mine, ensemble.instance_metrics(h.download(), my_sizes),
            len(sizes), local)
        res["gathered_instances"] = int(np.isfinite(metrics[:, 0]).sum())
    h.close()
    if world == 1:
        loop_steps = 3
        hs = []
        start = 0
        for i, nb in enumerate(sizes):
            hi = nbx.Simulation(bodies[start:start + int(nb)], theta=0.5, device=local)
            hi.step(1)
            hs.append(hi)
            start += int(nb)
        for hi in hs:
            hi.sync()
        torch.cuda.synchronize(local)
        # sequential loop: each instance's step completes before the next
        # one starts, as a driver looping Simulation::step over instances
        t0 = time.perf_counter()
        for _ in range(loop_steps):
            for hi in hs:
                hi.step(1)
                hi.sync()
        seq_ms = (time.perf_counter() - t0) * 1e3 / loop_steps
        # concurrent loop: all instances' step graphs enqueued back to back
        # on their own streams, one synchronisation at the end
        t0 = time.perf_counter()
        for _ in range(loop_steps):
            for hi in hs:
                hi.step(1)
        for hi in hs:
            hi.sync()
        loop_ms = (time.perf_counter() - t0) * 1e3 / loop_steps
        for hi in hs:
            hi.close()
        res["looped_ms_per_step"] = seq_ms
        res["looped_body_steps_per_s"] = total / (seq_ms * 1e-3)
        res["speedup_vs_looped"] = seq_ms / ms
        res["looped_concurrent_ms_per_step"] = loop_ms
        res["speedup_vs_looped_concurrent"] = loop_ms / ms
    return res


# ------------------------------------------------------------------ b200
def run_b200(args):
    world, rank, local, dist = dist_setup(args)
    import torch
    torch.cuda.set_device(local)
    import nbx
    n = args.n
    bodies = nbx.two_discs(n, 0, 0.2)
    sim = nbx.Simulation(bodies, theta=THETA, device=local)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)

    # the library's autotuner picks the force walk's block shape, leaf width
    # and grid for this workload (leaf capacity stays the reference's 16);
    # it restores the state it timed from
    tuned = (sim.autotune(allow_leaf=False, steps=3) if not args.no_autotune else
             {"force_block": 0, "leaf_pairs": 1, "force_blocks": 0, "leaf_capacity": 16})
    sim.step(args.warmup)
    sim.sync()
    kernels_per_step = sim.step_kernels()
    # state at the start of the timed region: a second handle replays the
    # timed steps afterwards to count each step's interactions
    start_state = sim.download()

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier(dist)
        torch.cuda.synchronize(local)
        sim.sync()
        e0.record(stream)
        # the step graph with CUDA events around each force launch
        sim.step_timed(args.steps)
        e1.record(stream)
        e1.synchronize()
        sim.sync()
        torch.cuda.synchronize(local)
        barrier(dist)
    ms_rank = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(dist, local, ms_rank)
    value = world * n / (ms * 1e-3)

    # dominant kernel: the force traversal.  Its per-step durations were
    # recorded inside the timed region; its work per step comes from a
    # replay of the same steps on a second handle, which counts each
    # step's interactions (the simulation is deterministic: the replay's
    # final state must equal the timed run's bit for bit).
    force_ms_steps = sim.force_times(args.steps)
    s = sim.download()
    replay = nbx.Simulation(start_state, theta=THETA, device=local,
                            force_blocks=tuned["force_blocks"],
                            force_block=tuned["force_block"], leaf_pairs=tuned["leaf_pairs"])
    inter_steps = np.empty((args.steps, 2), np.float64)
    # the replay also checks the forces every 100 steps (and after the last)
    # against the FP64 direct sum on the same 4096 sampled bodies (by id)
    check_ids = np.random.default_rng(12345).choice(n, 4096, replace=False)
    force_checks = []
    for k in range(args.steps):
        replay.step(1)
        c = replay.interactions()
        inter_steps[k] = c["far"], c["near"]
        if (k + 1) % 100 == 0 or k + 1 == args.steps:
            cur = replay.download()
            where = np.empty(n, np.int64)
            where[cur["id"]] = np.arange(n)
            st, _ = replay.force_error(where[check_ids].astype(np.uint32))
            force_checks.append({"step": k + 1, "p50": st["median"], "p99": st["p99"],
                                 "max": st["max"]})
    replay_same = replay.download().tobytes() == s.tobytes()
    replay.close()
    inter = {"far": inter_steps[:, 0].mean(), "near": inter_steps[:, 1].mean()}
    force_ms = float(force_ms_steps.mean())
    flops = FLOP_PER_INTERACTION * (inter["far"] + inter["near"])
    achieved = (FLOP_PER_INTERACTION * inter_steps.sum()
                / (force_ms_steps.astype(np.float64).sum() * 1e-3) / 1e12)
    peak = nbx.fp32_peak_tflops()
    # the rest of the step against the measured HBM copy bandwidth
    hbm_peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            hbm_peak = float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    other_ms = ms - force_ms
    other_gbs = ALG_BYTES_PER_BODY_STEP * n / (other_ms * 1e-3) / 1e9

    # force error against the FP64 direct sum on 4096 sampled bodies
    rng = np.random.default_rng(12345)
    ids = rng.choice(n, 4096, replace=False)
    pos = np.empty(n, np.int64)
    pos[s["id"]] = np.arange(n)
    err_stats, _ = sim.force_error(pos[ids].astype(np.uint32))

    # e2e: host-owned bodies in pinned memory, one nbx_step_io per step
    # (the drop-in Simulation::step: H2D of every body record, the step,
    # D2H of every record, the copy overlapped with the force ranges)
    e2e_steps = max(3, min(args.steps, 100))
    host = torch.empty(n * 36, dtype=torch.uint8, pin_memory=True)
    hb = host.numpy().view(nbx.BODY_DTYPE)
    hb[:] = s
    ptr = host.data_ptr()

    def timed_host_loop(one_step):
        one_step()  # warm: captures the graphs this path launches
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        barrier(dist)
        t0 = time.perf_counter()
        g0.record(stream)
        for _ in range(e2e_steps):
            one_step()
        g1.record(stream)
        g1.synchronize()
        wall = time.perf_counter() - t0
        ms = max(g0.elapsed_time(g1), wall * 1e3) / e2e_steps
        return max_over_ranks(dist, local, ms)

    def separate_calls():
        sim.upload_ptr(ptr, n)
        sim.step(1)
        sim.download_ptr(ptr, n)

    e2e_sep_ms = timed_host_loop(separate_calls)
    e2e_ms = timed_host_loop(lambda: sim.step_io_ptr(ptr, ptr, n))
    e2e_value = world * n / (e2e_ms * 1e-3)

    learned = forms_leg(nbx, torch, sim, n, local, ids, args) if not args.quick else None
    sim_keep = sim
    ens = ensemble_leg(nbx, torch, world, rank, local, dist, args) if not args.quick else None
    naive = naive_leg(nbx, torch, local, args) if not args.quick else None
    cold = cold_square_leg(nbx, torch, local) if not args.quick else None
    render = render_leg(nbx, sim_keep, n) if not args.quick else None
    c0 = ref_gpu = None
    if rank == 0 and world == 1 and not args.quick and not args.no_cpu_baseline:
        c0 = c0_leg(nbx, torch, local)
        # the reference's own CUDA path on the same GPU, headline workload
        ref_gpu = dict(reference_gpu(n, "two_discs", THETA, 3, min(max(args.steps, 5), 20)),
                       workload=WORKLOAD["workload"])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, cores, cms = reference_rate(n, 8, 1, bodies)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                   "host": host_cpu(),
                   "sample": f"8 Simulation::step calls of the same {n}-body "
                             f"workload after 1 warm-up step ({cms:.0f} ms/step), "
                             "reference built with its own flags (-Ofast -fopenmp)"}
        except Exception as ex:  # reference build absent
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {ex}"}

    clk = clocks.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": dict(WORKLOAD, parallelism=parallelism(world)),
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": 36 * n, "d2h_bytes_per_step": 36 * n,
                "ms_per_step": e2e_ms,
                "api": "nbx_step_io (pinned host bodies in and out)",
                "ms_per_step_upload_step_download": e2e_sep_ms},
        "roofline": {
            "kernel": "k_forces (warp-cooperative traversal)",
            "bound": "fp32", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
            "traffic": FORCE_TRAFFIC_BYTES if n == N_BODIES else None,
            "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of one "
                            "launch, ncu capture at step 3 (a constant)",
            "peak_note": "FP32 FMA peak measured live by a probe kernel "
                         "(MEASURED_PEAKS.json holds no FP32 figure)",
            "flops_per_launch": flops, "launch_ms": force_ms,
            "launch_ms_first_last": [float(force_ms_steps[0]), float(force_ms_steps[-1])],
            "force_share_of_step": force_ms / ms,
            "interactions_per_body": (inter["far"] + inter["near"]) / n,
            "timing": "CUDA events around every force launch of the timed "
                      "steps (event-record nodes in the step graph, same stream); "
                      "FLOPs from a replay of the same steps counting "
                      "interactions per step",
            "replay_bit_identical": replay_same,
        },
        "roofline_other_phases": {
            "bound": "hbm", "achieved": other_gbs, "peak": hbm_peak,
            "unit": "GB/s", "frac": other_gbs / hbm_peak if hbm_peak else None,
            "algorithmic_bytes_per_body_step": ALG_BYTES_PER_BODY_STEP,
            "ms_per_step": other_ms,
            "note": "step time minus the event-timed force pass; compulsory "
                    "bytes of integrate, collision, bounds, Morton, one sort "
                    "pass, gather, build; peak of measured (MEASURED_PEAKS.json "
                    "hbm_gbs)"},
        "force_error_fp64": {"p50": err_stats["median"], "p99": err_stats["p99"],
                             "max": err_stats["max"], "samples": 4096,
                             "every_100_steps": force_checks},
        "interactions_per_s": (inter["far"] + inter["near"]) * 1e3 / ms,
        "gpu_launches": kernels_per_step * args.steps,
        "autotune": {k: tuned[k] for k in ("force_block", "leaf_pairs", "force_blocks",
                                            "leaf_capacity")},
        "clocks": clk,
    }
    if learned is not None:
        line["learned_theta"] = learned
    if ens is not None:
        line["ensemble"] = ens
    if naive is not None:
        line["naive"] = naive
    if cold is not None:
        line["cold_square"] = cold
    if render is not None:
        line["render"] = render
    if c0 is not None:
        line["c0_disc10k"] = c0
    if ref_gpu is not None:
        line["reference_gpu_baseline"] = ref_gpu
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim_keep.close()
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
