"""Writes tests/golden/golden_ref.npz from the reference itself.

Run in a checkout where the reference sources are present: oracle/Makefile
compiles them (unmodified, read in place) into oracle/_ref/, and every array
below is produced by the reference's own code through that build:

  * libref_omp.so  -- the reference's own flags (-Ofast -march=native): the
    initial conditions (uniformDisc, src/Utils.cpp:6-54);
  * libref_parity.so -- the same sources built serial and IEEE
    (-O2 -ffp-contract=off): Morton codes (TreeKernels.cuh:62-66), the
    breadth-first tree (splitNode/sumNode/finishNode), accelerationAt,
    QuadTree::build + acceleration, collide(), Simulation::step.

The GPU tests never read the reference: they compare against the CPU
restatement (oracle/), which tests/test_oracle_golden.py pins to this file.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import Reference, build  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_ref.npz")


def stable_perm(codes):
    return np.argsort(codes, kind="stable").astype(np.uint32)


def tree_arrays(R, bodies):
    x, y = bodies["px"], bodies["py"]
    mn = np.array([x.min(), y.min()], np.float32)
    mx = np.array([x.max(), y.max()], np.float32)
    root = np.array([(mn[0] + mx[0]) * np.float32(0.5),
                     (mn[1] + mx[1]) * np.float32(0.5),
                     max(mx[0] - mn[0], mx[1] - mn[1])], np.float32)
    codes = R.morton(x, y, root)
    perm = stable_perm(codes)
    sb = bodies[perm]
    t = R.build_tree(codes[perm], sb["px"], sb["py"], sb["mass"], root)
    return root, codes, perm, sb, t


def main():
    build(ref=True)
    Ro, Rp = Reference("omp"), Reference("parity")
    g = {}
    # initial conditions (reference's own build)
    disc = Ro.uniform_disc(4096)
    g["disc4096"] = disc
    for n in (10000, 1 << 19):
        g[f"disc{n}_sha256"] = np.frombuffer(
            hashlib.sha256(Ro.uniform_disc(n).tobytes()).digest(), np.uint8)
    g["disc4096_seed7"] = Ro.uniform_disc(4096, 7)
    # Morton path + tree + traversal on the disc
    root, codes, perm, sb, t = tree_arrays(Rp, disc)
    g["root"], g["codes"], g["perm"] = root, codes, perm
    for k, v in t.trimmed().items():
        g[f"tree_{k}"] = v
    g["tree_levels"] = np.array([t.level_count], np.int32)
    for theta in (1.0, 0.5):
        ax, ay = Rp.tree_forces(sb["px"], sb["py"], sb["mass"], t, theta, 1.0)
        g[f"forces_t{theta}"] = np.stack([ax, ay])
        q = Rp.quadtree_forces(disc, theta, 1.0)
        g[f"quadtree_t{theta}"] = q
    # a colliding state: 150 reference steps, then iterate(), as
    # stateBeforeCollide (CheckCuda.cu:186-196)
    st, _ = Rp.simulate(disc, steps=150)
    st = Rp.iterate(st, 0.05)
    g["collide_in"] = st
    g["collide_out"] = Rp.collide(st)
    # Simulation::step trajectories (QuadTree.cpp tree, sequential collide)
    small = Ro.uniform_disc(2048)
    g["sim_in"] = small
    for theta in (1.0, 0.5):
        out, _ = Rp.simulate(small, theta=theta, steps=10)
        g[f"sim10_t{theta}"] = out
    # NaiveSimulation: attract on the disc, 5 steps from a 1024-body disc
    g["naive_acc"] = np.stack([Rp.naive_attract(small)["ax"], Rp.naive_attract(small)["ay"]])
    g["naive_in"] = Ro.uniform_disc(1024, 3)
    g["naive5"], _ = Rp.naive_simulate(g["naive_in"], steps=5)
    np.savez_compressed(OUT, **g)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
