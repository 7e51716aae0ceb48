"""ctypes bindings for the CPU checker (test infrastructure only).

``Oracle`` wraps liboracle.so, the CPU restatement of the reference's
per-step path (nbody_oracle.c).  ``Reference`` wraps oracle/_ref/, the
reference's own sources compiled by oracle/Makefile.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module,
and only to check or time against; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

BODY_DTYPE = np.dtype([
    ("px", "<f4"), ("py", "<f4"), ("vx", "<f4"), ("vy", "<f4"),
    ("ax", "<f4"), ("ay", "<f4"), ("mass", "<f4"), ("radius", "<f4"),
    ("id", "<u4"),
])
assert BODY_DTYPE.itemsize == 36

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_bodyp = np.ctypeslib.ndpointer(BODY_DTYPE, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and _ref/ when the reference sources exist)."""
    targets = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


class _Tree(C.Structure):
    _fields_ = [(k, C.POINTER(C.c_float)) for k in
                ("comX", "comY", "mass", "centerX", "centerY", "size")] + \
               [(k, C.POINTER(C.c_int32)) for k in
                ("children", "next", "start", "end")] + \
               [("capacity", C.c_int32), ("nodeCount", C.c_int32),
                ("levelCount", C.c_int32)]


FLOAT_FIELDS = ("comX", "comY", "mass", "centerX", "centerY", "size")
INT_FIELDS = ("children", "next", "start", "end")


class TreeArrays:
    """Host node arrays (TreeKernels.cuh NodeArrays layout)."""

    def __init__(self, capacity: int):
        self.capacity = capacity
        self.f = {k: np.zeros(capacity, np.float32) for k in FLOAT_FIELDS}
        self.i = {k: np.zeros(capacity, np.int32) for k in INT_FIELDS}
        self.node_count = 0
        self.level_count = 0

    def struct(self) -> _Tree:
        t = _Tree()
        for k in FLOAT_FIELDS:
            setattr(t, k, self.f[k].ctypes.data_as(C.POINTER(C.c_float)))
        for k in INT_FIELDS:
            setattr(t, k, self.i[k].ctypes.data_as(C.POINTER(C.c_int32)))
        t.capacity = self.capacity
        return t

    def trimmed(self) -> dict:
        n = self.node_count
        out = {k: v[:n].copy() for k, v in self.f.items()}
        out.update({k: v[:n].copy() for k, v in self.i.items()})
        return out


class Oracle:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        self.L = L
        L.orc_integrate.argtypes = [C.c_size_t, _bodyp, C.c_float]
        L.orc_root_square.argtypes = [C.c_size_t, _f32p, _f32p, _f32p]
        L.orc_morton.argtypes = [C.c_size_t, _f32p, _f32p, _f32p, _u64p]
        L.orc_stable_perm.argtypes = [C.c_size_t, _u64p, _u32p]
        L.orc_build_tree.argtypes = [C.c_size_t, _u64p, _f32p, _f32p, _f32p,
                                     _f32p, C.c_int, C.POINTER(_Tree)]
        L.orc_build_tree.restype = C.c_int
        L.orc_tree_forces.argtypes = [C.c_size_t, _f32p, _f32p, _f32p,
                                      C.POINTER(_Tree), C.c_float, C.c_float,
                                      _f32p, _f32p]
        L.orc_interaction_counts.argtypes = [C.c_size_t, _u32p, _f32p, _f32p,
                                             C.POINTER(_Tree), C.c_float, _f64p]
        L.orc_quadtree_forces.argtypes = [C.c_size_t, _bodyp, C.c_float,
                                          C.c_float, C.c_int]
        L.orc_quadtree_forces.restype = C.c_int
        L.orc_collision_pairs.argtypes = [C.c_size_t, _bodyp, _i32p, _i32p,
                                          C.c_int64]
        L.orc_collision_pairs.restype = C.c_int64
        L.orc_collide.argtypes = [C.c_size_t, _bodyp]
        L.orc_collide.restype = C.c_int64
        L.orc_step.argtypes = [C.c_size_t, _bodyp, C.c_float, C.c_float,
                               C.c_float, C.c_int, C.c_int]
        L.orc_step.restype = C.c_int
        L.orc_naive_forces.argtypes = [C.c_size_t, _f32p, _f32p, _f32p,
                                       C.c_float, _f32p, _f32p]
        L.orc_naive_step.argtypes = [C.c_size_t, _bodyp, C.c_float, C.c_float,
                                     C.c_int]
        L.orc_naive_step.restype = C.c_int
        L.orc_attractor.argtypes = [C.c_size_t, _f32p, _f32p, C.c_float, C.c_float,
                                    C.c_float, C.c_float, _f32p, _f32p]
        L.orc_render.argtypes = [C.c_size_t, _bodyp] + [C.c_float] * 3 + [C.c_int] + \
                                [C.c_float] * 4 + [C.c_uint32, C.c_uint32, _f32p, _f32p]
        L.orc_direct_fp64.argtypes = [C.c_size_t, _f32p, _f32p, _f32p,
                                      C.c_double, C.c_size_t, _u32p, _f64p,
                                      _f64p]
        L.orc_energy_momentum.argtypes = [C.c_size_t, _bodyp, _f64p]
        L.orc_potential_fp64.argtypes = [C.c_size_t, _bodyp, C.c_double]
        L.orc_potential_fp64.restype = C.c_double

    # -- building blocks -------------------------------------------------
    def integrate(self, b: np.ndarray, dt: float) -> np.ndarray:
        b = np.ascontiguousarray(b.copy())
        self.L.orc_integrate(len(b), b, dt)
        return b

    def root_square(self, x, y) -> np.ndarray:
        out = np.zeros(3, np.float32)
        self.L.orc_root_square(len(x), np.ascontiguousarray(x, np.float32),
                               np.ascontiguousarray(y, np.float32), out)
        return out

    def morton(self, x, y, root=None) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        if root is None:
            root = self.root_square(x, y)
        codes = np.zeros(len(x), np.uint64)
        self.L.orc_morton(len(x), x, y, np.ascontiguousarray(root, np.float32),
                          codes)
        return codes

    def stable_perm(self, codes) -> np.ndarray:
        perm = np.zeros(len(codes), np.uint32)
        self.L.orc_stable_perm(len(codes), np.ascontiguousarray(codes, np.uint64),
                               perm)
        return perm

    def build_tree(self, sorted_codes, x, y, m, root, leaf=16) -> TreeArrays:
        n = len(x)
        t = TreeArrays(8 * n + 8)
        s = t.struct()
        rc = self.L.orc_build_tree(n, np.ascontiguousarray(sorted_codes, np.uint64),
                                   np.ascontiguousarray(x, np.float32),
                                   np.ascontiguousarray(y, np.float32),
                                   np.ascontiguousarray(m, np.float32),
                                   np.ascontiguousarray(root, np.float32), leaf,
                                   C.byref(s))
        if rc != 0:
            raise RuntimeError("oracle tree: node capacity exceeded")
        t.node_count, t.level_count = s.nodeCount, s.levelCount
        t._s = s
        return t

    def tree_forces(self, x, y, m, tree: TreeArrays, theta, eps):
        n = len(x)
        ax = np.zeros(n, np.float32)
        ay = np.zeros(n, np.float32)
        s = tree.struct()
        s.nodeCount, s.levelCount = tree.node_count, tree.level_count
        self.L.orc_tree_forces(n, np.ascontiguousarray(x, np.float32),
                               np.ascontiguousarray(y, np.float32),
                               np.ascontiguousarray(m, np.float32), C.byref(s),
                               theta, eps, ax, ay)
        return ax, ay

    def interaction_counts(self, targets, x, y, tree: TreeArrays, theta):
        out = np.zeros(3, np.float64)
        s = tree.struct()
        s.nodeCount, s.levelCount = tree.node_count, tree.level_count
        self.L.orc_interaction_counts(len(targets),
                                      np.ascontiguousarray(targets, np.uint32),
                                      np.ascontiguousarray(x, np.float32),
                                      np.ascontiguousarray(y, np.float32),
                                      C.byref(s), theta, out)
        return out

    def morton_build(self, b: np.ndarray, leaf=16):
        """Root, codes, stable perm, bodies in Morton order, tree."""
        root = self.root_square(b["px"], b["py"])
        codes = self.morton(b["px"], b["py"], root)
        perm = self.stable_perm(codes)
        sb = np.ascontiguousarray(b[perm])
        tree = self.build_tree(codes[perm], sb["px"], sb["py"], sb["mass"],
                               root, leaf)
        return root, codes, perm, sb, tree

    def quadtree_forces(self, b: np.ndarray, theta, eps, leaf=16):
        b = np.ascontiguousarray(b.copy())
        if self.L.orc_quadtree_forces(len(b), b, theta, eps, leaf) != 0:
            raise RuntimeError("QuadTree restatement: depth guard hit")
        return b

    def collision_pairs(self, b: np.ndarray):
        b = np.ascontiguousarray(b)
        cap = max(16, 4 * len(b))
        while True:
            later = np.zeros(cap, np.int32)
            earlier = np.zeros(cap, np.int32)
            k = self.L.orc_collision_pairs(len(b), b, later, earlier, cap)
            if k >= 0:
                return later[:k], earlier[:k]
            cap = -k

    def collide(self, b: np.ndarray):
        b = np.ascontiguousarray(b.copy())
        k = self.L.orc_collide(len(b), b)
        if k < 0:
            raise RuntimeError("oracle collide failed")
        return b, k

    def step(self, b: np.ndarray, dt=0.05, theta=1.0, eps=1.0, leaf=16,
             collisions=True, steps=1):
        b = np.ascontiguousarray(b.copy())
        for _ in range(steps):
            if self.L.orc_step(len(b), b, dt, theta, eps, leaf,
                               int(collisions)) != 0:
                raise RuntimeError("oracle step failed")
        return b

    def naive_forces(self, x, y, m, eps):
        """NaiveSimulation::attract (NaiveSimulation.cpp:17-57)."""
        x, y, m = (np.ascontiguousarray(v, np.float32) for v in (x, y, m))
        ax = np.zeros(len(x), np.float32)
        ay = np.zeros(len(x), np.float32)
        self.L.orc_naive_forces(len(x), x, y, m, eps, ax, ay)
        return ax, ay

    def naive_step(self, b: np.ndarray, dt=0.05, eps=1.0, collisions=True, steps=1):
        """NaiveSimulation::step (NaiveSimulation.cpp:10-15)."""
        b = np.ascontiguousarray(b.copy())
        for _ in range(steps):
            if self.L.orc_naive_step(len(b), b, dt, eps, int(collisions)) != 0:
                raise RuntimeError("oracle naive step failed")
        return b

    def attractor(self, x, y, ax, ay, at, mass=1e6, softening=50.0):
        """attractorKernel (CudaSimulation.cu:14-31), IEEE; returns new ax, ay."""
        ax = np.array(ax, np.float32, copy=True)
        ay = np.array(ay, np.float32, copy=True)
        self.L.orc_attractor(len(ax), np.ascontiguousarray(x, np.float32),
                             np.ascontiguousarray(y, np.float32), at[0], at[1],
                             mass, softening, ax, ay)
        return ax, ay

    def render(self, b, width, height, center=(0.0, 0.0), scale=1.0, mode=1,
               point_scale=1.0, min_point=1.5, brightness=0.6, speed_max=60.0):
        """The viewer's splat drawing restated; returns (rgba[h, w, 4], stats)."""
        img = np.zeros((height, width, 4), np.float32)
        st = np.zeros(3, np.float32)
        self.L.orc_render(len(b), np.ascontiguousarray(b), center[0], center[1], scale,
                          mode, point_scale, min_point, brightness, speed_max, width,
                          height, img.reshape(-1), st)
        return img, st

    def direct_fp64(self, b: np.ndarray, eps, targets):
        targets = np.ascontiguousarray(targets, np.uint32)
        ax = np.zeros(len(targets), np.float64)
        ay = np.zeros(len(targets), np.float64)
        self.L.orc_direct_fp64(len(b), np.ascontiguousarray(b["px"]),
                               np.ascontiguousarray(b["py"]),
                               np.ascontiguousarray(b["mass"]), eps,
                               len(targets), targets, ax, ay)
        return ax, ay

    def energy_momentum(self, b: np.ndarray) -> np.ndarray:
        out = np.zeros(5, np.float64)
        self.L.orc_energy_momentum(len(b), np.ascontiguousarray(b), out)
        return out

    def potential(self, b: np.ndarray, eps) -> float:
        return self.L.orc_potential_fp64(len(b), np.ascontiguousarray(b), eps)


class ReferenceCuda:
    """The reference's own CUDA path (oracle/_ref/libref_cuda.so:
    CudaSimulation built for sm_100a from its unmodified sources).  The
    reference exits the process on any CUDA error, so run it in a child
    process."""

    def __init__(self):
        path = os.path.join(HERE, "_ref", "libref_cuda.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = C.CDLL(path)
        self.L.ref_cuda_simulate.argtypes = [C.c_size_t, _bodyp, C.c_float, C.c_float,
                                             C.c_float, C.c_int, C.c_int, C.c_int]
        self.L.ref_cuda_simulate.restype = C.c_double

    def simulate(self, b, dt=0.05, theta=1.0, eps=1.0, collisions=True, warmup=0,
                 steps=1):
        """(final state, ms of the timed steps)."""
        b = np.ascontiguousarray(b.copy())
        ms = self.L.ref_cuda_simulate(len(b), b, dt, theta, eps, int(collisions),
                                      warmup, steps)
        return b, ms


class Reference:
    """The reference's own code (oracle/_ref): serial IEEE ("parity"), its
    own -Ofast OpenMP ("omp") or -Ofast serial ("serial") build."""

    def __init__(self, kind: str = "parity"):
        path = os.path.join(HERE, "_ref", f"libref_{kind}.so")
        if not os.path.exists(path):
            build(ref=True)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        self.L = L
        L.ref_threads.restype = C.c_int
        L.ref_uniform_disc.argtypes = [C.c_size_t, C.c_uint, _bodyp]
        L.ref_two_discs.argtypes = [C.c_size_t, C.c_uint, C.c_float, _bodyp]
        L.ref_iterate.argtypes = [C.c_size_t, _bodyp, C.c_float]
        L.ref_collide.argtypes = [C.c_size_t, _bodyp]
        L.ref_quadtree_forces.argtypes = [C.c_size_t, _bodyp, C.c_float,
                                          C.c_float, C.c_int]
        L.ref_simulate.argtypes = [C.c_size_t, _bodyp, C.c_float, C.c_float,
                                   C.c_float, C.c_int, C.c_int, C.c_int]
        L.ref_simulate.restype = C.c_double
        L.ref_naive_attract.argtypes = [C.c_size_t, _bodyp]
        L.ref_naive_simulate.argtypes = [C.c_size_t, _bodyp, C.c_float, C.c_int]
        L.ref_naive_simulate.restype = C.c_double
        L.ref_morton.argtypes = [C.c_size_t, _f32p, _f32p, _f32p, _u64p]
        L.ref_build_tree.argtypes = [C.c_size_t, _u64p, _f32p, _f32p, _f32p,
                                     _f32p, C.c_int] + [_f32p] * 6 + \
                                    [_i32p] * 4 + [C.POINTER(C.c_int)]
        L.ref_build_tree.restype = C.c_int
        L.ref_tree_forces.argtypes = [C.c_size_t, _f32p, _f32p, _f32p] + \
                                     [_f32p] * 6 + [_i32p] * 4 + \
                                     [C.c_float, C.c_float, _f32p, _f32p]

    @staticmethod
    def available(kind: str = "parity") -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", f"libref_{kind}.so"))

    def threads(self) -> int:
        return self.L.ref_threads()

    def uniform_disc(self, n: int, seed: int = 0) -> np.ndarray:
        b = np.zeros(n, BODY_DTYPE)
        self.L.ref_uniform_disc(n, seed, b)
        return b

    def two_discs(self, n: int, seed: int = 0, approach: float = 0.2) -> np.ndarray:
        """The two-disc workload from the reference's own uniformDisc."""
        b = np.zeros(n, BODY_DTYPE)
        self.L.ref_two_discs(n, seed, approach, b)
        return b

    def iterate(self, b, dt):
        b = np.ascontiguousarray(b.copy())
        self.L.ref_iterate(len(b), b, dt)
        return b

    def collide(self, b):
        b = np.ascontiguousarray(b.copy())
        self.L.ref_collide(len(b), b)
        return b

    def quadtree_forces(self, b, theta, eps, leaf=16):
        b = np.ascontiguousarray(b.copy())
        self.L.ref_quadtree_forces(len(b), b, theta, eps, leaf)
        return b

    def simulate(self, b, dt=0.05, theta=1.0, eps=1.0, leaf=16, steps=1,
                 collisions=True):
        b = np.ascontiguousarray(b.copy())
        ms = self.L.ref_simulate(len(b), b, dt, theta, eps, leaf, steps,
                                 int(collisions))
        return b, ms

    def naive_attract(self, b):
        b = np.ascontiguousarray(b.copy())
        self.L.ref_naive_attract(len(b), b)
        return b

    def naive_simulate(self, b, dt=0.05, steps=1):
        b = np.ascontiguousarray(b.copy())
        ms = self.L.ref_naive_simulate(len(b), b, dt, steps)
        return b, ms

    def morton(self, x, y, root):
        codes = np.zeros(len(x), np.uint64)
        self.L.ref_morton(len(x), np.ascontiguousarray(x, np.float32),
                          np.ascontiguousarray(y, np.float32),
                          np.ascontiguousarray(root, np.float32), codes)
        return codes

    def build_tree(self, sorted_codes, x, y, m, root):
        n = len(x)
        t = TreeArrays(8 * n + 8)
        levels = C.c_int(0)
        cnt = self.L.ref_build_tree(n, np.ascontiguousarray(sorted_codes, np.uint64),
                                    np.ascontiguousarray(x, np.float32),
                                    np.ascontiguousarray(y, np.float32),
                                    np.ascontiguousarray(m, np.float32),
                                    np.ascontiguousarray(root, np.float32),
                                    t.capacity,
                                    *[t.f[k] for k in FLOAT_FIELDS],
                                    *[t.i[k] for k in INT_FIELDS],
                                    C.byref(levels))
        if cnt < 0:
            raise RuntimeError("reference tree: capacity exceeded")
        t.node_count, t.level_count = cnt, levels.value
        return t

    def tree_forces(self, x, y, m, tree: TreeArrays, theta, eps):
        n = len(x)
        ax = np.zeros(n, np.float32)
        ay = np.zeros(n, np.float32)
        self.L.ref_tree_forces(n, np.ascontiguousarray(x, np.float32),
                               np.ascontiguousarray(y, np.float32),
                               np.ascontiguousarray(m, np.float32),
                               *[tree.f[k] for k in FLOAT_FIELDS],
                               *[tree.i[k] for k in INT_FIELDS], theta, eps,
                               ax, ay)
        return ax, ay
