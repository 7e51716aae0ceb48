"""Python binding of the C ABI in include/nbx.h (ctypes over lib/libnbx.so).

The library is the product: this module only marshals numpy arrays in and
out.  It raises if the shared library is missing -- there is no fallback.

    sim = Simulation(nbx.uniform_disc(10000))   # one instance
    sim.step(100)
    bodies = sim.download(id_order=True)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnbx.so")

BODY_DTYPE = np.dtype([
    ("px", "<f4"), ("py", "<f4"), ("vx", "<f4"), ("vy", "<f4"),
    ("ax", "<f4"), ("ay", "<f4"), ("mass", "<f4"), ("radius", "<f4"),
    ("id", "<u4"),
])
assert BODY_DTYPE.itemsize == 36

# Every entry point declared in include/nbx.h.
EXPORTS = (
    "nbx_params_default", "nbx_create", "nbx_destroy", "nbx_set_params",
    "nbx_get_params", "nbx_upload_bodies", "nbx_download_bodies", "nbx_step",
    "nbx_step_io",
    "nbx_sync", "nbx_phase", "nbx_get_morton", "nbx_tree_size", "nbx_get_tree",
    "nbx_get_pairs", "nbx_direct_fp64", "nbx_force_error_fp64",
    "nbx_energy_momentum_fp64", "nbx_status_bits", "nbx_last_error",
    "nbx_uniform_disc", "nbx_two_discs", "nbx_cold_square", "nbx_version",
    "nbx_get_stream", "nbx_step_kernel_count", "nbx_interaction_count",
    "nbx_fp32_peak_tflops", "nbx_profile_step", "nbx_mlp_set_params",
    "nbx_mlp_get_params", "nbx_mlp_init", "nbx_mlp_harvest", "nbx_mlp_train",
    "nbx_mlp_gradient", "nbx_mlp_eval", "nbx_ensemble_sizes", "nbx_autotune",
    "nbx_direct_fp64_noalloc", "nbx_step_timed", "nbx_force_times",
    "nbx_make_scenario", "nbx_renumber", "nbx_add_heavy_body", "nbx_add_cluster",
    "nbx_set_attractor", "nbx_reset", "nbx_nbs2_record", "nbx_nbs2_flush",
    "nbx_nbs2_open", "nbx_nbs2_write_packed", "nbx_nbs2_close",
    "nbx_draw_default", "nbx_render", "nbx_body_stats", "nbx_debug_expire_wait",
    "nbx_potential_fp64", "nbx_collision_stats", "nbx_law_error_fp64",
)
SCENARIOS = {"disc": 0, "two_galaxies": 1, "cold_square": 2}
MLP_PARAMS = 1442
MLP_ROW = 12

PHASE = {"iterate": 0, "collide": 1, "build": 2, "forces": 3, "attract": 4,
         "step": 5}
ERRORS = {1: "NBX_ERR_ARG", 2: "NBX_ERR_CUDA", 3: "NBX_ERR_CAPACITY",
          4: "NBX_ERR_NONFINITE", 5: "NBX_ERR_TIMEOUT", 6: "NBX_ERR_STATE",
          7: "NBX_ERR_NOMEM"}


class Params(C.Structure):
    _fields_ = [("dt", C.c_float), ("theta", C.c_float), ("epsilon", C.c_float),
                ("leaf_capacity", C.c_int32), ("collisions", C.c_int32),
                ("exact_math", C.c_int32), ("use_mlp", C.c_int32),
                ("node_factor", C.c_float), ("pair_factor", C.c_float),
                ("force_blocks", C.c_int32), ("device", C.c_int32),
                ("mlp_band", C.c_float), ("force_law", C.c_int32),
                ("force_block", C.c_int32), ("leaf_pairs", C.c_int32)]


class Camera(C.Structure):
    _fields_ = [("center_x", C.c_float), ("center_y", C.c_float), ("scale", C.c_float)]


class Draw(C.Structure):
    _fields_ = [("mode", C.c_int32), ("point_scale", C.c_float),
                ("min_point_px", C.c_float), ("brightness", C.c_float),
                ("speed_max", C.c_float)]


DRAW_MODES = {"speed": 0, "glow": 1}


class NbxError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `make -C {HERE}` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    bodyp = np.ctypeslib.ndpointer(BODY_DTYPE, flags="C_CONTIGUOUS")
    sig = {
        "nbx_params_default": [C.POINTER(Params)],
        "nbx_create": [C.POINTER(Params), C.c_uint32, u32p, C.POINTER(vp)],
        "nbx_destroy": [vp],
        "nbx_set_params": [vp, C.POINTER(Params)],
        "nbx_get_params": [vp, C.POINTER(Params)],
        "nbx_upload_bodies": [vp, vp, C.c_size_t],
        "nbx_download_bodies": [vp, vp, C.c_size_t, C.c_int],
        "nbx_step": [vp, C.c_uint32],
        "nbx_step_io": [vp, vp, vp, C.c_size_t],
        "nbx_step_timed": [vp, C.c_uint32],
        "nbx_force_times": [vp, vp, C.c_uint32],
        "nbx_make_scenario": [C.c_int, C.c_uint32, C.c_uint32, vp],
        "nbx_set_attractor": [vp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float],
        "nbx_draw_default": [C.POINTER(Draw)],
        "nbx_render": [vp, C.POINTER(Camera), C.POINTER(Draw), C.c_uint32, C.c_uint32,
                       vp, vp],
        "nbx_body_stats": [vp, vp],
        "nbx_debug_expire_wait": [vp],
        "nbx_reset": [vp, vp, C.c_size_t],
        "nbx_sync": [vp],
        "nbx_phase": [vp, C.c_int],
        "nbx_get_morton": [vp, C.c_uint32, u64p, u32p, C.c_size_t],
        "nbx_tree_size": [vp, C.c_uint32, C.POINTER(C.c_uint32),
                          C.POINTER(C.c_uint32)],
        "nbx_get_tree": [vp, C.c_uint32] + [vp] * 10 + [C.c_size_t],
        "nbx_get_pairs": [vp, i32p, i32p, C.c_int64, C.POINTER(C.c_int64)],
        "nbx_direct_fp64": [vp, u32p, C.c_uint32, f64p, f64p],
        "nbx_force_error_fp64": [vp, u32p, C.c_uint32, f64p, vp],
        "nbx_energy_momentum_fp64": [vp, f64p],
        "nbx_potential_fp64": [vp, vp, C.c_uint32, vp, C.POINTER(C.c_double)],
        "nbx_collision_stats": [vp, C.POINTER(C.c_int64), C.POINTER(C.c_uint32)],
        "nbx_law_error_fp64": [vp, u32p, C.c_uint32, f64p],
        "nbx_status_bits": [vp, C.POINTER(C.c_uint32)],
        "nbx_last_error": [vp],
        "nbx_uniform_disc": [C.c_uint32, C.c_uint32, bodyp],
        "nbx_two_discs": [C.c_uint32, C.c_uint32, C.c_float, bodyp],
        "nbx_cold_square": [C.c_uint32, C.c_uint32, bodyp],
        "nbx_version": [],
        "nbx_get_stream": [vp, C.POINTER(vp)],
        "nbx_step_kernel_count": [vp, C.POINTER(C.c_uint32)],
        "nbx_interaction_count": [vp, f64p],
        "nbx_fp32_peak_tflops": [C.POINTER(C.c_double)],
        "nbx_profile_step": [vp, C.c_uint32, vp, vp, C.POINTER(C.c_uint32)],
        "nbx_mlp_set_params": [vp, vp, C.c_uint32],
        "nbx_mlp_get_params": [vp, vp, C.c_uint32],
        "nbx_mlp_init": [vp, C.c_uint32],
        "nbx_mlp_harvest": [vp, vp, C.c_uint32, C.c_float, C.c_float, vp,
                            C.c_uint32, C.POINTER(C.c_uint32)],
        "nbx_mlp_train": [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                          C.c_uint32, vp],
        "nbx_mlp_gradient": [vp, vp, C.c_uint32, vp, vp],
        "nbx_mlp_eval": [vp, vp, C.c_uint32, vp, C.c_int],
        "nbx_ensemble_sizes": [C.c_uint32, C.c_uint32, C.c_uint32, vp],
        "nbx_autotune": [vp, C.c_int, C.c_uint32, C.POINTER(Params),
                         C.POINTER(C.c_float)],
        "nbx_accel_at": [vp, vp, vp, C.c_uint32, vp, vp],
        "nbx_direct_fp64_noalloc": [vp, vp, vp, C.c_uint32, vp, C.c_uint32,
                                    C.c_double, vp, vp, vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.nbx_renumber.argtypes = [vp, C.c_size_t]
    L.nbx_renumber.restype = None
    L.nbx_add_heavy_body.argtypes = [vp, C.c_size_t, C.c_float, C.c_float, C.c_float]
    L.nbx_add_heavy_body.restype = C.c_size_t
    L.nbx_add_cluster.argtypes = [vp, C.c_size_t, C.c_float, C.c_float, C.c_float,
                                  C.c_float, C.c_size_t, C.c_uint32]
    L.nbx_add_cluster.restype = C.c_size_t
    L.nbx_nbs2_open.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_float, vp, vp, C.POINTER(vp)]
    L.nbx_nbs2_record.argtypes = [vp, vp]
    L.nbx_nbs2_flush.argtypes = [vp]
    L.nbx_nbs2_close.argtypes = [vp]
    L.nbx_last_error.restype = C.c_char_p
    L.nbx_version.restype = C.c_char_p
    _lib = L
    return L


def default_params(**kw) -> Params:
    p = Params()
    lib().nbx_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def fp32_peak_tflops() -> float:
    v = C.c_double()
    _check(None, lib().nbx_fp32_peak_tflops(C.byref(v)))
    return v.value


def uniform_disc(n: int, seed: int = 0) -> np.ndarray:
    b = np.zeros(n, BODY_DTYPE)
    _check(None, lib().nbx_uniform_disc(n, seed, b))
    return b


def two_discs(n: int, seed: int = 0, approach: float = 0.2) -> np.ndarray:
    b = np.zeros(n, BODY_DTYPE)
    _check(None, lib().nbx_two_discs(n, seed, approach, b))
    return b


def cold_square(n: int, seed: int = 0) -> np.ndarray:
    b = np.zeros(n, BODY_DTYPE)
    _check(None, lib().nbx_cold_square(n, seed, b))
    return b


class Nbs2Writer:
    """An NBS2 output file (src/Main.cpp:13-49): header, mass and radius by
    id, then frames written by Handle.nbs2_record or write_frame."""

    def __init__(self, path, n, total_steps, every, dt, mass_by_id, radius_by_id):
        m = np.ascontiguousarray(mass_by_id, np.float32)
        r = np.ascontiguousarray(radius_by_id, np.float32)
        f = C.c_void_p()
        _check(None, lib().nbx_nbs2_open(str(path).encode(), n, total_steps, every,
                                         dt, m.ctypes.data, r.ctypes.data, C.byref(f)))
        self.f = f

    def close(self):
        if self.f:
            _check(None, lib().nbx_nbs2_close(self.f))
            self.f = None


def save_ppm(rgba: np.ndarray, path) -> None:
    """Writes a rendered image as an 8-bit binary PPM (top row first)."""
    rgb = np.clip(rgba[::-1, :, :3], 0.0, 1.0)
    data = (rgb * 255.0 + 0.5).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (data.shape[1], data.shape[0]))
        f.write(data.tobytes())


def make_scenario(kind: str, n: int, seed: int = 0) -> np.ndarray:
    """The viewer's makeScenario (viewer/Scenarios.cpp:28-62)."""
    b = np.zeros(n, BODY_DTYPE)
    _check(None, lib().nbx_make_scenario(SCENARIOS[kind], n, seed, b.ctypes.data))
    return b


def add_heavy_body(bodies: np.ndarray, x: float, y: float, mass: float) -> np.ndarray:
    """addHeavyBody (viewer/Scenarios.cpp:64-70) on a copy."""
    out = np.zeros(len(bodies) + 1, BODY_DTYPE)
    out[:len(bodies)] = bodies
    lib().nbx_add_heavy_body(out.ctypes.data, len(bodies), x, y, mass)
    return out


def add_cluster(bodies: np.ndarray, x, y, vx, vy, count: int, seed: int) -> np.ndarray:
    """addCluster (viewer/Scenarios.cpp:72-86) on a copy."""
    out = np.zeros(len(bodies) + count, BODY_DTYPE)
    out[:len(bodies)] = bodies
    lib().nbx_add_cluster(out.ctypes.data, len(bodies), x, y, vx, vy, count, seed)
    return out


def renumber(bodies: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(bodies.copy())
    lib().nbx_renumber(out.ctypes.data, len(out))
    return out


def ensemble_sizes(count: int, lo: int = 2000, hi: int = 200000) -> np.ndarray:
    s = np.zeros(count, np.uint32)
    _check(None, lib().nbx_ensemble_sizes(count, lo, hi, s.ctypes.data))
    return s


def ensemble_bodies(sizes) -> np.ndarray:
    """Instance i is uniformDisc(sizes[i], seed i); instances back to back."""
    return np.concatenate([uniform_disc(int(n), i) for i, n in enumerate(sizes)])


def _check(h, rc):
    if rc != 0:
        msg = lib().nbx_last_error(h).decode() if h else ""
        raise NbxError(rc, msg)


class Handle:
    """One nbx handle: one or more instances advanced together."""

    def __init__(self, sizes, params: Params | None = None, **kw):
        self.sizes = np.ascontiguousarray(np.atleast_1d(sizes), np.uint32)
        self.n = int(self.sizes.sum())
        self.starts = np.concatenate([[0], np.cumsum(self.sizes)[:-1]]).astype(np.int64)
        p = params if params is not None else default_params(**kw)
        h = C.c_void_p()
        _check(None, lib().nbx_create(C.byref(p), len(self.sizes), self.sizes,
                                      C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().nbx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc):
        _check(self.h, rc)

    @property
    def params(self) -> Params:
        p = Params()
        self._c(lib().nbx_get_params(self.h, C.byref(p)))
        return p

    def set_params(self, **kw):
        p = self.params
        for k, v in kw.items():
            setattr(p, k, v)
        self._c(lib().nbx_set_params(self.h, C.byref(p)))

    def upload(self, bodies: np.ndarray):
        b = np.ascontiguousarray(bodies, BODY_DTYPE)
        self._c(lib().nbx_upload_bodies(self.h, b.ctypes.data, len(b)))

    def upload_ptr(self, ptr: int, n: int):
        self._c(lib().nbx_upload_bodies(self.h, ptr, n))

    def download(self, id_order: bool = False, out: np.ndarray | None = None):
        if out is None:
            out = np.zeros(self.n, BODY_DTYPE)
        self._c(lib().nbx_download_bodies(self.h, out.ctypes.data, self.n,
                                          int(id_order)))
        return out

    def download_ptr(self, ptr: int, n: int, id_order: bool = False):
        self._c(lib().nbx_download_bodies(self.h, ptr, n, int(id_order)))

    def step_io(self, bodies: np.ndarray, out: np.ndarray | None = None):
        """One step on host bodies (upload, step, download in the bodies'
        order after the step); out may be bodies itself."""
        if out is None:
            out = np.empty(self.n, BODY_DTYPE)
        self._c(lib().nbx_step_io(self.h, bodies.ctypes.data, out.ctypes.data, self.n))
        return out

    def step_io_ptr(self, ptr_in: int, ptr_out: int, n: int):
        self._c(lib().nbx_step_io(self.h, ptr_in, ptr_out, n))

    def step(self, steps: int = 1):
        self._c(lib().nbx_step(self.h, steps))

    def render(self, width: int, height: int, center=(0.0, 0.0), scale=1.0,
               mode="glow", point_scale=1.0, min_point=1.5, brightness=0.6,
               speed_max=60.0):
        """The viewer's splat drawing on the GPU: (rgba[height, width, 4]
        premultiplied, row 0 at the bottom; {com_x, com_y, max_speed})."""
        cam = Camera(center[0], center[1], scale)
        d = Draw(DRAW_MODES[mode] if isinstance(mode, str) else int(mode), point_scale,
                 min_point, brightness, speed_max)
        img = np.zeros((height, width, 4), np.float32)
        st = np.zeros(3, np.float32)
        self._c(lib().nbx_render(self.h, C.byref(cam), C.byref(d), width, height,
                                 img.ctypes.data, st.ctypes.data))
        return img, {"com_x": float(st[0]), "com_y": float(st[1]), "max_speed": float(st[2])}

    def body_stats(self) -> dict:
        st = np.zeros(3, np.float32)
        self._c(lib().nbx_body_stats(self.h, st.ctypes.data))
        return {"com_x": float(st[0]), "com_y": float(st[1]), "max_speed": float(st[2])}

    def nbs2_record(self, writer: "Nbs2Writer"):
        """Records the current state as writer's next frame (device path)."""
        self._c(lib().nbx_nbs2_record(self.h, writer.f))

    def nbs2_flush(self):
        self._c(lib().nbx_nbs2_flush(self.h))

    def set_attractor(self, active: bool, x=0.0, y=0.0, mass=1e6, softening=50.0):
        """The viewer's attractor (CudaSimulation.cuh:9-15)."""
        self._c(lib().nbx_set_attractor(self.h, int(active), x, y, mass, softening))

    def reset(self, bodies: np.ndarray):
        """CudaSimulation::reset: replace every body (any count)."""
        b = np.ascontiguousarray(bodies, BODY_DTYPE)
        self._c(lib().nbx_reset(self.h, b.ctypes.data, len(b)))
        self.sizes = np.array([len(b)], np.uint32)
        self.n = len(b)
        self.starts = np.zeros(1, np.int64)

    def step_timed(self, steps: int):
        """Like step(), recording each step's force-pass duration on the
        handle's stream (read them with force_times())."""
        self._c(lib().nbx_step_timed(self.h, steps))

    def force_times(self, count: int) -> np.ndarray:
        out = np.empty(count, np.float32)
        self._c(lib().nbx_force_times(self.h, out.ctypes.data, count))
        return out

    def sync(self):
        self._c(lib().nbx_sync(self.h))

    def phase(self, name: str):
        self._c(lib().nbx_phase(self.h, PHASE[name]))

    def morton(self, instance: int = 0):
        m = int(self.sizes[instance])
        codes = np.zeros(m, np.uint64)
        perm = np.zeros(m, np.uint32)
        self._c(lib().nbx_get_morton(self.h, instance, codes, perm, m))
        return codes, perm

    def tree(self, instance: int = 0) -> dict:
        nodes, levels = C.c_uint32(), C.c_uint32()
        self._c(lib().nbx_tree_size(self.h, instance, C.byref(nodes),
                                    C.byref(levels)))
        c = nodes.value
        out = {k: np.zeros(c, np.float32) for k in
               ("comX", "comY", "mass", "centerX", "centerY", "size")}
        out.update({k: np.zeros(c, np.int32) for k in
                    ("children", "next", "start", "end")})
        order = ("comX", "comY", "mass", "centerX", "centerY", "size",
                 "children", "next", "start", "end")
        self._c(lib().nbx_get_tree(self.h, instance,
                                   *[out[k].ctypes.data for k in order], c))
        out["node_count"] = c
        out["level_count"] = levels.value
        return out

    def pairs(self):
        cnt = C.c_int64()
        empty = np.zeros(1, np.int32)
        self._c(lib().nbx_get_pairs(self.h, empty, empty, 0, C.byref(cnt)))
        k = cnt.value
        later = np.zeros(max(k, 1), np.int32)
        earlier = np.zeros(max(k, 1), np.int32)
        self._c(lib().nbx_get_pairs(self.h, later, earlier, k, C.byref(cnt)))
        return later[:k], earlier[:k]

    def collision_stats(self):
        """(pairs, longest chain of dependent pairs) of the last collide."""
        p = C.c_int64()
        d = C.c_uint32()
        self._c(lib().nbx_collision_stats(self.h, C.byref(p), C.byref(d)))
        return p.value, d.value

    def direct_fp64(self, targets):
        t = np.ascontiguousarray(targets, np.uint32)
        ax = np.zeros(len(t), np.float64)
        ay = np.zeros(len(t), np.float64)
        self._c(lib().nbx_direct_fp64(self.h, t, len(t), ax, ay))
        return ax, ay

    def law_error(self, targets):
        """Error of the reference's fastInvSqrt law against the exact law,
        both summed in FP64 over every body, at the given targets."""
        t = np.ascontiguousarray(targets, np.uint32)
        st = np.zeros(4, np.float64)
        self._c(lib().nbx_law_error_fp64(self.h, t, len(t), st))
        return {"median": st[0], "p99": st[1], "max": st[2], "mean": st[3]}

    def accel_at(self, px, py):
        """QuadTree::acceleration at arbitrary points from instance 0's last
        tree with the handle's theta and epsilon."""
        x = np.ascontiguousarray(px, np.float32)
        y = np.ascontiguousarray(py, np.float32)
        ax = np.zeros(len(x), np.float32)
        ay = np.zeros(len(x), np.float32)
        self._c(lib().nbx_accel_at(self.h, x.ctypes.data, y.ctypes.data, len(x),
                                   ax.ctypes.data, ay.ctypes.data))
        return ax, ay

    def force_error(self, targets):
        t = np.ascontiguousarray(targets, np.uint32)
        stats = np.zeros(4, np.float64)
        err = np.zeros(len(t), np.float64)
        self._c(lib().nbx_force_error_fp64(self.h, t, len(t), stats,
                                           err.ctypes.data))
        return {"median": stats[0], "p99": stats[1], "max": stats[2],
                "mean": stats[3]}, err

    def energy_momentum(self):
        out = np.zeros(5, np.float64)
        self._c(lib().nbx_energy_momentum_fp64(self.h, out))
        return out

    def potential(self, targets=None):
        """FP64 potential energy: exact over all pairs (targets None), or
        (estimate, per-target potential per unit mass) for a sample."""
        u = C.c_double()
        if targets is None:
            self._c(lib().nbx_potential_fp64(self.h, None, 0, None, C.byref(u)))
            return u.value
        t = np.ascontiguousarray(targets, np.uint32)
        phi = np.zeros(len(t), np.float64)
        self._c(lib().nbx_potential_fp64(self.h, t.ctypes.data, len(t),
                                         phi.ctypes.data, C.byref(u)))
        return u.value, phi

    def stream(self) -> int:
        s = C.c_void_p()
        self._c(lib().nbx_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def step_kernels(self) -> int:
        k = C.c_uint32()
        self._c(lib().nbx_step_kernel_count(self.h, C.byref(k)))
        return k.value

    def interactions(self):
        out = np.zeros(5, np.float64)
        self._c(lib().nbx_interaction_count(self.h, out))
        return {"far": out[0], "near": out[1], "visits": out[2],
                "warp_iters": out[3], "leaf_chunks": out[4]}

    def profile_step(self) -> dict:
        """One eager step; milliseconds per stage."""
        m = 48
        labels = C.create_string_buffer(32 * m)
        ms = np.zeros(m, np.float32)
        cnt = C.c_uint32()
        self._c(lib().nbx_profile_step(self.h, m, labels, ms.ctypes.data,
                                       C.byref(cnt)))
        raw = labels.raw
        return {raw[32 * k: 32 * k + 32].split(b"\0")[0].decode(): float(ms[k])
                for k in range(cnt.value)}

    def autotune(self, allow_leaf=False, steps=3):
        p = Params()
        ms = C.c_float()
        self._c(lib().nbx_autotune(self.h, int(allow_leaf), steps, C.byref(p),
                                   C.byref(ms)))
        return {"leaf_capacity": p.leaf_capacity, "force_blocks": p.force_blocks,
                "force_block": p.force_block, "leaf_pairs": p.leaf_pairs,
                "ms_per_step": ms.value}

    # -- learned far-field correction --------------------------------
    def mlp_set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == MLP_PARAMS
        self._c(lib().nbx_mlp_set_params(self.h, p.ctypes.data, MLP_PARAMS))

    def mlp_get_params(self) -> np.ndarray:
        p = np.zeros(MLP_PARAMS, np.float32)
        self._c(lib().nbx_mlp_get_params(self.h, p.ctypes.data, MLP_PARAMS))
        return p

    def mlp_init(self, seed: int = 0):
        self._c(lib().nbx_mlp_init(self.h, seed))

    def mlp_harvest(self, targets, theta: float, band: float,
                    max_rows: int = 1 << 20) -> np.ndarray:
        t = np.ascontiguousarray(targets, np.uint32)
        rows = np.zeros((max_rows, MLP_ROW), np.float32)
        cnt = C.c_uint32()
        self._c(lib().nbx_mlp_harvest(self.h, t.ctypes.data, len(t), theta, band,
                                      rows.ctypes.data, max_rows, C.byref(cnt)))
        return rows[:cnt.value]

    def mlp_train(self, rows, epochs=10, batch=4096, lr=1e-3, seed=0):
        r = np.ascontiguousarray(rows, np.float32)
        losses = np.zeros(epochs, np.float32)
        self._c(lib().nbx_mlp_train(self.h, r.ctypes.data, len(r), epochs, batch,
                                    lr, seed, losses.ctypes.data))
        return losses

    def mlp_gradient(self, rows):
        r = np.ascontiguousarray(rows, np.float32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = C.c_float()
        self._c(lib().nbx_mlp_gradient(self.h, r.ctypes.data, len(r), g.ctypes.data,
                                       C.byref(loss)))
        return g, loss.value

    def mlp_eval(self, features, tensor_cores=True):
        f = np.ascontiguousarray(features, np.float32).reshape(-1, 9)
        out = np.zeros((len(f), 2), np.float32)
        self._c(lib().nbx_mlp_eval(self.h, f.ctypes.data, len(f), out.ctypes.data,
                                   int(tensor_cores)))
        return out

    def status_bits(self) -> int:
        b = C.c_uint32()
        self._c(lib().nbx_status_bits(self.h, C.byref(b)))
        return b.value


class Simulation(Handle):
    """One simulation: the reference's Simulation / CudaSimulation."""

    def __init__(self, bodies: np.ndarray, **kw):
        super().__init__([len(bodies)], **kw)
        self.upload(bodies)
