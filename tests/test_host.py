"""Host-side product code: the C ABI library loads and exports every entry
point of include/nbx.h; the generators reproduce the reference's initial
conditions bit for bit.  No GPU needed (no compute calls are made)."""
import hashlib
import os
import re

import numpy as np
import pytest

from conftest import ROOT, same_bits


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "nbx.h")).read()
    return sorted(set(re.findall(r"\b(nbx_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(nbx):
    lib = nbx.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [s for s in names if not hasattr(lib, s)]
    assert not missing, missing
    assert set(names) >= set(nbx.EXPORTS)


def test_uniform_disc_matches_reference(nbx, golden):
    assert same_bits(nbx.uniform_disc(4096), golden["disc4096"])
    assert same_bits(nbx.uniform_disc(4096, 7), golden["disc4096_seed7"])
    for n in (10000, 1 << 19):
        h = hashlib.sha256(nbx.uniform_disc(n).tobytes()).digest()
        assert h == golden[f"disc{n}_sha256"].tobytes(), n


def test_reference_arm_input_is_the_products(nbx):
    """bench.py's reference arm builds the two-disc workload with the
    reference's own uniformDisc (oracle/_ref), so that it maps no product
    code; both arms must start from the same bytes."""
    from oracle import Reference
    if not Reference.available("omp"):
        pytest.skip("reference build absent")
    R = Reference("omp")
    for n in (4096, 1 << 20):
        assert same_bits(R.two_discs(n, 0, 0.2), nbx.two_discs(n, 0, 0.2)), n


def test_params_default_are_reference_defaults(nbx):
    p = nbx.default_params()
    assert (p.dt, p.theta, p.epsilon, p.leaf_capacity, p.collisions) == (
        np.float32(0.05), 1.0, 1.0, 16, 1)


@pytest.mark.parametrize("bad", [dict(use_mlp=3), dict(leaf_capacity=0),
                                 dict(leaf_capacity=65), dict(theta=-1.0)])
def test_invalid_params_rejected_before_device(nbx, bad):
    with pytest.raises(nbx.NbxError) as e:
        nbx.Handle([16], **bad)
    assert e.value.code == 1  # NBX_ERR_ARG


def test_two_discs_layout(nbx):
    n = 2048
    b = nbx.two_discs(n, 0, 0.2)
    assert np.array_equal(b["id"], np.arange(n))
    left, right = b[: n // 2], b[n // 2:]
    assert left["px"].mean() < 0 < right["px"].mean()
    assert (left["mass"] == 1e6).sum() == 1 and (right["mass"] == 1e6).sum() == 1
    # opposite spins: angular momentum about each centre has opposite sign
    def lz(d):
        x = d["px"] - d["px"][d["mass"] > 1e5][0]
        y = d["py"] - d["py"][d["mass"] > 1e5][0]
        vy = d["vy"] - d["vy"][d["mass"] > 1e5][0]
        vx = d["vx"] - d["vx"][d["mass"] > 1e5][0]
        return float((d["mass"] * (x * vy - y * vx)).sum())
    assert lz(left) * lz(right) < 0


def test_cold_square(nbx):
    b = nbx.cold_square(1000, 3)
    h = 3 * np.sqrt(1000)
    assert np.all(np.abs(b["px"]) <= h) and np.all(np.abs(b["py"]) <= h)
    assert np.all(b["vx"] == 0) and np.all(b["radius"] == 1) and np.all(b["mass"] == 1)


def test_create_without_device_reports_error(nbx):
    """On a machine without a GPU nbx_create returns an error code instead
    of exiting (the reference's CUDA_CHECK aborts the process)."""
    import subprocess, sys
    code = ("import sys; sys.path.insert(0, %r); import nbx\n"
            "try:\n    nbx.Handle([16])\n    print('created')\n"
            "except nbx.NbxError as e:\n    print('error', e.code)\n"
            % os.path.join(ROOT, "n-body-simulation_b200"))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True,
                         text=True, env=env, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("error"), out.stdout


def read_nbs2(path):
    """Reads an NBS2 file (layout of the reference's Main.cpp:13-49)."""
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw[:28], np.dtype([
        ("magic", "S4"), ("n", "<u4"), ("steps", "<u4"), ("every", "<u4"),
        ("frames", "<u4"), ("completed", "<u4"), ("dt", "<f4")]))[0]
    n = int(hdr["n"])
    mass = np.frombuffer(raw[28:28 + 4 * n], "<f4")
    radius = np.frombuffer(raw[28 + 4 * n:28 + 8 * n], "<f4")
    body = raw[28 + 8 * n:]
    k = len(body) // (16 * n) if n else 0
    frames = np.frombuffer(body[:16 * n * k], "<f4").reshape(k, n, 4)
    return hdr, mass, radius, frames


def test_nbs2_writer(nbx, tmp_path):
    import ctypes as C
    L = nbx.lib()
    L.nbx_nbs2_open.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_float, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_void_p)]
    L.nbx_nbs2_write_frame.argtypes = [C.c_void_p, C.c_void_p]
    L.nbx_nbs2_close.argtypes = [C.c_void_p]
    b = nbx.uniform_disc(300)
    b = np.sort(b, order="id")
    path = str(tmp_path / "t.bin")
    w = C.c_void_p()
    assert L.nbx_nbs2_open(path.encode(), 300, 20, 10, 0.05,
                           np.ascontiguousarray(b["mass"]).ctypes.data,
                           np.ascontiguousarray(b["radius"]).ctypes.data,
                           C.byref(w)) == 0
    written = []
    for k in range(2):
        assert L.nbx_nbs2_write_frame(w, b.ctypes.data) == 0
        written.append(b.copy())
        hdr, _, _, frames = read_nbs2(path)
        assert hdr["completed"] == k + 1 and len(frames) == k + 1  # live counter
        b["px"] += 1.0
    assert L.nbx_nbs2_close(w) == 0
    hdr, mass, radius, frames = read_nbs2(path)
    assert hdr["magic"] == b"NBS2" and hdr["n"] == 300 and hdr["frames"] == 3
    assert hdr["completed"] == 2 and np.float32(hdr["dt"]) == np.float32(0.05)
    assert np.array_equal(mass, b["mass"]) and np.array_equal(radius, b["radius"])
    assert np.array_equal(frames[1][:, 0], written[1]["px"])
    assert np.array_equal(frames[0][:, 2], written[0]["vx"])


def test_draw_defaults_are_the_viewers(nbx):
    """DrawSettings defaults (viewer/Renderer.h:14-20); no GPU needed."""
    d = nbx.Draw()
    nbx.lib().nbx_draw_default(nbx.C.byref(d))
    assert (d.mode, d.point_scale, d.min_point_px) == (1, 1.0, 1.5)
    assert abs(d.brightness - 0.6) < 1e-7 and d.speed_max == 60.0


def test_scenario_arguments_checked(nbx):
    with pytest.raises(nbx.NbxError):
        nbx.make_scenario("disc", 0)
    with pytest.raises(nbx.NbxError):
        nbx.make_scenario("two_galaxies", 1)
    assert nbx.lib().nbx_make_scenario(7, 10, 0, None) != 0  # unknown kind
    b = nbx.make_scenario("cold_square", 5000, 2)
    assert np.array_equal(b["id"], np.arange(5000)) and (b["mass"] == 1).all()
    h = 3.0 * np.sqrt(5000)
    assert np.abs(b["px"]).max() <= h and np.abs(b["py"]).max() <= h
    assert nbx.cold_square(5000, 2).tobytes() == b.tobytes()
