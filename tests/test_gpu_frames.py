"""Device-path NBS2 frames (nbx_nbs2_record): id-order scatter on the GPU,
copy and file write overlapped with the following steps.  The file must
hold exactly the frames an id-order download gives at the same points."""
import numpy as np
import pytest

from conftest import same_bits
from test_host import read_nbs2

pytestmark = pytest.mark.gpu

POINTS = [0, 1, 3, 4, 10, 11, 25]  # steps after which a frame is recorded


def expected_frames(nbx, bodies, **kw):
    sim = nbx.Simulation(bodies, **kw)
    out, done = [], 0
    for p in POINTS:
        if p > done:
            sim.step(p - done)
            done = p
        d = sim.download(id_order=True)
        out.append(np.stack([d["px"], d["py"], d["vx"], d["vy"]], axis=1))
    sim.close()
    return np.stack(out)


@pytest.mark.parametrize("kw", [dict(theta=0.5), dict(force_law=1)])
def test_recorded_frames_equal_downloads(nbx, tmp_path, kw):
    b = nbx.uniform_disc(20000)
    exp = expected_frames(nbx, b, **kw)
    sim = nbx.Simulation(b, **kw)
    d0 = sim.download(id_order=True)
    path = tmp_path / "run.bin"
    w = nbx.Nbs2Writer(path, len(b), POINTS[-1], 1, 0.05, d0["mass"], d0["radius"])
    done = 0
    for p in POINTS:  # no synchronisation between steps and records
        if p > done:
            sim.step(p - done)
            done = p
        sim.nbs2_record(w)
    sim.nbs2_flush()
    w.close()
    hdr, mass, radius, frames = read_nbs2(path)
    assert hdr["completed"] == len(POINTS)
    assert same_bits(mass, d0["mass"]) and same_bits(radius, d0["radius"])
    assert same_bits(frames, exp)
    sim.close()


def test_record_then_reset_and_ensemble_rejected(nbx, tmp_path):
    b = nbx.uniform_disc(5000)
    sim = nbx.Simulation(b)
    d0 = sim.download(id_order=True)
    w = nbx.Nbs2Writer(tmp_path / "a.bin", len(b), 2, 1, 0.05, d0["mass"], d0["radius"])
    sim.nbs2_record(w)
    sim.step(1)
    sim.nbs2_record(w)
    sim.reset(nbx.uniform_disc(3000, 2))  # writes the pending frames first
    w.close()
    hdr, _, _, frames = read_nbs2(tmp_path / "a.bin")
    assert hdr["completed"] == 2 and frames.shape == (2, 5000, 4)
    sim.step(1)  # the handle works at its new size
    assert len(sim.download()) == 3000
    sim.close()
    h = nbx.Handle([100, 200])
    h.upload(np.concatenate([nbx.uniform_disc(100), nbx.uniform_disc(200, 1)]))
    w = nbx.Nbs2Writer(tmp_path / "b.bin", 300, 1, 1, 0.05, np.ones(300), np.ones(300))
    with pytest.raises(nbx.NbxError):
        h.nbs2_record(w)
    w.close()
    h.close()
