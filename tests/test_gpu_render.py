"""Headless splat renderer (nbx_render) against its C restatement in the
oracle: the same per-pixel float operations in the same draw order, so the
images are bit-identical; the body statistics to FP64-sum tolerance."""
import numpy as np
import pytest

from conftest import same_bits

pytestmark = pytest.mark.gpu


def fit(b, width, height):
    span = max(float(np.ptp(b["px"])), float(np.ptp(b["py"])), 1.0) * 1.1
    return (float(b["px"].mean()), float(b["py"].mean())), min(width, height) / span


CASES = [
    # (bodies, width, height, zoom): zoom > 1 gives points of many pixels
    ("disc2000", 320, 240, 1.0),
    ("disc3000_zoom", 256, 256, 12.0),
    ("stepped20000", 641, 479, 1.0),
]


def bodies(nbx, name):
    if name == "disc2000":
        return nbx.uniform_disc(2000)
    if name == "disc3000_zoom":
        return nbx.uniform_disc(3000, 1)
    sim = nbx.Simulation(nbx.uniform_disc(20000), theta=0.5)
    sim.step(20)
    b = sim.download()  # Morton order: the draw order of a running handle
    sim.close()
    return b


@pytest.mark.parametrize("name,w,h,zoom", CASES)
@pytest.mark.parametrize("mode", ["glow", "speed"])
def test_render_bit_identical(nbx, oracle, name, w, h, zoom, mode):
    b = bodies(nbx, name)
    centre, scale = fit(b, w, h)
    scale *= zoom
    sim = nbx.Simulation(b)
    img, st = sim.render(w, h, centre, scale, mode=mode, speed_max=30.0)
    ref, rst = oracle.render(b, w, h, centre, scale, mode=1 if mode == "glow" else 0,
                             speed_max=30.0)
    assert same_bits(img, ref), int((img != ref).sum())
    assert (img[..., 3] > 1.0).any() if mode == "glow" else True  # splats landed
    assert st["max_speed"] == rst[2]
    for k, i in (("com_x", 0), ("com_y", 1)):
        assert abs(st[k] - rst[i]) <= 1e-5 * max(1.0, abs(rst[i]))
    assert st == sim.body_stats()
    sim.close()


def test_render_offscreen_nan_and_empty_image_parts(nbx, oracle):
    b = nbx.uniform_disc(1000)
    b["px"][:10] += 1e7          # far off screen
    b["py"][10:12] = np.nan     # never drawn
    sim = nbx.Simulation(b, collisions=0)
    img, _ = sim.render(200, 100, (0.0, 0.0), 0.05, mode="speed")
    ref, _ = oracle.render(b, 200, 100, (0.0, 0.0), 0.05, mode=0)
    assert same_bits(img, ref)
    sim.close()


def test_render_rejects_oversized_work(nbx):
    sim = nbx.Simulation(nbx.uniform_disc(20000))
    with pytest.raises(nbx.NbxError):  # every point covers the 4096^2 image:
        # 20000 bodies x 65536 tiles > 2^30 (tile, body) pairs
        sim.render(4096, 4096, (0.0, 0.0), 0.1, point_scale=1e5)
    with pytest.raises(nbx.NbxError):
        sim.render(0, 10)
    img, _ = sim.render(64, 64, (0.0, 0.0), 1e-3)  # still usable afterwards
    assert img.shape == (64, 64, 4)
    sim.close()
