"""The reference-facing layer on the GPU: the sim_b200 command line (NBS2
output) and the C++ Simulation / QuadTree / collide interfaces."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ORACLE, PKG, ROOT, rel_err, same_bits
from test_host import read_nbs2

pytestmark = pytest.mark.gpu
SIM = os.path.join(PKG, "bin", "sim_b200")


def test_cli_nbs2(nbx, oracle, tmp_path):
    out = str(tmp_path / "b200.bin")
    r = subprocess.run([SIM, "2000", "10", "5", out], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "BH: n=2000" in r.stderr and "frames_written=3 (expected 3)" in r.stderr
    hdr, mass, radius, frames = read_nbs2(out)
    assert hdr["completed"] == 3 and frames.shape == (3, 2000, 4)
    ref0 = np.sort(nbx.uniform_disc(2000), order="id")
    assert same_bits(mass, ref0["mass"]) and same_bits(radius, ref0["radius"])
    assert same_bits(frames[0][:, 0], ref0["px"]) and same_bits(frames[0][:, 3], ref0["vy"])
    o = np.sort(oracle.step(nbx.uniform_disc(2000), steps=10), order="id")
    e = rel_err(frames[2][:, 0], frames[2][:, 1], o["px"], o["py"])
    assert np.median(e) < 1e-5 and e.max() < 1e-3
    # the reference's own command line, where its build is present
    ref_sim = os.path.join(ORACLE, "_ref", "sim")
    if os.path.exists(ref_sim):
        rp = str(tmp_path / "ref.bin")
        r = subprocess.run([ref_sim, "2000", "10", "5", rp], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0
        rh, rm, rr, rf = read_nbs2(rp)
        assert same_bits(rm, mass) and same_bits(rf[0], frames[0])
        e = rel_err(frames[2][:, 0], frames[2][:, 1], rf[2][:, 0], rf[2][:, 1])
        assert np.median(e) < 1e-4 and e.max() < 1e-3


SHIM_CHECK = r'''
#include "nbody/Collision.h"
#include "nbody/Simulation.h"
#include "nbody/Utils.h"
#include "nbody_oracle.h"
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
static double relerr(Vec2 a, float bx, float by) {
  double dx = a.x - bx, dy = a.y - by;
  return std::sqrt(dx * dx + dy * dy) / std::fmax(std::sqrt((double)bx * bx + (double)by * by), 1e-30);
}
int main() {
  int fails = 0;
  // Simulation: 10 steps against the oracle's step
  Simulation sim(3000);
  std::vector<orc_body> o(sim.bodies.size());
  std::memcpy(o.data(), sim.bodies.data(), o.size() * sizeof(orc_body));
  for (int k = 0; k < 10; ++k) { sim.step(); orc_step(o.size(), o.data(), 0.05f, 1.0f, 1.0f, 16, 1); }
  double worst = 0;
  std::vector<orc_body> byId(o.size());
  for (auto &b : o) byId[b.id] = b;
  for (auto &b : sim.bodies) worst = std::fmax(worst, relerr(b.pos, byId[b.id].px, byId[b.id].py));
  std::printf("[%s] Simulation 10 steps max rel err %.3g\n", worst < 1e-3 ? "PASS" : "FAIL", worst);
  fails += worst >= 1e-3;
  if (sim.frame != 10) { std::printf("[FAIL] frame\n"); ++fails; }
  // QuadTree: build + acceleration against the partition tree restatement
  std::vector<Body> bodies = uniformDisc(5000);
  std::vector<orc_body> q(bodies.size());
  std::memcpy(q.data(), bodies.data(), q.size() * sizeof(orc_body));
  orc_quadtree_forces(q.size(), q.data(), 1.0f, 1.0f, 16);
  std::vector<Vec2> want(q.size());
  for (auto &b : q) want[b.id] = Vec2(b.ax, b.ay);
  QuadTree tree(1.0f, 1.0f, 16);
  tree.build(bodies);
  double tmax = 0;
  for (auto &b : bodies) tmax = std::fmax(tmax, relerr(tree.acceleration(b.pos, bodies), want[b.id].x, want[b.id].y));
  std::printf("[%s] QuadTree acceleration max rel err %.3g\n", tmax < 1e-3 ? "PASS" : "FAIL", tmax);
  fails += tmax >= 1e-3;
  Vec2 off(bodies[7].pos.x + 0.25f, bodies[7].pos.y - 0.5f);
  Vec2 a = tree.acceleration(off, bodies);
  const bool finite = std::isfinite(a.x) && std::isfinite(a.y) && (a.x != 0 || a.y != 0);
  std::printf("[%s] acceleration at a free point\n", finite ? "PASS" : "FAIL");
  fails += !finite;
  // collide(): bit-exact against the sequential restatement
  std::vector<Body> st = sim.bodies;
  for (int k = 0; k < 200; ++k) sim.step();
  sim.iterate();
  st = sim.bodies;
  std::vector<orc_body> c(st.size());
  std::memcpy(c.data(), st.data(), c.size() * sizeof(orc_body));
  long long pairs = orc_collide(c.size(), c.data());
  collide(st);
  const bool same = std::memcmp(st.data(), c.data(), c.size() * sizeof(orc_body)) == 0;
  std::printf("[%s] collide vs sequential resolve (%lld pairs)\n", same && pairs > 0 ? "PASS" : "FAIL", pairs);
  fails += !(same && pairs > 0);
  std::printf("%s\n", fails ? "FAILED" : "ALL PASSED");
  return fails ? 1 : 0;
}
'''


def test_cpp_interfaces(tmp_path):
    src = tmp_path / "shim_check.cpp"
    src.write_text(SHIM_CHECK)
    exe = str(tmp_path / "shim_check")
    lib = os.path.join(PKG, "lib")
    subprocess.run(["make", "-s", "-C", ORACLE, "oracle"], check=True)
    subprocess.run(["g++", "-std=c++17", "-O2", str(src), "-I", os.path.join(PKG, "host"),
                    "-I", ORACLE, "-L", lib, "-lnbody_b200", "-lnbx", "-L", ORACLE,
                    "-loracle", f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{ORACLE}", "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
