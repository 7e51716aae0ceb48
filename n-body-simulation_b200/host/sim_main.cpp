// sim_b200 -- the reference's command line (src/Main.cpp:65-82,
// src/cuda/MainCuda.cu:22-40) on the B200 path:
//
//   sim_b200 <n_bodies> <total_steps> <output_every> [output_path] [--key=value ...]
//
// Same initial state (uniformDisc(n, 0)), same defaults (dt 0.05, theta 1,
// epsilon 1, leaf 16, collisions on), same NBS2 output (header, mass and
// radius in id order, frames of {x, y, vx, vy} in id order, live
// completed_frames) and the same stderr summary lines, so load_sim.py and
// cluster/times.sh read its output unchanged.  The state stays on the GPU;
// frames are copied back in id order only when written (as sim_cuda).
// Optional trailing flags: --theta= --eps= --dt= --leaf= --collisions=0/1
// --scenario=disc|two|cold --seed= --exact=0/1 --naive=0/1 (the direct
// all-pairs law of sim_naive / sim_cuda_naive, MainNaive.cpp).
#include "nbx.h"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

namespace {
bool flag(const std::string &a, const char *key, std::string &v) {
  const std::string k = std::string("--") + key + "=";
  if (a.compare(0, k.size(), k) != 0) return false;
  v = a.substr(k.size());
  return true;
}
int fail(const char *what, nbx_handle *h) {
  std::cerr << what << ": " << (h ? nbx_last_error(h) : "error") << "\n";
  return 1;
}
} // namespace

int main(int argc, char **argv) {
  std::vector<std::string> pos;
  nbx_params p;
  nbx_params_default(&p);
  std::string scenario = "disc", v;
  uint32_t seed = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a.rfind("--", 0) != 0) {
      pos.push_back(a);
      continue;
    }
    if (flag(a, "theta", v)) p.theta = std::stof(v);
    else if (flag(a, "eps", v)) p.epsilon = std::stof(v);
    else if (flag(a, "dt", v)) p.dt = std::stof(v);
    else if (flag(a, "leaf", v)) p.leaf_capacity = std::stoi(v);
    else if (flag(a, "collisions", v)) p.collisions = std::stoi(v);
    else if (flag(a, "exact", v)) p.exact_math = std::stoi(v);
    else if (flag(a, "naive", v)) p.force_law = std::stoi(v) ? 1 : 0;
    else if (flag(a, "scenario", v)) scenario = v;
    else if (flag(a, "seed", v)) seed = (uint32_t)std::stoul(v);
    else {
      std::cerr << "unknown option " << a << "\n";
      return 1;
    }
  }
  if (pos.size() != 3 && pos.size() != 4) {
    std::cerr << "Usage: " << argv[0]
              << " <n_bodies> <total_steps> <output_every> [output_path]\n"
              << "  (no output_path: run without writing any output)\n";
    return 1;
  }
  const uint32_t n = (uint32_t)std::stoul(pos[0]);
  const uint32_t totalSteps = (uint32_t)std::stoul(pos[1]);
  const uint32_t every = (uint32_t)std::stoul(pos[2]);
  const bool writeOutput = pos.size() == 4;
  if (every == 0) {
    std::cerr << "output_every must be >= 1\n";
    return 1;
  }

  std::vector<nbx_body> bodies(n);
  int rc = scenario == "two"    ? nbx_two_discs(n, seed, 0.2f, bodies.data())
           : scenario == "cold" ? nbx_cold_square(n, seed, bodies.data())
                                : nbx_uniform_disc(n, seed, bodies.data());
  if (rc != NBX_OK) {
    std::cerr << "unknown scenario\n";
    return 1;
  }
  nbx_handle *h = nullptr;
  if (nbx_create(&p, 1, &n, &h) != NBX_OK) return fail("nbx_create", h);
  if (nbx_upload_bodies(h, bodies.data(), n) != NBX_OK) return fail("upload", h);

  nbx_nbs2 *out = nullptr;
  uint32_t completed = 0;
  // frame 0 (and mass / radius) in id order, as Main.cpp's first sortById
  if (nbx_download_bodies(h, bodies.data(), n, 1) != NBX_OK) return fail("download", h);
  if (writeOutput) {
    std::vector<float> mass(n), radius(n);
    for (uint32_t i = 0; i < n; ++i) {
      mass[i] = bodies[i].mass;
      radius[i] = bodies[i].radius;
    }
    if (nbx_nbs2_open(pos[3].c_str(), n, totalSteps, every, p.dt, mass.data(),
                      radius.data(), &out) != NBX_OK) {
      std::cerr << "Failed to open output file: " << pos[3] << "\n";
      return 1;
    }
    if (nbx_nbs2_write_frame(out, bodies.data()) != NBX_OK) return fail("write", h);
    ++completed;
  }

  // compute time = the stepping alone, frame output excluded (Main.cpp:167-186)
  double computeMs = 0.0;
  const auto loopStart = std::chrono::steady_clock::now();
  uint32_t step = 0;
  while (step < totalSteps) {
    uint32_t chunk = totalSteps - step;
    if (writeOutput) chunk = std::min(chunk, every - step % every);
    const auto t0 = std::chrono::steady_clock::now();
    if (nbx_step(h, chunk) != NBX_OK || nbx_sync(h) != NBX_OK) return fail("step", h);
    computeMs += std::chrono::duration<double, std::milli>(
                     std::chrono::steady_clock::now() - t0)
                     .count();
    step += chunk;
    if (writeOutput && step % every == 0) {
      // device path: id-order scatter on the GPU, copy and file write
      // overlapped with the following steps
      if (nbx_nbs2_record(h, out) != NBX_OK) return fail("record frame", h);
      ++completed;
    }
  }
  if (out && nbx_nbs2_flush(h) != NBX_OK) return fail("write", h);
  const double loopMs = std::chrono::duration<double, std::milli>(
                            std::chrono::steady_clock::now() - loopStart)
                            .count();
  if (out && nbx_nbs2_close(out) != NBX_OK) {
    std::cerr << "Error while writing output file: " << pos[3] << "\n";
    return 1;
  }
  nbx_destroy(h);
  std::cerr << "Done. n=" << n << " steps=" << totalSteps << " output_every=" << every
            << " frames_written=" << completed << " (expected "
            << (writeOutput ? 1 + totalSteps / every : 0) << ") -> "
            << (writeOutput ? pos[3] : std::string("(no output)")) << "\n";
  std::cerr << "BH: n=" << n << " threads=1 steps=" << totalSteps
            << " total_time=" << loopMs << " ms avg_step="
            << (totalSteps ? loopMs / totalSteps : 0.0) << " ms compute_time=" << computeMs
            << " ms avg_compute_step=" << (totalSteps ? computeMs / totalSteps : 0.0)
            << " ms output_time=" << (loopMs - computeMs) << " ms\n";
  return 0;
}
