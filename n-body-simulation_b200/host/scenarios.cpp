// scenarios.cpp -- initial conditions, on the host.
//
// nbx_uniform_disc restates the reference's uniformDisc (src/Utils.cpp:6-54)
// with the same random stream (std::mt19937 + uniform_real_distribution
// <float>), the same float expressions in the same order and the same
// std::sort by |pos|^2, and is compiled with the reference's flags
// (-Ofast -march=native), so it reproduces the reference's bodies bit for
// bit (checked against the reference's own build in tests).  The two-disc
// and cold-square generators follow viewer/Scenarios.cpp:8-57.
#include "nbx.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

namespace {

struct V2 {
  float x, y;
};
inline V2 operator*(V2 a, float s) { return {a.x * s, a.y * s}; }
inline float mag_sq(V2 a) { return a.x * a.x + a.y * a.y; }

struct Rec {
  V2 pos, vel, acc;
  float mass, radius;
  uint32_t id;
};
static_assert(sizeof(Rec) == sizeof(nbx_body), "36-byte bodies");

std::vector<Rec> disc(uint32_t n, uint32_t seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> unit(0.0f, 1.0f);
  const float inner = 25.0f;
  const float outer = std::sqrt(static_cast<float>(n)) * 5.0f;
  std::vector<Rec> out;
  out.reserve(n);
  if (n == 0) return out;
  out.push_back(Rec{{0.0f, 0.0f}, {0.0f, 0.0f}, {0.0f, 0.0f}, 1e6f, inner, 0u});
  uint32_t next = 1;
  while (out.size() < n) {
    const float angle = unit(rng) * static_cast<float>(M_PI) * 2.0f;
    const float s = std::sin(angle);
    const float c = std::cos(angle);
    const float t = inner / outer;
    const float r = unit(rng) * (1.0f - t * t) + t * t;
    const V2 pos = V2{c, s} * outer * std::sqrt(r);
    const V2 vel = V2{s, -c};
    const float mass = 1.0f;
    out.push_back(Rec{pos, vel, {0.0f, 0.0f}, mass, std::cbrt(mass), next++});
  }
  std::sort(out.begin(), out.end(), [](const Rec &a, const Rec &b) {
    return mag_sq(a.pos) < mag_sq(b.pos);
  });
  float enclosed = 0.0f;
  for (uint32_t i = 0; i < n; ++i) {
    enclosed += out[i].mass;
    if (out[i].pos.x == 0.0f && out[i].pos.y == 0.0f) continue;
    const float v = std::sqrt(enclosed / std::sqrt(mag_sq(out[i].pos)));
    out[i].vel = out[i].vel * v;
  }
  return out;
}

} // namespace

extern "C" int nbx_uniform_disc(uint32_t n, uint32_t seed, nbx_body *out) {
  if (!out && n) return NBX_ERR_ARG;
  const std::vector<Rec> v = disc(n, seed);
  std::copy(v.begin(), v.end(), reinterpret_cast<Rec *>(out));
  return NBX_OK;
}

extern "C" int nbx_two_discs(uint32_t n, uint32_t seed, float approach,
                             nbx_body *out) {
  if (!out && n) return NBX_ERR_ARG;
  const uint32_t half = n / 2;
  const float R = 5.0f * std::sqrt(static_cast<float>(half));
  const float totalMass = 2.0f * (1e6f + static_cast<float>(half));
  const float v = approach * std::sqrt(totalMass / (6.0f * R));
  Rec *o = reinterpret_cast<Rec *>(out);
  uint32_t k = 0;
  for (int side = 0; side < 2; ++side) {
    const uint32_t m = side == 0 ? half : n - half;
    const float x = side == 0 ? -3.0f * R : 3.0f * R;
    const float vy = side == 0 ? v : -v;
    for (Rec b : disc(m, seed + side)) {
      if (side == 1) b.vel = b.vel * -1.0f; // opposite spin
      b.pos.x += x;
      b.vel.y += vy;
      b.id = k;
      o[k++] = b;
    }
  }
  return NBX_OK;
}

extern "C" int nbx_cold_square(uint32_t n, uint32_t seed, nbx_body *out) {
  // the viewer's ColdSquare, built with the viewer's flags (edits.cpp)
  return nbx_make_scenario(NBX_SCENARIO_COLD_SQUARE, n, seed, out);
}

// Instance sizes of the batched ensemble: N_i = round(exp(U(ln lo, ln hi)))
// drawn from mt19937(i) for instance i.
extern "C" int nbx_ensemble_sizes(uint32_t count, uint32_t lo, uint32_t hi,
                                  uint32_t *sizes) {
  if ((count && !sizes) || lo == 0 || hi < lo) return NBX_ERR_ARG;
  for (uint32_t i = 0; i < count; ++i) {
    std::mt19937 rng(i);
    std::uniform_real_distribution<double> u(std::log((double)lo), std::log((double)hi));
    sizes[i] = (uint32_t)std::llround(std::exp(u(rng)));
  }
  return NBX_OK;
}
