// edits.cpp -- the viewer's initial conditions and state edits as C calls,
// so scenarios can be injected into a handle without a GUI:
// makeScenario, renumber, addHeavyBody and addCluster
// (src/viewer/Scenarios.cpp:8-86, Scenarios.h:1-23).  A caller edits a host
// copy of the bodies (nbx_download_bodies), then nbx_reset()s the handle
// with it, as the viewer's editBodies does (viewer/main.cpp:122-129).
//
// Built with the viewer's own flags (-O2, no -ffast-math, no -march), so
// the float arithmetic rounds as the viewer's build does; uniformDisc comes
// from nbx_uniform_disc, which is built with the reference's -Ofast like
// the reference's own Utils.cpp.
#include "nbx.h"

#include <cmath>
#include <cstring>
#include <random>

namespace {

struct Rec {
  float px, py, vx, vy, ax, ay, mass, radius;
  uint32_t id;
};
static_assert(sizeof(Rec) == sizeof(nbx_body), "36-byte bodies");

// uniformDisc(n, seed) moved to (x, y) with bulk velocity (vx, vy); reverse
// flips its rotation (appendDisc, Scenarios.cpp:8-19).
int append_disc(Rec *out, uint32_t n, uint32_t seed, float x, float y, float vx,
                float vy, bool reverse) {
  if (n == 0) return NBX_OK;
  int rc = nbx_uniform_disc(n, seed, reinterpret_cast<nbx_body *>(out));
  if (rc != NBX_OK) return rc;
  for (uint32_t i = 0; i < n; ++i) {
    Rec &b = out[i];
    if (reverse) {
      b.vx = b.vx * -1.0f;
      b.vy = b.vy * -1.0f;
    }
    b.px += x;
    b.py += y;
    b.vx += vx;
    b.vy += vy;
  }
  return NBX_OK;
}

} // namespace

extern "C" void nbx_renumber(nbx_body *bodies, size_t n) {
  Rec *b = reinterpret_cast<Rec *>(bodies);
  for (size_t i = 0; i < n; ++i) b[i].id = static_cast<uint32_t>(i);
}

extern "C" int nbx_make_scenario(int kind, uint32_t n, uint32_t seed, nbx_body *out) {
  if (!out && n) return NBX_ERR_ARG;
  // uniformDisc(0) still returns its central body, so the reference's
  // makeScenario gives more bodies than asked for a disc of 0 or two
  // galaxies of fewer than 2; those sizes are rejected here
  if ((kind == NBX_SCENARIO_DISC && n < 1) || (kind == NBX_SCENARIO_TWO_GALAXIES && n < 2))
    return NBX_ERR_ARG;
  Rec *o = reinterpret_cast<Rec *>(out);
  int rc = NBX_OK;
  switch (kind) {
  case NBX_SCENARIO_DISC:
    rc = nbx_uniform_disc(n, seed, out);
    break;
  case NBX_SCENARIO_TWO_GALAXIES: {
    // two discs on a glancing course, rotating opposite ways
    const uint32_t half = n / 2;
    const float radius = 5.0f * std::sqrt(static_cast<float>(half));
    const float sep = 2.5f * radius;
    const float totalMass = 2.0f * (1e6f + static_cast<float>(half));
    const float v = 0.3f * std::sqrt(totalMass / sep);
    rc = append_disc(o, half, seed, -sep / 2, -radius / 3, v, 0.0f, false);
    if (rc == NBX_OK)
      rc = append_disc(o + half, n - half, seed + 1, sep / 2, radius / 3, -v, 0.0f, true);
    break;
  }
  case NBX_SCENARIO_COLD_SQUARE: {
    std::mt19937 rng(seed);
    const float half = 3.0f * std::sqrt(static_cast<float>(n));
    std::uniform_real_distribution<float> coord(-half, half);
    for (uint32_t i = 0; i < n; ++i) {
      // the reference passes both draws to one constructor call; g++
      // evaluates those arguments last to first, so y is drawn before x
      const float y = coord(rng);
      const float x = coord(rng);
      o[i] = Rec{x, y, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 1.0f, 0u};
    }
    break;
  }
  default:
    return NBX_ERR_ARG;
  }
  if (rc != NBX_OK) return rc;
  nbx_renumber(out, n);
  return NBX_OK;
}

extern "C" size_t nbx_add_heavy_body(nbx_body *bodies, size_t n, float x, float y,
                                     float mass) {
  if (!bodies) return n;
  // same density as the central body: radius grows with the cube root
  const float radius = 25.0f * std::cbrt(mass / 1e6f);
  reinterpret_cast<Rec *>(bodies)[n] =
      Rec{x, y, 0.0f, 0.0f, 0.0f, 0.0f, mass, std::fmax(radius, 1.0f),
          static_cast<uint32_t>(n)};
  return n + 1;
}

extern "C" size_t nbx_add_cluster(nbx_body *bodies, size_t n, float x, float y, float vx,
                                  float vy, size_t count, uint32_t seed) {
  if (!bodies) return n;
  Rec *b = reinterpret_cast<Rec *>(bodies);
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> unit(0.0f, 1.0f);
  const float spread = 2.0f * std::sqrt(static_cast<float>(count));
  for (size_t i = 0; i < count; ++i) {
    const float a = unit(rng) * 6.2831853f;
    const float r = spread * std::sqrt(unit(rng));
    b[n + i] = Rec{x + r * std::cos(a), y + r * std::sin(a), vx, vy, 0.0f, 0.0f,
                   1.0f, 1.0f, static_cast<uint32_t>(n + i)};
  }
  return n + count;
}
