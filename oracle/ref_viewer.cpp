// ref_viewer.cpp -- C entry points around the UNMODIFIED viewer scenario
// code of the reference (src/viewer/Scenarios.cpp), for pinning the
// product's nbx_make_scenario / nbx_add_* (host/edits.cpp).
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile builds it into
// oracle/_ref/libref_viewer.so as the reference's CMakeLists.txt builds the
// viewer: Scenarios.cpp and this file with -O2, Utils.cpp (uniformDisc)
// with -Ofast -ffast-math -march=native.  Every call lands in the
// reference's code.
#include "Scenarios.h"

#include <cstring>
#include <vector>

static_assert(sizeof(Body) == 36, "Body is 36 bytes");

extern "C" {

// makeScenario(kind, n, seed) into out, which must hold what it returns
// (n bodies, except for sizes where uniformDisc(0) adds a central body).
std::size_t refv_make_scenario(int kind, std::size_t n, unsigned seed, Body *out,
                               std::size_t cap) {
  const std::vector<Body> b = makeScenario(static_cast<Scenario>(kind), n, seed);
  if (b.size() <= cap) std::memcpy(out, b.data(), b.size() * sizeof(Body));
  return b.size();
}

// addHeavyBody on a copy of in[n]; out must hold n + 1.
std::size_t refv_add_heavy_body(const Body *in, std::size_t n, float x, float y,
                                float mass, Body *out) {
  std::vector<Body> b(in, in + n);
  addHeavyBody(b, x, y, mass);
  std::memcpy(out, b.data(), b.size() * sizeof(Body));
  return b.size();
}

// addCluster on a copy of in[n]; out must hold n + count.
std::size_t refv_add_cluster(const Body *in, std::size_t n, float x, float y,
                             float vx, float vy, std::size_t count, unsigned seed,
                             Body *out) {
  std::vector<Body> b(in, in + n);
  addCluster(b, x, y, vx, vy, count, seed);
  std::memcpy(out, b.data(), b.size() * sizeof(Body));
  return b.size();
}

} // extern "C"
