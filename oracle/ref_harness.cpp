// ref_harness.cpp -- C entry points around the UNMODIFIED reference sources.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together
// with the reference's own src/Simulation.cpp, src/QuadTree.cpp,
// src/Collision.cpp, src/Utils.cpp and src/naive/NaiveSimulation.cpp (read
// in place, never copied) into
// oracle/_ref/.  It is used to pin the CPU restatement (nbody_oracle.c),
// to write golden fixtures, and as the timed CPU baseline.  Nothing here
// re-implements the reference: every call lands in the reference's code.
#include "Collision.h"
#include "NaiveSimulation.h"
#include "QuadTree.h"
#include "Simulation.h"
#include "Utils.h"
#include "cuda/TreeKernels.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

static_assert(sizeof(Body) == 36, "Body is 36 bytes");

namespace {
std::vector<Body> toVec(const Body *b, std::size_t n) {
  return std::vector<Body>(b, b + n);
}
} // namespace

extern "C" {

int ref_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// uniformDisc(n, seed) -- src/Utils.cpp:6-54.
void ref_uniform_disc(std::size_t n, unsigned seed, Body *out) {
  std::vector<Body> v = uniformDisc(n, seed);
  std::memcpy(out, v.data(), n * sizeof(Body));
}

// The two-disc workload built from the reference's own uniformDisc
// (src/Utils.cpp:6-54) for seeds seed and seed+1: discs of n/2 and n - n/2
// bodies, centres at (-+3R, 0) with R = 5 sqrt(n/2), bulk velocities
// (0, +-f v) with v = sqrt(M_total / (6R)), M_total = 2 (1e6 + n/2), the
// second disc's spin reversed, ids 0..n-1 (the shape of
// viewer/Scenarios.cpp:36-48).  The timed CPU baseline builds its input
// here, so that it maps no product code.
void ref_two_discs(std::size_t n, unsigned seed, float approach, Body *out) {
  const std::size_t half = n / 2;
  const float R = 5.0f * std::sqrt(static_cast<float>(half));
  const float totalMass = 2.0f * (1e6f + static_cast<float>(half));
  const float v = approach * std::sqrt(totalMass / (6.0f * R));
  std::size_t k = 0;
  for (int side = 0; side < 2; ++side) {
    const std::size_t m = side == 0 ? half : n - half;
    const float x = side == 0 ? -3.0f * R : 3.0f * R;
    const float vy = side == 0 ? v : -v;
    for (Body b : uniformDisc(m, seed + side)) {
      if (side == 1) b.vel = b.vel * -1.0f;
      b.pos.x += x;
      b.vel.y += vy;
      b.id = k;
      out[k++] = b;
    }
  }
}

// Body::update for every body (src/Simulation.cpp:44-50).
void ref_iterate(std::size_t n, Body *b, float dt) {
  for (std::size_t i = 0; i < n; ++i) b[i].update(dt);
}

// ::collide (src/Collision.cpp:135).
void ref_collide(std::size_t n, Body *b) {
  std::vector<Body> v = toVec(b, n);
  collide(v);
  std::memcpy(b, v.data(), n * sizeof(Body));
}

// QuadTree(theta, eps, leaf).build + acceleration per body, as
// Simulation::attract (src/Simulation.cpp:18-42).  Reorders b.
void ref_quadtree_forces(std::size_t n, Body *b, float theta, float eps,
                         int leaf) {
  std::vector<Body> v = toVec(b, n);
  QuadTree tree(theta, eps, static_cast<std::size_t>(leaf));
  tree.build(v);
#pragma omp parallel for schedule(dynamic, 128)
  for (std::size_t i = 0; i < n; ++i) v[i].acc = tree.acceleration(v[i].pos, v);
  std::memcpy(b, v.data(), n * sizeof(Body));
}

// `steps` calls of Simulation::step on the given state with the given
// parameters (the public members of Simulation, src/Simulation.h:9-12).
// collisions == 0 replaces step() by iterate(); attract(); as
// CudaSimulation does with collisions off.  Returns ms of the step loop.
double ref_simulate(std::size_t n, Body *b, float dt, float theta, float eps,
                    int leaf, int steps, int collisions) {
  Simulation sim(1);
  sim.bodies = toVec(b, n);
  sim.quadtree = QuadTree(theta, eps, static_cast<std::size_t>(leaf));
  sim.dt = dt;
  const auto t0 = std::chrono::steady_clock::now();
  for (int k = 0; k < steps; ++k) {
    if (collisions) {
      sim.step();
    } else {
      sim.iterate();
      sim.attract();
      sim.frame += 1;
    }
  }
  const auto t1 = std::chrono::steady_clock::now();
  std::memcpy(b, sim.bodies.data(), n * sizeof(Body));
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// NaiveSimulation::attract (NaiveSimulation.cpp:17-57) on the given
// bodies: writes their accelerations.
void ref_naive_attract(std::size_t n, Body *b) {
  NaiveSimulation sim(1);
  sim.bodies = toVec(b, n);
  sim.attract();
  std::memcpy(b, sim.bodies.data(), n * sizeof(Body));
}

// `steps` NaiveSimulation::step() calls (iterate -> collide -> attract);
// returns the wall time in ms.
double ref_naive_simulate(std::size_t n, Body *b, float dt, int steps) {
  NaiveSimulation sim(1);
  sim.bodies = toVec(b, n);
  sim.dt = dt;
  const auto t0 = std::chrono::steady_clock::now();
  for (int k = 0; k < steps; ++k) sim.step();
  const auto t1 = std::chrono::steady_clock::now();
  std::memcpy(b, sim.bodies.data(), n * sizeof(Body));
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// Host compile of the reference's Morton path (TreeKernels.cuh:37-66 with
// the origin/scale of CudaQuadTree.cu:41-44).
void ref_morton(std::size_t n, const float *x, const float *y,
                const float root[3], std::uint64_t *codes) {
  const double x0 = static_cast<double>(root[0]) - 0.5 * root[2];
  const double y0 = static_cast<double>(root[1]) - 0.5 * root[2];
  const double scale = root[2] > 0.0f ? 4294967296.0 / root[2] : 0.0;
  for (std::size_t i = 0; i < n; ++i)
    codes[i] = tree_detail::mortonCode(x[i], y[i], x0, y0, scale);
}

// Host-loop build with the reference's splitNode/sumNode/finishNode
// (TreeKernels.cuh:117-177), driven level by level as buildHostLoop
// (CudaQuadTree.cu:452-498).  Arrays must hold `capacity` nodes.
// Returns node count, or -1 on overflow.  levels_out gets the level count.
int ref_build_tree(std::size_t n, const std::uint64_t *codes, const float *x,
                   const float *y, const float *m, const float root[3],
                   int capacity, float *comX, float *comY, float *mass,
                   float *centerX, float *centerY, float *size, int *children,
                   int *next, int *start, int *end, int *levels_out) {
  using namespace tree_detail;
  NodeArrays t{comX, comY, mass, centerX, centerY, size,
               children, next, start, end};
  if (n == 0) {
    *levels_out = 0;
    return 0;
  }
  initNode(t, 0, root[0], root[1], root[2], 0, 0, static_cast<int>(n));
  std::vector<std::pair<int, int>> levels;
  int lb = 0, le = 1;
  for (int depth = 0; lb < le; ++depth) {
    levels.emplace_back(lb, le);
    int count = le;
    for (int k = lb; k < le; ++k) {
      if (shouldSplit(t, k, depth)) {
        if (count + 4 > capacity) return -1;
        splitNode(t, k, count, depth, codes);
        count += 4;
      }
    }
    if (count == le) break;
    lb = le;
    le = count;
  }
  TreeBodies tb{x, y, m};
  for (auto it = levels.rbegin(); it != levels.rend(); ++it)
    for (int k = it->first; k < it->second; ++k) sumNode(t, k, tb);
  for (int k = 0; k < le; ++k) finishNode(t, k);
  *levels_out = static_cast<int>(levels.size());
  return le;
}

// accelerationAt (TreeKernels.cuh:197-245) for every body.
void ref_tree_forces(std::size_t n, const float *x, const float *y,
                     const float *m, float *comX, float *comY, float *mass,
                     float *centerX, float *centerY, float *size,
                     int *children, int *next, int *start, int *end,
                     float theta, float eps, float *ax, float *ay) {
  using namespace tree_detail;
  NodeArrays t{comX, comY, mass, centerX, centerY, size,
               children, next, start, end};
  TreeBodies tb{x, y, m};
  for (std::size_t i = 0; i < n; ++i)
    accelerationAt(x[i], y[i], t, tb, ax[i], ay[i], theta * theta, eps * eps);
}

} // extern "C"
