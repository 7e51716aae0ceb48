// Simulation.h -- the reference's Simulation (src/Simulation.h:7-20): same
// public members and methods; step() = iterate -> collide -> attract runs on
// the GPU.  `bodies` stays a host vector owned by the caller, so every call
// uploads it and downloads the result (the drop-in contract); a driver that
// keeps the state on the device uses the C ABI (nbx.h) directly.
#pragma once
#include "Body.h"
#include "QuadTree.h"
#include <cstddef>
#include <memory>
#include <vector>

class Simulation {
public:
  float dt;
  std::size_t frame;
  std::vector<Body> bodies;
  QuadTree quadtree;

  explicit Simulation(std::size_t n);
  ~Simulation();

  void step();
  void attract();
  void iterate();
  void collide();

private:
  std::unique_ptr<NbxContext> ctx_;
};
