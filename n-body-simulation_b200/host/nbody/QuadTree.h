// QuadTree.h -- the reference's QuadTree interface (src/QuadTree.h:72-86),
// computed on the GPU.  build() reorders `bodies` (into Morton order, where
// the reference partitions in place) and evaluates every body's
// acceleration in one traversal; acceleration() then returns the cached
// value for a body position, or runs the GPU traversal for any other point.
#pragma once
#include "Body.h"
#include <cstddef>
#include <memory>
#include <vector>

struct NbxContext; // a lazily created nbx handle

class QuadTree {
public:
  static constexpr int ROOT = 0;

  QuadTree(float theta, float epsilon, std::size_t leafCapacity);
  QuadTree(const QuadTree &o);
  QuadTree &operator=(const QuadTree &o);
  ~QuadTree();

  void build(std::vector<Body> &bodies);
  Vec2 acceleration(const Vec2 &pos, const std::vector<Body> &bodies) const;

  float theta() const { return theta_; }
  float epsilon() const { return epsilon_; }
  std::size_t leafCapacity() const { return leaf_; }

private:
  float theta_, epsilon_;
  std::size_t leaf_;
  std::unique_ptr<NbxContext> ctx_;
};
