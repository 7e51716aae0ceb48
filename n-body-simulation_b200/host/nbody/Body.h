// Body.h -- the reference's body record (src/Body.h:5-23): 36 bytes, the
// same layout as nbx_body, so a std::vector<Body> goes through the C ABI
// without conversion.
#pragma once
#include "Vec2.h"
#include <cstdint>

struct Body {
  Vec2 pos;
  Vec2 vel;
  Vec2 acc;
  float mass;
  float radius;
  std::uint32_t id;

  Body(const Vec2 &p, const Vec2 &v, float m, float r, std::uint32_t i = 0)
      : pos(p), vel(v), acc(0.0f, 0.0f), mass(m), radius(r), id(i) {}

  void update(float dt) {
    vel += acc * dt;
    pos += vel * dt;
  }
};
static_assert(sizeof(Body) == 36, "Body must stay 36 bytes");
