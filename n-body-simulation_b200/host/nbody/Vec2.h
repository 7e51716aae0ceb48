// Vec2.h -- the reference's 2-D float vector value type (src/Vec2.h), kept
// identical so that code written against the reference's Simulation /
// QuadTree / Collision interfaces compiles unchanged against this library.
#pragma once
#include <cmath>

struct Vec2 {
  float x, y;
  Vec2() : x(0.0f), y(0.0f) {}
  Vec2(float x_, float y_) : x(x_), y(y_) {}
  Vec2 operator+(const Vec2 &o) const { return {x + o.x, y + o.y}; }
  Vec2 operator-(const Vec2 &o) const { return {x - o.x, y - o.y}; }
  Vec2 operator*(float s) const { return {x * s, y * s}; }
  Vec2 operator/(float s) const { return {x / s, y / s}; }
  Vec2 &operator+=(const Vec2 &o) { x += o.x; y += o.y; return *this; }
  Vec2 &operator-=(const Vec2 &o) { x -= o.x; y -= o.y; return *this; }
  Vec2 &operator*=(float s) { x *= s; y *= s; return *this; }
  Vec2 &operator/=(float s) { x /= s; y /= s; return *this; }
  bool operator==(const Vec2 &o) const { return x == o.x && y == o.y; }
  bool operator!=(const Vec2 &o) const { return !(*this == o); }
  float magSq() const { return x * x + y * y; }
  float mag() const { return std::sqrt(magSq()); }
  float dot(const Vec2 &o) const { return x * o.x + y * o.y; }
  static Vec2 zero() { return Vec2(0.0f, 0.0f); }
  static Vec2 one() { return Vec2(1.0f, 1.0f); }
};
inline Vec2 operator*(float s, const Vec2 &v) { return v * s; }
