// Collision.h -- the reference's collide() (src/Collision.h:9): every
// overlapping box pair resolved in sorted-pair order, on the GPU.
#pragma once
#include "Body.h"
#include <vector>

void collide(std::vector<Body> &bodies);
