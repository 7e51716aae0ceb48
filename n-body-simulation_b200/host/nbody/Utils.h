// Utils.h -- the reference's initial conditions (src/Utils.h:6-9).
#pragma once
#include "Body.h"
#include <cstddef>
#include <vector>

std::vector<Body> uniformDisc(std::size_t n, unsigned seed = 0);
